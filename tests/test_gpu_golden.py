"""GPU: the golden vectors of the reference's own tests, through the C ABI, every entry point.

Bit-exact: every path returns the reference's value in the arithmetic of its precision (the
reference's tests allow 1e-5 / 1e-7; these checks are equality).
"""

import os

import numpy as np
import pytest

import ssdf_b200 as S
from conftest import golden_mesh, load_golden_json

pytestmark = pytest.mark.gpu


class env:
    def __init__(self, **kv):
        self.kv = kv

    def __enter__(self):
        self.old = {k: os.environ.get(k) for k in self.kv}
        for k, v in self.kv.items():
            os.environ[k] = str(v)

    def __exit__(self, *a):
        for k, v in self.old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


SELECT_MODES = [dict(), dict(SSDF_USE_BVH=0), dict(SSDF_USE_BVH=0, SSDF_USE_CELL_LIST=0),
                dict(SSDF_USE_BVH=0, SSDF_CELL_VALIDATE=1), dict(SSDF_B200_PRECISION="f64"),
                dict(SSDF_B200_PRECISION="f32x"), dict(SSDF_B200_LEAF=1), dict(SSDF_B200_LEAF=16)]


@pytest.mark.parametrize("mode", SELECT_MODES, ids=lambda m: ",".join(f"{k}={v}" for k, v in m.items()) or "default")
def test_single_triangle_float(mode):
    g = load_golden_json()["ssdf_test"]
    mesh = golden_mesh(g, np.float32)
    pts = np.array([g["x"], g["y"], g["z"]], dtype=np.float32)
    init = np.full(5, g["out_init"], np.float32)
    with env(**mode):
        out = S.edf_select(pts, mesh, out=init, dtype=np.float32)
    assert np.array_equal(out, np.array(g["edf_select"], np.float32))
    assert np.all(np.abs(out - np.array(g["brute"], np.float32)) < g["tolerance"])


@pytest.mark.parametrize("mode", SELECT_MODES, ids=lambda m: ",".join(f"{k}={v}" for k, v in m.items()) or "default")
def test_brute_force_double(mode):
    g = load_golden_json()["ssdf_brute_force"]
    mesh = golden_mesh(g)
    pts = np.array([g["x"], g["y"], g["z"]])
    with env(**mode):
        out = S.edf_select(pts, mesh, out=np.full(20, g["out_init"]))
    assert np.array_equal(out, np.array(g["edf"]))
    assert np.max(np.abs(out - np.array(g["brute"]))) <= g["tolerance"]


def test_every_entry_point_on_the_brute_force_vectors():
    g = load_golden_json()["ssdf_brute_force"]
    mesh = golden_mesh(g)
    pts = np.array([g["x"], g["y"], g["z"]])
    init = np.full(20, g["out_init"])
    want = np.array(g["edf"])
    assert np.array_equal(S.edf(pts, mesh, out=init), want)
    assert np.array_equal(S.edf_celllist(pts, mesh, out=init), want)
    assert np.array_equal(S.edf_bvh(pts, mesh, out=init), want)
    with env(SSDF_B200_PRECISION="f64"):
        assert np.array_equal(S.edf_bvh(pts, mesh, out=init), want)
    d, tri = S.edf_index(pts, mesh, out=init)
    assert np.array_equal(d, want) and np.all(tri >= 0)
    # <float, double>: double result of the float-rounded inputs
    got = S.edf_bvh(pts, mesh, out=init, gdtype=np.float32, tdtype=np.float64)
    assert np.max(np.abs(got - want)) < 1e-6
