"""The command-line driver ssdf_sdf (drivers/sdf.exe.cpp's arguments, raw files and environment).

On CPU: usage and the file checks, which fail before any device work. On the GPU: the distance to
the union of two surfaces, bitwise the oracle's edf chained over the surfaces (the driver's in/out
`out`), for the default float arithmetic, SSDF_DOUBLE_PRECISION, SSDF_INPUT_SDF,
SSDF_INIT_WITH_VOLUME_BOX and the SSDF_USE_BVH=0 dispatch.
"""

import os
import subprocess

import numpy as np
import pytest

import oracle
from conftest import ROOT
from ssdf_b200 import workloads as W

CLI = os.path.join(ROOT, "ssdf_b200", "_lib", "ssdf_sdf")


def write_surface(folder, mesh):
    os.makedirs(folder, exist_ok=True)
    v = mesh.vertices.astype(np.float32)
    for a, name in enumerate("xyz"):
        v[:, a].tofile(os.path.join(folder, f"{name}.float32"))
    for a in range(3):
        mesh.triangles[:, a].astype(np.int32).tofile(os.path.join(folder, f"i{a}.int32"))
    return W.Mesh(v.astype(np.float64), mesh.triangles.astype(np.int32))  # the float surface, exactly


def write_points(folder, pts):
    os.makedirs(folder, exist_ok=True)
    p = pts.astype(np.float32)
    for a, name in enumerate("xyz"):
        p[a].tofile(os.path.join(folder, f"{name}.float32"))
    return p


def run(args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([CLI, *args], capture_output=True, text=True, env=e, timeout=300)


def test_usage_and_file_checks(tmp_path):
    assert os.path.exists(CLI), "build the library first (python -m ssdf_b200.build)"
    r = run([])
    assert r.returncode == 1 and "Usage" in r.stderr
    surf = tmp_path / "s"
    write_surface(str(surf), W.icosphere(1))
    r = run([str(surf), str(tmp_path / "missing"), str(tmp_path / "out.raw")])
    assert r.returncode == 1 and "Cannot open" in r.stderr
    np.zeros(5, np.float32).tofile(str(surf / "y.float32"))  # ragged coordinates
    r = run([str(surf), str(tmp_path / "missing"), str(tmp_path / "out.raw")])
    assert r.returncode == 1 and "mismatched sizes" in r.stderr


@pytest.fixture(scope="module")
def scene(tmp_path_factory):
    d = tmp_path_factory.mktemp("cli")
    a = write_surface(str(d / "a"), W.icosphere(3, radius=0.6, seed=2, center=(0.2, 0.0, 0.1)))
    b = write_surface(str(d / "b"), W.torus(0.7, 0.2, nu=40, nv=16, jitter=0.01, seed=3, center=(-0.3, 0.2, 0.0)))
    pts = write_points(str(d / "p"), W.uniform_points(20000, -1.5, 1.5, seed=9))
    return d, [a, b], pts


def chained(meshes, pts, init, dtype):
    out = np.array(init, dtype=dtype)
    for m in meshes:
        out = oracle.edf(pts.astype(dtype), m, out=out, dtype=dtype)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["float", "double", "host_dispatch"])
def test_union_distance(scene, mode):
    d, meshes, pts = scene
    env = {"SSDF_DOUBLE_PRECISION": "1"} if mode == "double" else ({"SSDF_USE_BVH": "0"} if mode == "host_dispatch" else {})
    out_file = str(d / f"out_{mode}.raw")
    r = run([str(d / "a"), str(d / "b"), str(d / "p"), out_file], env)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out_file, dtype=np.float32)
    init = np.full(pts.shape[1], np.finfo(np.float32).max, np.float32)
    if mode == "double":
        want = chained(meshes, pts, init.astype(np.float64), np.float64).astype(np.float32)
    else:
        want = chained(meshes, pts, init, np.float32)
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_warm_start_and_volume_box(scene):
    d, meshes, pts = scene
    n = pts.shape[1]
    start = np.random.default_rng(1).uniform(0.0, 0.5, n).astype(np.float32)
    start.tofile(str(d / "start.raw"))
    r = run([str(d / "b"), str(d / "p"), str(d / "warm.raw")], {"SSDF_INPUT_SDF": str(d / "start.raw")})
    assert r.returncode == 0, r.stderr
    assert np.array_equal(np.fromfile(str(d / "warm.raw"), np.float32), chained(meshes[1:], pts, start, np.float32))
    r = run([str(d / "a"), str(d / "p"), str(d / "box.raw")], {"SSDF_INIT_WITH_VOLUME_BOX": "1"})
    assert r.returncode == 0, r.stderr
    box = oracle.compute_aabb(pts, np.float32)
    init = np.abs(oracle.all_points_aabb_signed_distance(pts, box, np.float32))
    assert np.array_equal(np.fromfile(str(d / "box.raw"), np.float32), chained(meshes[:1], pts, init, np.float32))
    r = run([str(d / "a"), str(d / "p"), str(d / "bad.raw")], {"SSDF_INPUT_SDF": str(d / "start_missing.raw")})
    assert r.returncode == 1
