"""Point lists of 4096 queries or more are visited in Morton order (a sort on the device, then
warp-packet traversal). Results are per query, so the visiting order must change nothing: the
sorted and the input-order launches agree bit for bit, on ragged lengths, duplicated points,
points far outside the mesh's box, float and double coordinates, and every output kind, and a
seeded sample agrees with the oracle."""

import numpy as np
import pytest

import oracle
import ssdf_b200 as S
from ssdf_b200 import workloads as W
from test_gpu_golden import env

pytestmark = pytest.mark.gpu


def _points(mesh, n, seed):
    rng = np.random.default_rng(seed)
    lo, hi = mesh.bbox()
    ext = hi - lo
    pts = rng.uniform(lo - 0.3 * ext, hi + 0.3 * ext, size=(n, 3))
    pts[: n // 10] = pts[n // 10: 2 * (n // 10)]  # duplicates
    pts[-50:] = lo + rng.uniform(-40, 40, size=(50, 3)) * ext  # far outside the root box
    v = mesh.vertices[mesh.triangles[rng.integers(0, mesh.nt, n // 5), 0]]
    pts[2 * (n // 10): 2 * (n // 10) + n // 5] = v  # on the surface (corners)
    return np.ascontiguousarray(pts.T)


@pytest.mark.parametrize("n", [4096, 4097, 70001])
def test_sorted_equals_input_order(n):
    mesh = W.torus_knot_tube(nu=192, nv=24)
    pts = _points(mesh, n, seed=n)
    for prec in ("f32x", "f64"):
        with env(SSDF_B200_PRECISION=prec):
            with env(SSDF_B200_SORT_POINTS=0):
                d0, t0 = S.edf_index(pts, mesh)
                s0, st0 = S.sdf_points(pts, mesh)
            d1, t1 = S.edf_index(pts, mesh)
            s1, st1 = S.sdf_points(pts, mesh)
        assert np.array_equal(d0, d1) and np.array_equal(t0, t1), prec
        assert np.array_equal(s0, s1) and np.array_equal(st0, st1), prec
    f = pts.astype(np.float32)
    with env(SSDF_B200_SORT_POINTS=0):
        g0 = S.edf_bvh(f, mesh, gdtype=np.float32)
    assert np.array_equal(g0, S.edf_bvh(f, mesh, gdtype=np.float32))
    ids = np.arange(0, n, 97)
    want, wtri = oracle.edf(pts[:, ids], mesh, with_index=True)
    assert np.array_equal(d1[ids], want) and np.array_equal(t1[ids], wtri)


def test_sorted_closest_point_and_incoming_values():
    mesh = W.icosphere(3)
    pts = _points(mesh, 9000, seed=4)
    init = np.where(np.arange(9000) % 3 == 0, 0.01, np.finfo(np.float64).max)
    with env(SSDF_B200_SORT_POINTS=0):
        a = S.closest_point_bvh(pts, mesh, outd=init)
    b = S.closest_point_bvh(pts, mesh, outd=init)
    for x, y, name in zip(a, b, ("d", "x", "y", "z", "tri")):
        assert np.array_equal(x, y), name
    ids = np.arange(0, 9000, 41)
    want = oracle.closest_point(pts[:, ids], mesh, outd=init[ids])
    for w, g, name in zip(want, b, ("d", "x", "y", "z", "tri")):
        assert np.array_equal(w, g[ids]), name


def test_sorted_inside_flags():
    mesh = W.icosphere(3)
    pts = _points(mesh, 6000, seed=8)
    with env(SSDF_B200_SORT_POINTS=0):
        a = S.points_inside_bvh(pts, mesh)
    assert np.array_equal(a, S.points_inside_bvh(pts, mesh))
