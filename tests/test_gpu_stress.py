"""Seeded random sweep over the query knobs: each case draws a mesh (a jittered torus, an icosphere,
a soup with degenerate and sliver triangles, or slivers split off a sphere), a point set (sizes
around the Morton-order threshold, some far outside) or a grid, and a setting of every switch that
must not change the result -- traversal (warp / thread), arity (2 / 4), leaf size, Morton order,
the fix-up packet budget (forced small), the fix-up window's stack -- then checks the fix-up and
FP64 paths against each other at every query and against the oracle on a sample, bit for bit."""

import numpy as np
import pytest

import oracle
import ssdf_b200 as S
from ssdf_b200 import workloads as W
from test_gpu_golden import env

pytestmark = pytest.mark.gpu


def random_mesh(rng):
    kind = rng.integers(4)
    if kind == 0:
        return W.torus(nu=int(rng.integers(16, 80)), nv=int(rng.integers(8, 40)), jitter=0.01)
    if kind == 1:
        return W.icosphere(int(rng.integers(1, 5)), displacement=float(rng.uniform(0, 0.05)), seed=int(rng.integers(99)))
    if kind == 2:
        n = int(rng.integers(50, 2000))
        c = rng.uniform(-1, 1, size=(n, 1, 3))
        v = c + rng.normal(0, 0.1, size=(n, 3, 3))
        v[: n // 10, 2] = v[: n // 10, 1]  # degenerate: repeated corner
        v[n // 10: n // 5, 2] = 0.5 * (v[n // 10: n // 5, 0] + v[n // 10: n // 5, 1]) + 1e-5  # slivers
        return W.Mesh(v.reshape(-1, 3), np.arange(3 * n, dtype=np.int32).reshape(-1, 3))
    base = W.icosphere(2, displacement=0.01, seed=3)
    v = list(base.vertices)
    tris = []
    for a, b, c in base.triangles:
        m = 0.5 * (base.vertices[a] + base.vertices[b]) + 1e-4 * (base.vertices[c] - base.vertices[a])
        v.append(m)
        im = len(v) - 1
        tris += [(a, im, c), (im, b, c), (a, b, im)]
    return W.Mesh(np.array(v), np.array(tris, dtype=np.int32))


def random_knobs(rng):
    return {
        "SSDF_B200_TRAVERSAL": ["warp", "thread"][rng.integers(2)],
        "SSDF_B200_ARITY": [2, 4][rng.integers(2)],
        "SSDF_B200_LEAF": [1, 2, 4, 8, 16][rng.integers(5)],
        "SSDF_B200_SORT_POINTS": int(rng.integers(2)),
        "SSDF_B200_WARP_BUDGET": [0, 16, 256, 2048][rng.integers(4)],
        "SSDF_B200_WINDOW_STACK": [1, 8, 64][rng.integers(3)],
        "SSDF_B200_ILL_MAX": [2, 0.5][rng.integers(2)],
    }


@pytest.mark.parametrize("seed", range(30))
def test_random_knobs_points(seed):
    rng = np.random.default_rng(1000 + seed)
    mesh = random_mesh(rng)
    lo, hi = mesh.bbox()
    ext = hi - lo
    n = int(rng.choice([100, 4095, 4096, 9000]))
    pts = rng.uniform(lo - 0.3 * ext, hi + 0.3 * ext, size=(n, 3))
    pts[:5] = lo + rng.uniform(-50, 50, size=(5, 3)) * ext
    pts = np.ascontiguousarray(pts.T)
    knobs = random_knobs(rng)
    with env(**knobs):
        with env(SSDF_B200_PRECISION="f32x"):
            d1, t1 = S.edf_index(pts, mesh)
            s1, st1 = S.sdf_points(pts, mesh)
        with env(SSDF_B200_PRECISION="f64"):
            d2, t2 = S.edf_index(pts, mesh)
            s2, st2 = S.sdf_points(pts, mesh)
    assert np.array_equal(d1, d2) and np.array_equal(t1, t2), knobs
    assert np.array_equal(s1, s2) and np.array_equal(st1, st2), knobs
    ids = rng.choice(n, size=min(n, 150), replace=False)
    want, wtri = oracle.edf(pts[:, ids], mesh, with_index=True)
    assert np.array_equal(d1[ids], want) and np.array_equal(t1[ids], wtri), knobs
    ws, wst = oracle.sdf_points(pts[:, ids], mesh)
    assert np.array_equal(s1[ids], ws) and np.array_equal(st1[ids], wst), knobs


@pytest.mark.parametrize("seed", range(30))
def test_random_knobs_grids(seed):
    rng = np.random.default_rng(2000 + seed)
    mesh = random_mesh(rng)
    lo, hi = mesh.bbox()
    shape = tuple(int(v) for v in rng.integers(3, 40, size=3))
    grid = W.Grid(shape, tuple(lo - 0.25), tuple(hi + 0.25))
    knobs = random_knobs(rng)
    with env(**knobs):
        with env(SSDF_B200_PRECISION="f32x"):
            d1, t1 = S.sample_sdf_bvh(mesh, grid, with_index=True)
        with env(SSDF_B200_PRECISION="f64"):
            d2, t2 = S.sample_sdf_bvh(mesh, grid, with_index=True)
    assert np.array_equal(d1, d2) and np.array_equal(t1, t2), knobs
    ids = rng.choice(grid.size, size=min(grid.size, 150), replace=False)
    want, wtri = oracle.sdf_points(oracle.grid_points(grid)[:, ids], mesh)
    assert np.array_equal(d1[ids], want) and np.array_equal(t1[ids], wtri), knobs
