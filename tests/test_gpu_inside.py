"""GPU: inside flags (ssdf::points_inside_bvh, ssdf::sample_inside_bvh through the C ABI).

Inside is where the signed distance (sample_sdf_bvh's pseudo-normal rule, checked against the oracle
elsewhere) is negative: the flags equal the oracle's sign, and on a sphere they agree with |p| < r
away from the surface. The voxel staircase gives a non-convex closed surface.
"""

import numpy as np
import pytest

import oracle
import ssdf_b200 as S
from ssdf_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_points_inside_sphere(dtype):
    mesh = W.icosphere(4, radius=1.0, displacement=0.0)
    p = W.uniform_points(20000, -1.3, 1.3, seed=3)
    got = S.points_inside_bvh(p.astype(dtype), mesh, dtype)
    if dtype == np.float64:
        sd, _ = oracle.sdf_points(p, mesh)
        assert np.array_equal(got, (sd < 0).astype(np.uint8))
    r = np.linalg.norm(p, axis=0)
    far = np.abs(r - 1.0) > 0.02  # the tessellation is within 0.02 of the sphere
    assert np.array_equal(got[far], (r[far] < 1.0).astype(np.uint8))


def test_sample_inside_knot_and_grid_convention():
    mesh = W.torus_knot_tube(nu=256, nv=24)
    grid = W.Grid.padded_nodes(mesh, 48, 0.2)
    got = S.sample_inside_bvh(mesh, grid)
    sd = S.sample_sdf_bvh(mesh, grid)
    assert np.array_equal(got, (sd < 0).astype(np.uint8))
    assert 0 < got.sum() < grid.size
    ids = np.random.default_rng(2).choice(grid.size, 2000, replace=False)
    want, _ = oracle.sdf_points(oracle.grid_points(grid)[:, ids], mesh)
    assert np.array_equal(got[ids], (want < 0).astype(np.uint8))
