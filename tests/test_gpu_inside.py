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


def ray_parity(points, mesh, direction):
    """Inside by the parity of a ray's crossings (the rule of the reference's cuBQL build), brute
    force in double: Moller-Trumbore against every triangle."""
    v = mesh.vertices[mesh.triangles]  # [m, 3, 3]
    a, e1, e2 = v[:, 0], v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]
    d = np.asarray(direction, dtype=np.float64)
    h = np.cross(d, e2)
    det = np.einsum("ij,ij->i", e1, h)
    ok = np.abs(det) > 1e-14
    inv = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0)
    flags = []
    for p in points.T:
        s = p - a
        u = inv * np.einsum("ij,ij->i", s, h)
        q = np.cross(s, e1)
        w = inv * (q @ d)
        t = inv * np.einsum("ij,ij->i", e2, q)
        hit = ok & (u >= 0) & (w >= 0) & (u + w <= 1) & (t > 0)
        flags.append(int(hit.sum()) % 2)
    return np.array(flags, dtype=np.uint8)


def test_inside_on_an_open_mesh():
    """An open mesh (a sphere with its top cap removed): the flags are the sign of the signed
    distance -- the side of the nearest surface its pseudo-normals face -- which needs no closed
    surface. The reference's ray parity is defined only for closed surfaces: on this open cup it depends
    on the ray's direction. On a closed sphere both rules agree away from the surface."""
    full = W.icosphere(3, radius=1.0, displacement=0.0)
    cen = full.vertices[full.triangles].mean(1)
    cup = W.Mesh(full.vertices, full.triangles[cen[:, 2] < 0.6])
    rng = np.random.default_rng(8)
    p = rng.uniform(-1.2, 1.2, size=(3, 3000))
    got = S.points_inside_bvh(p, cup)
    sd, _ = oracle.sdf_points(p, cup)
    assert np.array_equal(got, (sd < 0).astype(np.uint8))  # what this library returns, everywhere
    # a point in the cup below the opening, near its axis: inside by the pseudo-normal rule; the ray
    # parity says inside towards the bottom (one crossing) and outside towards the opening (none).
    # The rays lean off the axis so that they cross triangle interiors, not the pole's vertex.
    q = np.array([[0.0], [0.0], [0.5]])
    assert S.points_inside_bvh(q, cup)[0] == 1
    assert ray_parity(q, cup, (0.0137, 0.0291, -1))[0] == 1
    assert ray_parity(q, cup, (0.0137, 0.0291, 1))[0] == 0
    # closed sphere: the two rules agree away from the surface
    r = np.linalg.norm(p, axis=0)
    far = np.abs(r - 1.0) > 0.05
    sub = p[:, far][:, :400]
    assert np.array_equal(S.points_inside_bvh(sub, full), ray_parity(sub, full, (0.3, 0.5, 0.81)))
