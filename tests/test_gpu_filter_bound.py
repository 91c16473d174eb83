"""GPU: the fix-up path where the FP32 filter's error bound is tightest, and its guards.

The fix-up window is sized from a forward error bound of the FP32 filter (input rounding of the
point and the corners, every fmaf, the quotient and reciprocal, the region decisions). The bound
grows with the coordinates' magnitude M against the triangles' size, so this sweeps:
  - unit-size meshes moved to offsets 1e5, 1e6 and 1e7 (M far above the triangle size; at 1e6 and
    beyond, float rounding collapses the triangles and the mesh is handed to the FP64 kernel);
  - meshes scaled down to 1e-3 and 1e-7 (below 2^-23 edges the filter's products underflow: FP64);
  - soups mixing triangles of size 1 with triangles of size 1e-4 (the window widens);
  - points beyond the filter's coordinate range (2^28), answered exactly by the second stage.
Every query of the fix-up path must equal the plain FP64 path bit for bit, and the oracle on samples.
"""

import numpy as np
import pytest
import torch

import oracle
import ssdf_b200 as S
from ssdf_b200 import workloads as W

pytestmark = pytest.mark.gpu


def both(dm, grid=None, points=None):
    outs = []
    for prec in (S.PREC_F32_FIXUP, S.PREC_F64):
        if grid is not None:
            out = torch.empty(grid.size, dtype=torch.float64, device="cuda")
            tri = torch.empty(grid.size, dtype=torch.int32, device="cuda")
            dm.query_grid(grid, out, tri, precision=prec, output=S.OUT_SDF)
        else:
            x, y, z = (torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda") for a in points)
            out = torch.full((len(points[0]),), np.finfo(np.float64).max, dtype=torch.float64, device="cuda")
            tri = torch.full((len(points[0]),), -1, dtype=torch.int32, device="cuda")
            dm.query_points(x, y, z, out, tri, precision=prec, output=S.OUT_EDF)
        torch.cuda.synchronize()
        outs.append((out.cpu().numpy(), tri.cpu().numpy()))
    return outs


def shifted(mesh, offset, scale=1.0):
    return W.Mesh(mesh.vertices * scale + np.asarray(offset, dtype=np.float64), mesh.triangles)


def check_grid(mesh, n=28, pad=0.15, sample=997):
    dm = S.DeviceMesh(mesh)
    info = dm.filter_info()
    lo, hi = mesh.bbox()
    ext = hi - lo
    grid = W.Grid((n, n, n), tuple(lo - pad * ext), tuple(hi + pad * ext))
    (d, t), (d64, t64) = both(dm, grid=grid)
    dm.close()
    assert np.array_equal(d, d64) and np.array_equal(t, t64)
    ids = np.arange(0, grid.size, max(1, grid.size // sample))
    want, wtri = oracle.sdf_points(oracle.grid_points(grid)[:, ids], mesh)
    assert np.array_equal(d[ids], want) and np.array_equal(t[ids], wtri)
    return info


@pytest.mark.parametrize("offset", [1e5, 1e6, 1e7])
def test_unit_meshes_at_large_offsets(offset):
    torus = W.torus(0.7, 0.2, nu=48, nv=24, jitter=0.01, seed=3)
    sphere = W.icosphere(3, radius=0.5)
    for mesh in (torus, sphere):
        info = check_grid(shifted(mesh, (offset, -0.37 * offset, 0.61 * offset)))
        if offset >= 1e6:  # float rounding (ulp 0.06 at 1e6) collapses these triangles: FP64 answers
            assert not info["float_filter"], info
        assert info["tau_rel"] >= 2.0 ** -16


@pytest.mark.parametrize("scale", [1e-3, 1e-7])
def test_small_meshes(scale):
    mesh = shifted(W.torus(0.7, 0.2, nu=40, nv=20, jitter=0.01, seed=4), (0.0, 0.0, 0.0), scale)
    info = check_grid(mesh)
    # edges of about 0.1 scale: float-filtered at 1e-3, below 2^-23 (underflow in the filter) at 1e-7
    assert info["float_filter"] == (scale > 1e-6), info


def test_mixed_scale_soup():
    """Unit triangles beside 1e-4 ones: the large records widen the window above 2^-16."""
    rng = np.random.default_rng(9)
    big = W.random_soup(40, seed=1, scale=1.0)
    small = []
    for c in rng.uniform(-1, 1, size=(300, 3)):
        v = c + rng.normal(scale=1e-4, size=(3, 3))
        small.append(v)
    small = np.concatenate(small)
    verts = np.concatenate([big.vertices, small])
    tris = np.concatenate([big.triangles, big.nv + np.arange(len(small)).reshape(-1, 3)]).astype(np.int32)
    mesh = W.Mesh(verts, tris)
    info = check_grid(mesh, n=32)
    assert info["float_filter"] and info["tau_rel"] > 2.0 ** -16, info


def test_single_large_triangles():
    """A mesh of a few triangles as large as its coordinates (the reference tests' single triangle):
    the window widens to cover the bound."""
    v = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.3, 0.2, 0.9]])
    mesh = W.Mesh(v, np.array([[0, 1, 2], [0, 1, 3], [1, 2, 3]], dtype=np.int32))
    info = check_grid(mesh, n=40, pad=0.5)
    assert info["float_filter"] and info["tau_rel"] > 2.0 ** -16, info


def test_points_beyond_the_filter_range():
    """Finite points past 2^28 (where the float filter's products could overflow) are answered
    exactly in the second stage; the rest of the launch is unaffected."""
    mesh = W.torus(0.7, 0.2, nu=48, nv=24, jitter=0.01, seed=5)
    dm = S.DeviceMesh(mesh)
    assert dm.filter_info()["float_filter"]
    pts = W.uniform_points(5000, -1.0, 1.0, seed=21)
    far = np.array([[3e8, -1.0, 0.5], [-2.0**40, 2.0**29, 1.0], [1e12, 1e12, -1e12], [0.1, 0.2, 5e8]]).T
    pts = np.concatenate([pts, far, W.uniform_points(3000, -2.0, 2.0, seed=22)], axis=1)
    (d, t), (d64, t64) = both(dm, points=pts)
    dm.close()
    assert np.array_equal(d, d64) and np.array_equal(t, t64)
    want, wtri = oracle.edf(pts[:, 4995:5009], mesh, with_index=True)
    assert np.array_equal(d[4995:5009], want) and np.array_equal(t[4995:5009], wtri)
