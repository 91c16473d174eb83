"""GPU: the sign fixture of ssdf's tests/sample_sdf_bvh_test.cpp:19-132 through sample_sdf_bvh.

A watertight, non-convex voxel staircase whose faces lie on the sampling grid's planes and whose
edges lie on its lines (the worst case for a sign): zero wrong signs and a worst distance error
below 1e-5 against the exact distance, on the float and the double entry point, as the reference
test asserts; and bitwise the oracle's values.
"""

import numpy as np
import pytest

import oracle
import ssdf_b200 as S
from ssdf_b200 import workloads as W
from test_gpu_golden import env

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("prec", ["f32x", "f64"])
def test_staircase(dtype, prec):
    mesh, lo, hi, filled = W.voxel_staircase()
    n = 5 * (4 + 2) + 1
    grid = W.Grid((n, n, n), (-0.25,) * 3, (1.25,) * 3)
    with env(SSDF_B200_PRECISION=prec):
        got = S.sample_sdf_bvh(mesh, grid, dtype=dtype)
    q = oracle.grid_points(grid, dtype=dtype)
    p = q.T
    d2 = np.full(p.shape[0], np.inf)
    for a, b in zip(lo, hi):
        c = np.clip(p, a, b)
        d2 = np.minimum(d2, ((p - c) ** 2).sum(1))
    d = np.sqrt(d2)
    inside = np.array([filled(*c) for c in np.floor(p / 0.25).astype(int)])
    keep = d >= 1e-6
    assert np.sum((got[keep] < 0) != inside[keep]) == 0
    assert np.max(np.abs(np.abs(got[keep].astype(np.float64)) - d[keep])) < 1e-5
    want, _ = oracle.sdf_points(q, mesh)
    assert np.array_equal(got, want.astype(dtype))
