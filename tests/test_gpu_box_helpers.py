"""GPU: the grid and box helpers (ssdf::compute_aabb, ssdf::all_points_aabb_signed_distance,
serial/edf/edf.hpp:500-557) through the C ABI, bitwise against the oracle.

Every (G, T) instantiation, sizes from one point to several million (one block, ragged tails, the
grid-stride loop), points on faces, edges and corners, the reference's own box_sdf golden vectors,
the device-array forms and the error behaviour.
"""

import numpy as np
import pytest

import oracle
import ssdf_b200 as S
from conftest import load_golden_json

pytestmark = pytest.mark.gpu

PAIRS = [(np.float32, np.float32), (np.float32, np.float64), (np.float64, np.float32), (np.float64, np.float64)]


def _points(n, seed, dtype):
    rng = np.random.default_rng(seed)
    p = rng.uniform(-3.0, 4.0, size=(3, n))
    p[:, : n // 4] = np.round(p[:, : n // 4])
    return p.astype(dtype)


@pytest.mark.parametrize("g,t", PAIRS)
@pytest.mark.parametrize("n", [1, 33, 4099, 3_000_017])
def test_compute_aabb(g, t, n):
    p = _points(n, n, g)
    got = np.array(S.compute_aabb(p, g, t))
    want = oracle.compute_aabb(p.astype(t), t)  # T(x[i]) first, as the reference
    assert np.array_equal(got, want)


@pytest.mark.parametrize("g,t", PAIRS)
@pytest.mark.parametrize("n", [1, 255, 257, 1_000_003])
def test_all_points_aabb_signed_distance(g, t, n):
    p = _points(n, 100 + n, g)
    box = np.array([-1, 2, 0, 3, -2, 1], dtype=t)
    got = S.all_points_aabb_signed_distance(p, box, g, t)
    want = oracle.all_points_aabb_signed_distance(p.astype(t), box, t)
    assert got.dtype == t
    assert np.array_equal(got, want)


def test_box_sdf_golden():
    g = load_golden_json()["box_sdf"]
    pts = np.array([g["x"], g["y"], g["z"]], dtype=np.float64)
    got = S.all_points_aabb_signed_distance(pts, g["box"])
    assert np.array_equal(got, np.array(g["reference"]))
    assert np.all(np.abs(got - np.array(g["expected"])) <= g["tolerance"])


def test_driver_initialisation_on_device():
    """The reference driver's warm start (drivers/sdf.exe.cpp:316-326): the points' own box, then
    |signed distance| to it, here on device arrays."""
    import torch

    p = _points(200_003, 5, np.float64)
    x, y, z = (torch.from_numpy(a.copy()).cuda() for a in p)
    box = torch.empty(6, dtype=torch.float64, device="cuda")
    S.points_aabb_device(x, y, z, box)
    b = box.cpu().numpy()
    assert np.array_equal(b, oracle.compute_aabb(p))
    out = torch.empty(p.shape[1], dtype=torch.float32, device="cuda")
    S.points_aabb_signed_distance_device(x, y, z, b, out, absolute=True)
    want = np.abs(oracle.all_points_aabb_signed_distance(p.astype(np.float32), b.astype(np.float32), np.float32))
    assert np.array_equal(out.cpu().numpy(), want)


def test_errors():
    with pytest.raises(S.SsdfError) as e:
        S.compute_aabb(np.zeros((3, 0)))
    assert e.value.status == S.SSDF_ERR_INVALID_ARGUMENT
    assert S.all_points_aabb_signed_distance(np.zeros((3, 0)), [0, 1, 0, 1, 0, 1]).shape == (0,)
