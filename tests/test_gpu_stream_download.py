"""GPU: the drop-in grid calls whose slab chunks are copied out while the query runs (grids of at
least 2^22 nodes): straight into page-locked output arrays, through page-locked staging slots into
ordinary pageable ones.

Each case calls the same C-ABI entry point twice: once streamed, and once with the streamed download
switched off (query, then one copy), and requires the same bits. The grids have ragged sizes, so the
last brick row, column and slab are partial; a tiny packet budget sends many queries to the fix-up's
second stage, whose values are patched in after the chunk copies.
"""

import ctypes as C
import os

import numpy as np
import pytest

import ssdf_b200 as S
from ssdf_b200 import capi
from ssdf_b200 import workloads as W

pytestmark = pytest.mark.gpu


def pinned(n, dtype):
    import torch

    return torch.empty(n, dtype=dtype, pin_memory=True).numpy()


def grid_call(fn, mesh, grid, out, dtype, tri=None):
    nx, ny, nz = (int(v) for v in grid.n)
    hm = capi._HostMesh(mesh, dtype)
    ct = C.c_double if np.dtype(dtype) == np.float64 else C.c_float
    args = [*hm.args(), nx, ny, nz, *[ct(v) for v in grid.lo], *[ct(v) for v in grid.hi],
            C.c_void_p(out.ctypes.data)]
    if tri is not None:
        args.append(C.cast(C.c_void_p(tri.ctypes.data), C.POINTER(C.c_int)))
    st = getattr(S.lib, fn)(*args)
    assert st == 0, S.last_error()


def plain_call(fn, mesh, grid, out, dtype, tri=None):
    """The same call with the streamed download off: the query, then one copy."""
    old = os.environ.get("SSDF_B200_STREAM_DOWNLOAD")
    os.environ["SSDF_B200_STREAM_DOWNLOAD"] = "0"
    try:
        grid_call(fn, mesh, grid, out, dtype, tri)
    finally:
        if old is None:
            os.environ.pop("SSDF_B200_STREAM_DOWNLOAD", None)
        else:
            os.environ["SSDF_B200_STREAM_DOWNLOAD"] = old


@pytest.fixture(scope="module")
def mesh():
    return W.torus_knot_tube(nu=512, nv=32)


@pytest.fixture(scope="module")
def grid(mesh):
    lo, hi = mesh.bbox()
    g = W.Grid((171, 165, 150), tuple(lo - 0.2), tuple(hi + 0.2))
    assert g.size >= 1 << 22
    return g


@pytest.mark.parametrize("budget", [None, "16"])
def test_streamed_sdf_matches_plain_download(mesh, grid, budget, monkeypatch):
    import torch

    if budget:
        monkeypatch.setenv("SSDF_B200_WARP_BUDGET", budget)
    want = np.full(grid.size, np.nan)
    plain_call("ssdf_b200_sample_sdf_bvh_dd", mesh, grid, want, np.float64)
    for _ in range(2):
        got = pinned(grid.size, torch.float64)
        got[:] = np.nan
        grid_call("ssdf_b200_sample_sdf_bvh_dd", mesh, grid, got, np.float64)
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
    if budget:  # the counting pass shows that second-stage values were patched in
        monkeypatch.setenv("SSDF_B200_COUNT", "1")
        got[:] = np.nan
        grid_call("ssdf_b200_sample_sdf_bvh_dd", mesh, grid, got, np.float64)
        assert S.last_query_counts()["fallback_queries"] > 1000
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64))


def test_streamed_index_and_float_outputs(mesh, grid, monkeypatch):
    import torch

    monkeypatch.setenv("SSDF_B200_WARP_BUDGET", "16")
    want, wtri = np.zeros(grid.size), np.full(grid.size, -7, dtype=np.int32)
    plain_call("ssdf_b200_sample_sdf_index_bvh_dd", mesh, grid, want, np.float64, wtri)
    got, gtri = pinned(grid.size, torch.float64), pinned(grid.size, torch.int32)
    got[:] = 0
    gtri[:] = -7
    grid_call("ssdf_b200_sample_sdf_index_bvh_dd", mesh, grid, got, np.float64, gtri)
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
    assert np.array_equal(gtri, wtri)
    # float grid, FP32 arithmetic
    wf = np.zeros(grid.size, dtype=np.float32)
    plain_call("ssdf_b200_sample_sqedf_bvh_ff", mesh, grid, wf, np.float32)
    gf = pinned(grid.size, torch.float32)
    gf[:] = 0
    grid_call("ssdf_b200_sample_sqedf_bvh_ff", mesh, grid, gf, np.float32)
    assert np.array_equal(gf.view(np.uint32), wf.view(np.uint32))


def test_streamed_squared_distance_keeps_incoming_bound(mesh, grid):
    """sample_sqedf_bvh takes the minimum with the incoming values, which the streamed call uploads
    first: a bound below every distance must come back untouched, others replaced."""
    import torch

    init = np.where(np.arange(grid.size) % 3 == 0, 1e-14, np.inf)
    want = init.copy()
    plain_call("ssdf_b200_sample_sqedf_bvh_dd", mesh, grid, want, np.float64)
    got = pinned(grid.size, torch.float64)
    got[:] = init
    grid_call("ssdf_b200_sample_sqedf_bvh_dd", mesh, grid, got, np.float64)
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
    assert np.all(got[::3] == 1e-14)


def test_streamed_switch_off(mesh, grid, monkeypatch):
    import torch

    want = np.zeros(grid.size)
    grid_call("ssdf_b200_sample_sdf_bvh_dd", mesh, grid, want, np.float64)
    monkeypatch.setenv("SSDF_B200_STREAM_DOWNLOAD", "0")
    got = pinned(grid.size, torch.float64)
    grid_call("ssdf_b200_sample_sdf_bvh_dd", mesh, grid, got, np.float64)
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
    assert os.environ["SSDF_B200_STREAM_DOWNLOAD"] == "0"


@pytest.mark.parametrize("shape", [(2048, 2049, 1), (33, 31, 4104)])
def test_streamed_flat_and_tall_grids(mesh, shape):
    """One slab (a single chunk) and thousands of slabs (many slabs per chunk)."""
    import torch

    lo, hi = mesh.bbox()
    grid = W.Grid(shape, tuple(lo - 0.1), tuple(hi + 0.1))
    assert grid.size >= 1 << 22
    want = np.zeros(grid.size)
    plain_call("ssdf_b200_sample_sdf_bvh_dd", mesh, grid, want, np.float64)
    got = pinned(grid.size, torch.float64)
    got[:] = np.nan
    grid_call("ssdf_b200_sample_sdf_bvh_dd", mesh, grid, got, np.float64)
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))


@pytest.mark.parametrize("page_locked", [True, False])
def test_streamed_calls_from_two_threads(mesh, grid, page_locked):
    """Each calling thread polls its own chunk flags and copies through its own staging slots: two
    threads streaming at once both get their own grid's bits, into page-locked or ordinary arrays."""
    import threading

    import torch

    lo, hi = mesh.bbox()
    grids = [grid, W.Grid((161, 170, 158), tuple(lo - 0.3), tuple(hi + 0.3))]
    wants = []
    for g in grids:
        w = np.zeros(g.size)
        plain_call("ssdf_b200_sample_sdf_bvh_dd", mesh, g, w, np.float64)
        wants.append(w)
    outs = [pinned(g.size, torch.float64) if page_locked else np.empty(g.size) for g in grids]
    errors = []

    def work(i):
        try:
            for _ in range(3):
                outs[i][:] = np.nan
                grid_call("ssdf_b200_sample_sdf_bvh_dd", mesh, grids[i], outs[i], np.float64)
                assert np.array_equal(outs[i].view(np.uint64), wants[i].view(np.uint64))
        except Exception as ex:  # reported on the main thread
            errors.append(repr(ex))

    threads = [threading.Thread(target=work, args=(i,)) for i in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors


@pytest.mark.parametrize("budget", [None, "16"])
def test_streamed_into_pageable_arrays(mesh, grid, budget, monkeypatch):
    """Ordinary numpy arrays (pageable, as the reference's callers pass std::vector memory) take the
    streamed download through the staging slots: the same bits as the plain call, twice in a row, with
    second-stage values patched in when the tiny budget sends thousands of queries there."""
    if budget:
        monkeypatch.setenv("SSDF_B200_WARP_BUDGET", budget)
    want, wtri = np.full(grid.size, np.nan), np.full(grid.size, -7, dtype=np.int32)
    plain_call("ssdf_b200_sample_sdf_index_bvh_dd", mesh, grid, want, np.float64, wtri)
    for _ in range(2):
        got, gtri = np.full(grid.size, np.nan), np.full(grid.size, -7, dtype=np.int32)
        grid_call("ssdf_b200_sample_sdf_index_bvh_dd", mesh, grid, got, np.float64, gtri)
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
        assert np.array_equal(gtri, wtri)


def test_streamed_mixed_page_locked_and_pageable(mesh, grid):
    """A page-locked distance array with a pageable index array, and the other way round."""
    import torch

    want, wtri = np.zeros(grid.size), np.zeros(grid.size, dtype=np.int32)
    plain_call("ssdf_b200_sample_sdf_index_bvh_dd", mesh, grid, want, np.float64, wtri)
    for out_pinned in (True, False):
        got = pinned(grid.size, torch.float64) if out_pinned else np.empty(grid.size)
        gtri = np.empty(grid.size, dtype=np.int32) if out_pinned else pinned(grid.size, torch.int32)
        got[:] = np.nan
        gtri[:] = -7
        grid_call("ssdf_b200_sample_sdf_index_bvh_dd", mesh, grid, got, np.float64, gtri)
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
        assert np.array_equal(gtri, wtri)


def test_streamed_pageable_float_grid_and_small_grids(mesh, grid):
    """A float grid (4-byte values) through the staging slots, then a larger grid on the same thread
    (the slots grow) and a grid below 2^22 nodes (the plain path)."""
    wf = np.zeros(grid.size, dtype=np.float32)
    plain_call("ssdf_b200_sample_sqedf_bvh_ff", mesh, grid, wf, np.float32)
    gf = np.zeros(grid.size, dtype=np.float32)
    grid_call("ssdf_b200_sample_sqedf_bvh_ff", mesh, grid, gf, np.float32)
    assert np.array_equal(gf.view(np.uint32), wf.view(np.uint32))
    lo, hi = mesh.bbox()
    for shape in [(200, 190, 180), (90, 80, 70)]:
        g = W.Grid(shape, tuple(lo - 0.2), tuple(hi + 0.2))
        want = np.zeros(g.size)
        plain_call("ssdf_b200_sample_sdf_bvh_dd", mesh, g, want, np.float64)
        got = np.full(g.size, np.nan)
        grid_call("ssdf_b200_sample_sdf_bvh_dd", mesh, g, got, np.float64)
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
