"""GPU: the allocation-free grid query (ssdf_query_grid_noalloc) through the C ABI.

Some callers cannot allocate device memory at query time -- a real-time loop that reserves all of
its memory up front, or a host application that owns every allocation and forbids the CUDA
allocator -- so this entry point keeps its scratch (the fix-up overflow list: query ids and their
final windows) in a fixed array inside the library. Checked against the allocating entry point
(ssdf_query_grid) and the plain double kernel on calls in a row, with the tolerance the other parity
tests use: bitwise equality.

The grids near the centre of an undisplaced icosphere send most of their queries through the
overflow list (every triangle is almost equidistant there), so the fixed array's ids and windows are
read by the second stage; the allocating query's counters show how many. A call with many overflows
followed by one with few shows that each call starts its list from zero. This file is collected
last and also passes alone in a fresh process.
"""

import ctypes as C
import os

import numpy as np
import pytest

import ssdf_b200 as S
from ssdf_b200 import workloads as W

pytestmark = pytest.mark.gpu


def call_noalloc(dm, grid, out, tri, stream):
    o = S.QueryOpts(S.PREC_F32_FIXUP, S.OUT_SDF, S.F64, S.F64)
    lo = (C.c_double * 3)(*grid.lo)
    hi = (C.c_double * 3)(*grid.hi)
    return S.lib.ssdf_query_grid_noalloc(dm._h, *(int(v) for v in grid.n), C.byref(lo), C.byref(hi), out.data_ptr(),
                                         C.cast(C.c_void_p(tri.data_ptr()), C.POINTER(C.c_int)), C.byref(o),
                                         stream.cuda_stream)


def allocating(dm, grid, prec, stream, count=False):
    """The allocating query (and, with count, how many queries its second stage answered)."""
    import torch

    out = torch.empty(grid.size, dtype=torch.float64, device="cuda")
    tri = torch.empty(grid.size, dtype=torch.int32, device="cuda")
    old = os.environ.get("SSDF_B200_COUNT")
    if count:
        os.environ["SSDF_B200_COUNT"] = "1"
    try:
        dm.query_grid(grid, out, tri, precision=prec, output=S.OUT_SDF, stream=stream)
        torch.cuda.synchronize()
    finally:
        if old is None:
            os.environ.pop("SSDF_B200_COUNT", None)
        else:
            os.environ["SSDF_B200_COUNT"] = old
    fallbacks = S.last_query_counts()["fallback_queries"] if count else None
    return out.cpu().numpy(), tri.cpu().numpy(), fallbacks


def noalloc(dm, grid, stream):
    import torch

    got = torch.full((grid.size,), -1.0, dtype=torch.float64, device="cuda")
    gtri = torch.full((grid.size,), -7, dtype=torch.int32, device="cuda")
    assert call_noalloc(dm, grid, got, gtri, stream) == S.SSDF_OK, S.last_error()
    torch.cuda.synchronize()
    return got.cpu().numpy(), gtri.cpu().numpy()


def centre_grid(n, r=2e-5):
    return W.Grid((n, n, n), (-r, -r, -r), (r, r, r))


def test_noalloc_matches_allocating_query_twice():
    import torch

    mesh = W.torus_knot_tube(nu=512, nv=32)
    dm = S.DeviceMesh(mesh)
    stream = torch.cuda.current_stream()
    grids = [W.Grid.padded_nodes(mesh, 96, 0.25), W.Grid((70, 50, 40), (-1.6, -1.5, -0.7), (1.7, 1.6, 0.8))]
    for grid in grids:
        assert grid.size <= S.lib.ssdf_query_grid_noalloc_max()
        want, wtri, _ = allocating(dm, grid, S.PREC_F32_FIXUP, stream)
        for _ in range(2):  # two calls in a row share the library's scratch array
            got, gtri = noalloc(dm, grid, stream)
            assert np.array_equal(got, want)
            assert np.array_equal(gtri, wtri)
    dm.close()


@pytest.mark.parametrize("sub", [2, 4])
def test_noalloc_overflow_list_in_the_fixed_array(sub):
    """Most queries overflow their windows: their ids and windows go through the fixed array."""
    import torch

    mesh = W.icosphere(sub, radius=1.0, displacement=0.0)
    dm = S.DeviceMesh(mesh)
    stream = torch.cuda.current_stream()
    grid = centre_grid(16)
    want, wtri, fallbacks = allocating(dm, grid, S.PREC_F32_FIXUP, stream, count=True)
    assert fallbacks > grid.size // 2, fallbacks  # the second stage answers most of these queries
    d64, t64, _ = allocating(dm, grid, S.PREC_F64, stream)
    assert np.array_equal(want, d64) and np.array_equal(wtri, t64)
    for _ in range(2):
        got, gtri = noalloc(dm, grid, stream)
        assert np.array_equal(got, d64) and np.array_equal(gtri, t64)
        assert np.all(got < 0)  # the centre is inside
    dm.close()


def test_noalloc_many_overflows_then_few():
    """A call whose list is long, then calls whose lists are short or empty, then the long one
    again: each call counts its overflows from zero, so no stale entry of an earlier call is read."""
    import torch

    sphere = S.DeviceMesh(W.icosphere(3, radius=1.0, displacement=0.0))
    knot_mesh = W.torus_knot_tube(nu=256, nv=32)
    knot = S.DeviceMesh(knot_mesh)
    stream = torch.cuda.current_stream()
    many = centre_grid(24)  # 13,824 queries, most of them overflow
    few = W.Grid.padded_nodes(knot_mesh, 40, 0.25)  # few or none overflow
    tiny = centre_grid(3)  # 27 queries
    cases = [(sphere, many), (knot, few), (sphere, tiny), (knot, few), (sphere, many)]
    want = {}
    for dm, grid in cases:
        key = (id(dm), grid.n)
        if key not in want:
            want[key] = allocating(dm, grid, S.PREC_F64, stream)[:2]
        got, gtri = noalloc(dm, grid, stream)
        assert np.array_equal(got, want[key][0]) and np.array_equal(gtri, want[key][1]), grid.n
    _, _, fb_many = allocating(sphere, many, S.PREC_F32_FIXUP, stream, count=True)
    _, _, fb_few = allocating(knot, few, S.PREC_F32_FIXUP, stream, count=True)
    assert fb_many > many.size // 2 and fb_few < fb_many // 100, (fb_many, fb_few)
    sphere.close()
    knot.close()


def test_noalloc_rejects_grids_over_its_limit():
    import torch

    mesh = W.icosphere(2)
    dm = S.DeviceMesh(mesh)
    side = int(round(S.lib.ssdf_query_grid_noalloc_max() ** (1 / 3))) + 2
    grid = W.Grid.padded_nodes(mesh, side, 0.2)
    out = torch.empty(grid.size, dtype=torch.float64, device="cuda")
    tri = torch.empty(grid.size, dtype=torch.int32, device="cuda")
    st = call_noalloc(dm, grid, out, tri, torch.cuda.current_stream())
    assert st == 4 and "at most" in S.last_error()
    dm.close()
