"""GPU: the allocation-free grid query (ssdf_query_grid_noalloc) through the C ABI.

Some callers cannot allocate device memory at query time -- a real-time loop that reserves all of
its memory up front, or a host application that owns every allocation and forbids the CUDA
allocator -- so this entry point keeps its scratch (the fix-up overflow list) in a fixed array
inside the library. Checked against the allocating entry point (ssdf_query_grid) on two calls in a
row, with the tolerance the other parity tests use: bitwise equality. This file is collected last
and also passes alone in a fresh process.
"""

import ctypes as C

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


def test_noalloc_matches_allocating_query_twice():
    import torch

    mesh = W.torus_knot_tube(nu=512, nv=32)
    dm = S.DeviceMesh(mesh)
    stream = torch.cuda.current_stream()
    grids = [W.Grid.padded_nodes(mesh, 96, 0.25), W.Grid((70, 50, 40), (-1.6, -1.5, -0.7), (1.7, 1.6, 0.8))]
    for grid in grids:
        assert grid.size <= S.lib.ssdf_query_grid_noalloc_max()
        want = torch.empty(grid.size, dtype=torch.float64, device="cuda")
        wtri = torch.empty(grid.size, dtype=torch.int32, device="cuda")
        dm.query_grid(grid, want, wtri, precision=S.PREC_F32_FIXUP, output=S.OUT_SDF, stream=stream)
        for _ in range(2):  # two calls in a row share the library's scratch array
            got = torch.full((grid.size,), -1.0, dtype=torch.float64, device="cuda")
            gtri = torch.full((grid.size,), -1, dtype=torch.int32, device="cuda")
            assert call_noalloc(dm, grid, got, gtri, stream) == S.SSDF_OK, S.last_error()
            torch.cuda.synchronize()
            assert np.array_equal(got.cpu().numpy(), want.cpu().numpy())
            assert np.array_equal(gtri.cpu().numpy(), wtri.cpu().numpy())
    dm.close()


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
