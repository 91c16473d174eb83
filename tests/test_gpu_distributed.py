"""pedf / pedf_update on the GPU through a one-rank NCCL group (this machine has one GPU): the
distances equal the single-process drop-in edf on the whole surface, bit for bit, for double and
float, both pedf modes, and pedf_update from a loose upper bound. The exchanges with several ranks
are tested on CPU (tests/test_distributed.py)."""

import socket

import numpy as np
import pytest

import ssdf_b200 as S
from ssdf_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def group():
    import torch.distributed as dist

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", rank=0, world_size=1, init_method=f"tcp://127.0.0.1:{port}")
    yield None
    dist.destroy_process_group()


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_pedf_equals_edf(group, dtype):
    import torch

    from ssdf_b200 import distributed as D

    mesh = W.torus(nu=96, nv=48, jitter=0.01)
    lo, hi = mesh.bbox()
    pts = W.uniform_points(20000, lo - 0.3, hi + 0.3, seed=3).astype(dtype)
    init = np.full(pts.shape[1], np.finfo(dtype).max, dtype=dtype)
    init[::7] = 0.05
    want = S.edf_bvh(pts, mesh, out=init, gdtype=dtype)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    x, y, z = (dev(a) for a in pts)
    s0, s1, s2 = (dev(a) for a in mesh.indices())
    sx, sy, sz = (dev(a.astype(dtype)) for a in mesh.coords())
    for mode in (True, False):
        out = dev(init)
        D.pedf(x, y, z, s0, s1, s2, sx, sy, sz, out, use_allgather=mode)
        assert np.array_equal(out.cpu().numpy(), want), mode
    # pedf_update from upper bounds 1.5x the answer (and the 0.05 incoming values kept)
    out = dev(np.minimum(init, want * dtype(1.5)))
    D.pedf_update(x, y, z, s0, s1, s2, sx, sy, sz, out)
    assert np.array_equal(out.cpu().numpy(), want)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_selection_steps_on_the_device(dtype):
    """ssdf_grown_box and ssdf_triangles_meeting_boxes against a brute-force selection: the grown box
    of points with distances (an empty point set gives the inverted box), and for several boxes the
    corners of every triangle meeting each, in triangle order, box after box."""
    import torch

    from ssdf_b200 import capi

    tdt = torch.float64 if dtype == np.float64 else torch.float32
    rng = np.random.default_rng(3)
    pts = rng.uniform(-1, 1, size=(3, 5003)).astype(dtype)
    out = rng.uniform(0.01, 0.3, size=5003)
    x, y, z = (torch.tensor(a, device="cuda") for a in pts)
    for odt in (torch.float64, torch.float32):
        r = torch.tensor(out, dtype=odt, device="cuda")
        box = capi.grown_box(x, y, z, r).cpu().numpy()
        rr = out.astype(np.float32 if odt == torch.float32 else np.float64).astype(dtype)
        want = np.concatenate([(pts - rr).min(1), (pts + rr).max(1)])
        assert np.array_equal(box, want)
    empty = torch.empty(0, dtype=tdt, device="cuda")
    big = np.finfo(dtype).max
    assert np.array_equal(capi.grown_box(empty, empty, empty, empty.double()).cpu().numpy(),
                          np.array([big, big, big, -big, -big, -big], dtype=dtype))
    mesh = W.random_soup(3000, seed=5, scale=1.5)
    v = mesh.vertices.astype(dtype)
    s = [torch.tensor(np.ascontiguousarray(a, dtype=np.int32), device="cuda") for a in mesh.indices()]
    sv = [torch.tensor(np.ascontiguousarray(v[:, d]), device="cuda") for d in range(3)]
    boxes = np.array([[-0.5, -0.5, -0.5, 0.2, 0.3, 0.1], [0.9, -2, -2, 2, 2, 2], [5, 5, 5, 6, 6, 6],
                      [-2, -2, -2, 2, 2, 2]], dtype=dtype)
    corners, counts = capi.triangles_meeting_boxes(*s, *sv, torch.tensor(boxes, device="cuda"))
    c = v[mesh.triangles]  # [m, 3 corners, 3 axes]
    tlo, thi = c.min(1), c.max(1)
    rows, want_counts = [], []
    for b in boxes:
        hit = ~((thi < b[:3]) | (tlo > b[3:])).any(1)
        rows.append(c[hit].reshape(-1, 9))
        want_counts.append(int(hit.sum()))
    assert counts == want_counts and counts[2] == 0 and counts[3] == mesh.nt
    assert np.array_equal(corners.cpu().numpy(), np.concatenate(rows))
    bad = s[0].clone()
    bad[7] = mesh.nv + 3
    with pytest.raises(S.SsdfError):
        capi.triangles_meeting_boxes(bad, s[1], s[2], *sv, torch.tensor(boxes, device="cuda"))


def one_rank_comm():
    """A one-rank NCCL communicator on the current device (this machine gives one GPU)."""
    import ctypes as C

    import torch

    torch.cuda.init()
    nccl = C.CDLL("libnccl.so.2")

    class UniqueId(C.Structure):
        _fields_ = [("internal", C.c_char * 128)]

    uid = UniqueId()
    assert nccl.ncclGetUniqueId(C.byref(uid)) == 0
    comm = C.c_void_p()
    assert nccl.ncclCommInitRank(C.byref(comm), 1, uid, 0) == 0
    return nccl, comm


@pytest.mark.parametrize("gt", [(np.float64, np.float64), (np.float32, np.float64), (np.float32, np.float32)])
@pytest.mark.parametrize("allgather", ["1", "0"])
def test_pedf_over_nccl_c_abi(gt, allgather, monkeypatch):
    """ssdf_pedf_nccl / ssdf_pedf_update_nccl (the C ABI under include/ssdf_distributed.hpp) on one rank:
    pedf equals the drop-in edf_bvh on the whole surface bit for bit, in both modes and every type pair,
    the incoming out kept where smaller; pedf_update from upper bounds gives the same values."""
    import ctypes as C

    import torch

    gdt, tdt = gt
    monkeypatch.setenv("SSDF_USE_ALLGATHER", allgather)
    mesh = W.torus(0.7, 0.25, nu=60, nv=30, jitter=0.01, seed=2)
    lo, hi = mesh.bbox()
    pts = W.uniform_points(7001, lo - 0.3, hi + 0.3, seed=12).astype(gdt)
    init = np.where(np.arange(7001) % 5 == 0, 0.02, np.finfo(tdt).max).astype(tdt)
    want = S.edf_bvh(pts, mesh, out=init, gdtype=gdt, tdtype=tdt)
    td = {np.float64: torch.float64, np.float32: torch.float32}
    x, y, z = (torch.tensor(np.ascontiguousarray(a), device="cuda") for a in pts)
    s0, s1, s2 = (torch.tensor(np.ascontiguousarray(a, dtype=np.int32), device="cuda") for a in mesh.indices())
    sx, sy, sz = (torch.tensor(np.ascontiguousarray(a, dtype=gdt), device="cuda") for a in mesh.coords())
    ct = S.F64 if gdt == np.float64 else S.F32
    ot = S.F64 if tdt == np.float64 else S.F32
    nccl, comm = one_rank_comm()
    stream = torch.cuda.current_stream().cuda_stream
    try:
        for fn, start in (("ssdf_pedf_nccl", init), ("ssdf_pedf_update_nccl", (want * 1.5).astype(tdt))):
            expect = S.edf_bvh(pts, mesh, out=start, gdtype=gdt, tdtype=tdt)
            out = torch.tensor(start, dtype=td[tdt], device="cuda")
            st = getattr(S.lib, fn)(comm, x.numel(), x.data_ptr(), y.data_ptr(), z.data_ptr(), s0.numel(),
                                    s0.data_ptr(), s1.data_ptr(), s2.data_ptr(), sx.numel(), sx.data_ptr(),
                                    sy.data_ptr(), sz.data_ptr(), ct, ot, out.data_ptr(), C.c_void_p(stream))
            assert st == S.SSDF_OK, S.last_error()
            # pedf_update from bounds 1.5x the answer: every triangle that can improve them is exchanged
            assert np.array_equal(out.cpu().numpy(), expect), fn
    finally:
        nccl.ncclCommDestroy(comm)
