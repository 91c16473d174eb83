"""GPU: many resident meshes in one persistent launch (ssdf_batch_*), replayed as a CUDA graph.

Every job's output in the batch equals the same job queried alone (bitwise), whatever the
composition, order or replay; and the alone results are the oracle's at sampled nodes.
"""

import numpy as np
import pytest

import oracle
import ssdf_b200 as S
from ssdf_b200 import workloads as W
from test_gpu_golden import env

pytestmark = pytest.mark.gpu


def mesh_set():
    out = []
    for k, (kind, size, side) in enumerate([("ico", 2, 20), ("torus", 24, 33), ("ico", 4, 17), ("torus", 96, 40),
                                           ("ico", 3, 9), ("torus", 12, 26), ("ico", 1, 31), ("torus", 160, 12)]):
        c = (k * 0.7, -k * 0.3, 0.2 * k)
        if kind == "ico":
            m = W.icosphere(size, radius=0.5 + 0.1 * k, seed=k, center=c)
        else:
            m = W.torus(0.8, 0.25, nu=size, nv=max(6, size // 3), jitter=0.01, seed=k, center=c)
        out.append((m, W.Grid.padded_nodes(m, side, 0.1 * m.diagonal())))
    return out


@pytest.fixture(scope="module")
def jobs():
    import torch

    res = []
    for m, g in mesh_set():
        dm = S.DeviceMesh(m)
        out = torch.empty(g.size, dtype=torch.float64, device="cuda")
        tri = torch.empty(g.size, dtype=torch.int32, device="cuda")
        dm.query_grid(g, out, tri)
        torch.cuda.synchronize()
        res.append(dict(mesh=m, grid=g, dm=dm, alone=out.cpu().numpy(), alone_tri=tri.cpu().numpy()))
    return res


def test_alone_matches_oracle(jobs):
    rng = np.random.default_rng(3)
    for j in jobs[:4]:
        ids = rng.choice(j["grid"].size, size=min(400, j["grid"].size), replace=False)
        q = oracle.grid_points(j["grid"])[:, ids]
        want, wtri = oracle.sdf_points(q, j["mesh"])
        assert np.array_equal(j["alone"][ids], want) and np.array_equal(j["alone_tri"][ids], wtri)


@pytest.mark.parametrize("use_graph", [False, True])
@pytest.mark.parametrize("traversal", [0, 2])
def test_batch_equals_alone(jobs, use_graph, traversal):
    import torch

    b = S.Batch(16, S.PREC_F32_FIXUP, traversal=traversal)
    outs = []
    for j in jobs:
        out = torch.full((j["grid"].size,), -7.0, dtype=torch.float64, device="cuda")
        tri = torch.full((j["grid"].size,), -7, dtype=torch.int32, device="cuda")
        b.add_grid(j["dm"], j["grid"], out, tri)
        outs.append((out, tri))
    for rep in range(2):  # first run captures, second replays
        for out, tri in outs:
            out.fill_(-7.0)
            tri.fill_(-7)
        b.run(use_graph=use_graph)
        torch.cuda.synchronize()
        for j, (out, tri) in zip(jobs, outs):
            assert np.array_equal(out.cpu().numpy(), j["alone"])
            assert np.array_equal(tri.cpu().numpy(), j["alone_tri"])
    # a different composition (subset, other order, plus a point-list job) replays the same graph
    b.clear()
    sub = [jobs[5], jobs[0], jobs[3]]
    outs2 = []
    for j in sub:
        out = torch.empty(j["grid"].size, dtype=torch.float64, device="cuda")
        b.add_grid(j["dm"], j["grid"], out)
        outs2.append(out)
    pts = torch.tensor(oracle.grid_points(jobs[2]["grid"]), dtype=torch.float64, device="cuda")
    pout = torch.empty(pts.shape[1], dtype=torch.float64, device="cuda")
    ptri = torch.empty(pts.shape[1], dtype=torch.int32, device="cuda")
    b.add_points(jobs[2]["dm"], pts[0].contiguous(), pts[1].contiguous(), pts[2].contiguous(), pout, ptri)
    b.run(use_graph=use_graph)
    torch.cuda.synchronize()
    for j, out in zip(sub, outs2):
        assert np.array_equal(out.cpu().numpy(), j["alone"])
    assert np.array_equal(pout.cpu().numpy(), jobs[2]["alone"])
    assert np.array_equal(ptri.cpu().numpy(), jobs[2]["alone_tri"])
    b.close()


def test_batch_fp64(jobs):
    import torch

    b = S.Batch(16, S.PREC_F64)
    outs = []
    for j in jobs:
        out = torch.empty(j["grid"].size, dtype=torch.float64, device="cuda")
        b.add_grid(j["dm"], j["grid"], out)
        outs.append(out)
    b.run(use_graph=True)
    torch.cuda.synchronize()
    for j, out in zip(jobs, outs):
        assert np.array_equal(out.cpu().numpy(), j["alone"])
    b.close()


def test_batch_rejects_mixed_precision(jobs):
    import torch

    b = S.Batch(4, S.PREC_F64)
    out = torch.empty(jobs[0]["grid"].size, dtype=torch.float64, device="cuda")
    bad = S.Batch(4, S.PREC_F32_FIXUP)
    with pytest.raises(S.SsdfError):
        o = S.QueryOpts(S.PREC_F32_FIXUP, S.OUT_SDF, S.F64, S.F64)
        lo = (S.C.c_double * 3)(*jobs[0]["grid"].lo)
        hi = (S.C.c_double * 3)(*jobs[0]["grid"].hi)
        S._check(S.lib.ssdf_batch_add_grid(b._h, jobs[0]["dm"]._h, *jobs[0]["grid"].n, S.C.byref(lo), S.C.byref(hi),
                                           out.data_ptr(), None, S.C.byref(o)), "ssdf_batch_add_grid")
    b.close()
    bad.close()


def test_alternating_graph_keys_after_reserve(jobs):
    """Point-only runs in input order (thread traversal) alternating with grid runs (warp packets): each
    key keeps its own captured graph, and lists reserved up front are large enough for every run."""
    import torch

    b = S.Batch(16, S.PREC_F32_FIXUP)
    b.reserve(sum(j["grid"].size for j in jobs))
    pts = torch.tensor(oracle.grid_points(jobs[1]["grid"]), dtype=torch.float64, device="cuda")
    for rep in range(3):
        b.clear()
        if rep % 2 == 0:
            out = torch.empty(pts.shape[1], dtype=torch.float64, device="cuda")
            tri = torch.empty(pts.shape[1], dtype=torch.int32, device="cuda")
            b.add_points(jobs[1]["dm"], pts[0].contiguous(), pts[1].contiguous(), pts[2].contiguous(), out, tri)
            want = jobs[1]
        else:
            out = torch.empty(jobs[3]["grid"].size, dtype=torch.float64, device="cuda")
            tri = torch.empty(jobs[3]["grid"].size, dtype=torch.int32, device="cuda")
            b.add_grid(jobs[3]["dm"], jobs[3]["grid"], out, tri)
            want = jobs[3]
        with env(SSDF_B200_SORT_POINTS=0):
            b.run(use_graph=True)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), want["alone"])
        assert np.array_equal(tri.cpu().numpy(), want["alone_tri"])
    b.close()


def test_sorted_point_jobs_in_a_batch(jobs):
    """Point jobs of 4096 queries or more are visited in Morton order inside a batch (warp packets,
    also beside grid jobs); every result equals the same query alone, with and without the sort."""
    import torch

    rng = np.random.default_rng(11)
    for sort in (1, 0):
        b = S.Batch(16, S.PREC_F32_FIXUP)
        outs = []
        for k, n in ((1, 5000), (2, 4095), (4, 20000)):
            lo, hi = jobs[k]["mesh"].bbox()
            pts = rng.uniform(lo - 0.2, hi + 0.2, size=(n, 3)).T.copy()
            want, wtri = S.sdf_points(pts, jobs[k]["mesh"])
            p = torch.tensor(pts, dtype=torch.float64, device="cuda")
            out = torch.empty(n, dtype=torch.float64, device="cuda")
            tri = torch.empty(n, dtype=torch.int32, device="cuda")
            b.add_points(jobs[k]["dm"], p[0].contiguous(), p[1].contiguous(), p[2].contiguous(), out, tri)
            outs.append((out, tri, want, wtri))
        gout = torch.empty(jobs[3]["grid"].size, dtype=torch.float64, device="cuda")
        b.add_grid(jobs[3]["dm"], jobs[3]["grid"], gout)
        with env(SSDF_B200_SORT_POINTS=sort):
            b.run(use_graph=True)
        torch.cuda.synchronize()
        for out, tri, want, wtri in outs:
            assert np.array_equal(out.cpu().numpy(), want) and np.array_equal(tri.cpu().numpy(), wtri)
        assert np.array_equal(gout.cpu().numpy(), jobs[3]["alone"])
        b.close()


@pytest.mark.parametrize("use_graph", [False, True])
def test_sliver_mesh_in_a_fixup_batch(use_graph):
    """The beam lattice (64 % slivers) beside tori in one fix-up batch: its jobs run in the batch's
    FP64 table (the arithmetic it gets alone), every job equals the same query alone, bitwise, and
    the batch's FP64 part costs about what the beam job costs alone."""
    import torch

    beams = W.beam_lattice(nbeams=4000, seed=7)
    dmb = S.DeviceMesh(beams)
    assert not dmb.filter_info()["float_filter"]  # a fix-up request on it runs the FP64 kernel
    items = [(dmb, W.Grid.padded_nodes(beams, 40, 0.1)), (dmb, W.Grid((23, 31, 17), (0.1, 0.2, 0.0), (0.9, 0.7, 1.0)))]
    tori = []
    for k in range(5):
        m = W.torus(0.6, 0.2, nu=24 + 16 * k, nv=12 + 4 * k, jitter=0.01, seed=30 + k, center=(k, 0.0, -k))
        dm = S.DeviceMesh(m)
        assert dm.filter_info()["float_filter"]
        tori.append(dm)
        items.append((dm, W.Grid.padded_nodes(m, 24 + 4 * k, 0.1)))
    alone = []
    for dm, g in items:
        out = torch.empty(g.size, dtype=torch.float64, device="cuda")
        tri = torch.empty(g.size, dtype=torch.int32, device="cuda")
        dm.query_grid(g, out, tri, precision=S.PREC_F32_FIXUP)
        torch.cuda.synchronize()
        alone.append((out.cpu().numpy(), tri.cpu().numpy()))
    b = S.Batch(len(items), S.PREC_F32_FIXUP)
    outs = []
    for run in range(2):
        b.clear()
        outs = []
        for dm, g in (items if run == 0 else items[::-1]):
            o = torch.full((g.size,), -1.0, dtype=torch.float64, device="cuda")
            t = torch.full((g.size,), -1, dtype=torch.int32, device="cuda")
            b.add_grid(dm, g, o, t)
            outs.append((o, t))
        b.run(use_graph=use_graph)
        torch.cuda.synchronize()
        order = items if run == 0 else items[::-1]
        want = alone if run == 0 else alone[::-1]
        for (o, t), (wd, wt), (_, g) in zip(outs, want, order):
            assert np.array_equal(o.cpu().numpy(), wd) and np.array_equal(t.cpu().numpy(), wt), g.n
    # the beam grid's nodes match the oracle on a sample
    g = items[0][1]
    ids = np.arange(0, g.size, 97)
    want, wtri = oracle.sdf_points(oracle.grid_points(g)[:, ids], beams)
    assert np.array_equal(alone[0][0][ids], want) and np.array_equal(alone[0][1][ids], wtri)
    b.close()
    for dm in [dmb] + tori:
        dm.close()


def test_grid_slabs_equal_the_whole_grid():
    """ssdf_batch_add_grid_slab: z-slabs of a grid, each a job of its own, keep the whole grid's node
    coordinates, so together they equal the whole-grid query bit for bit (float grids too)."""
    import torch

    mesh = W.torus(0.8, 0.25, nu=64, nv=24, jitter=0.01, seed=9)
    dm = S.DeviceMesh(mesh)
    grid = W.Grid((37, 29, 41), (-1.2, -1.17, -0.4), (1.13, 1.2, 0.43))
    for prec, ct in ((S.PREC_F32_FIXUP, S.F64), (S.PREC_F64, S.F64), (S.PREC_F32_FIXUP, S.F32)):
        whole = torch.empty(grid.size, dtype=torch.float64, device="cuda")
        wtri = torch.empty(grid.size, dtype=torch.int32, device="cuda")
        dm.query_grid(grid, whole, wtri, precision=prec, coord_type=ct)
        out = torch.full((grid.size,), -1.0, dtype=torch.float64, device="cuda")
        tri = torch.full((grid.size,), -1, dtype=torch.int32, device="cuda")
        b = S.Batch(8, prec)
        plane = grid.n[0] * grid.n[1]
        for z0, nz in ((0, 7), (7, 1), (8, 20), (28, 13)):
            b.add_grid_slab(dm, grid, z0, nz, out[z0 * plane:(z0 + nz) * plane], tri[z0 * plane:(z0 + nz) * plane],
                            coord_type=ct)
        b.run(use_graph=False)
        torch.cuda.synchronize()
        assert torch.equal(out, whole) and torch.equal(tri, wtri)
        b.close()
    dm.close()
