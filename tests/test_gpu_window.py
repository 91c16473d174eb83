"""GPU: the fix-up path's second stage -- queries whose float window holds more near-tied triangles
than the window slots -- bitwise against the plain double result and the oracle.

Grid nodes within 2e-5 of the centre of an undisplaced icosphere are nearly equidistant from
dozens of triangles (the icosahedral symmetry makes exact ties), so every one of them overflows
and is answered by the warp-per-query walk. SSDF_B200_WINDOW_STACK lowers that walk's shared stack
so the lanes' own subtree walks run too. In a batch, such jobs sit among ordinary ones.
"""

import os

import numpy as np
import pytest
import torch

import oracle
import ssdf_b200 as S
from ssdf_b200 import workloads as W
from test_gpu_golden import env

pytestmark = pytest.mark.gpu


def centre_grid(n=16, r=2e-5):
    return W.Grid((n, n, n), (-r, -r, -r), (r, r, r))


def run(dm, grid, prec, stack=None):
    out = torch.empty(grid.size, dtype=torch.float64, device="cuda")
    tri = torch.empty(grid.size, dtype=torch.int32, device="cuda")
    env = {"SSDF_B200_COUNT": "1"}
    if stack is not None:
        env["SSDF_B200_WINDOW_STACK"] = str(stack)
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        dm.query_grid(grid, out, tri, precision=prec, output=S.OUT_SDF)
        torch.cuda.synchronize()
        counts = S.last_query_counts()
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v
    return out.cpu().numpy(), tri.cpu().numpy(), counts


@pytest.mark.parametrize("sub", [2, 4])
@pytest.mark.parametrize("stack", [None, 40, 1])
def test_overflowed_windows_match_double(sub, stack):
    mesh = W.icosphere(sub, radius=1.0, displacement=0.0)
    grid = centre_grid()
    dm = S.DeviceMesh(mesh)
    d, t, c = run(dm, grid, S.PREC_F32_FIXUP, stack)
    d64, t64, _ = run(dm, grid, S.PREC_F64)
    dm.close()
    assert c["fallback_queries"] > grid.size // 2, c  # the second stage answered most of them
    assert np.array_equal(d, d64) and np.array_equal(t, t64)
    want, wtri = oracle.sdf_points(oracle.grid_points(grid), mesh)
    assert np.array_equal(d, want) and np.array_equal(t, wtri)
    assert np.all(d < 0)  # the centre is inside


def test_batch_with_overflowing_jobs():
    jobs = []
    for k in range(12):
        if k % 3 == 0:
            m = W.icosphere(2 + k % 4, radius=0.5 + 0.1 * k, displacement=0.0)
            jobs.append((m, centre_grid(8 + k)))
        else:
            m = W.torus(0.7, 0.2, nu=24 + 8 * k, nv=12 + 2 * k, jitter=0.01, seed=k)
            jobs.append((m, W.Grid.padded_nodes(m, 20 + 3 * k, 0.1)))
    dms = [S.DeviceMesh(m) for m, _ in jobs]
    outs = [torch.empty(g.size, dtype=torch.float64, device="cuda") for _, g in jobs]
    tris = [torch.empty(g.size, dtype=torch.int32, device="cuda") for _, g in jobs]
    for use_graph in (False, True):
        b = S.Batch(len(jobs), S.PREC_F32_FIXUP)
        for dm, (m, g), o, t in zip(dms, jobs, outs, tris):
            b.add_grid(dm, g, o, t)
        b.run(use_graph=use_graph)
        torch.cuda.synchronize()
        b.close()
        for dm, (m, g), o, t in zip(dms, jobs, outs, tris):
            d64, t64, _ = run(dm, g, S.PREC_F64)
            assert np.array_equal(o.cpu().numpy(), d64) and np.array_equal(t.cpu().numpy(), t64)
    for dm in dms:
        dm.close()


def sliver_mesh(sub, height):
    """An icosphere whose every triangle (a, b, c) is split at a point m just off the middle of ab:
    (a, m, c), (m, b, c) and the sliver (a, b, m) of relative height `height`."""
    base = W.icosphere(sub, radius=1.0, displacement=0.01, seed=4)
    v = list(base.vertices)
    tris = []
    for a, b, c in base.triangles:
        pa, pb, pc = base.vertices[a], base.vertices[b], base.vertices[c]
        m = 0.5 * (pa + pb) + height * np.linalg.norm(pb - pa) * (pc - 0.5 * (pa + pb)) / np.linalg.norm(pc - 0.5 * (pa + pb))
        v.append(m)
        im = len(v) - 1
        tris += [(a, im, c), (im, b, c), (a, b, im)]
    return W.Mesh(np.array(v), np.array(tris, dtype=np.int32))


@pytest.mark.parametrize("height", [1e-3, 1e-6, 0.0])
def test_slivers_fixup_equals_double(height):
    """Ill-conditioned triangles (needles, slivers, collinear) are filtered through well-conditioned
    proxies in the fix-up path, so its result stays the double one at every query. A third of this
    mesh is slivers, so the proxy path is forced (SSDF_B200_ILL_MAX above 1)."""
    mesh = sliver_mesh(2, height)
    dm = S.DeviceMesh(mesh)
    lo, hi = mesh.bbox()
    grid = W.Grid((40, 40, 40), tuple(lo - 0.3), tuple(hi + 0.3))
    res = {}
    for prec in (S.PREC_F32_FIXUP, S.PREC_F64):
        out = torch.full((grid.size,), np.finfo(np.float64).max, dtype=torch.float64, device="cuda")
        tri = torch.full((grid.size,), -1, dtype=torch.int32, device="cuda")
        with env(SSDF_B200_ILL_MAX=2, SSDF_B200_COUNT=1):
            dm.query_grid(grid, out, tri, precision=prec, output=S.OUT_EDF)
            torch.cuda.synchronize()
        if prec == S.PREC_F32_FIXUP:
            assert S.last_query_counts()["fixup_evaluations"] > 0  # the fix-up kernel ran
        res[prec] = (out.cpu().numpy(), tri.cpu().numpy())
    dm.close()
    assert np.array_equal(res[S.PREC_F32_FIXUP][0], res[S.PREC_F64][0])
    assert np.array_equal(res[S.PREC_F32_FIXUP][1], res[S.PREC_F64][1])
    ids = np.random.default_rng(0).choice(grid.size, 500, replace=False)
    want, wtri = oracle.edf(oracle.grid_points(grid)[:, ids], mesh, with_index=True)
    assert np.array_equal(res[S.PREC_F64][0][ids], want) and np.array_equal(res[S.PREC_F64][1][ids], wtri)


def test_sliver_heavy_mesh_is_handed_to_fp64():
    """A mesh with more than the limit's share of ill-conditioned triangles (a third here; the limit is
    a half by default, set to a fifth) answers fix-up requests with the FP64 kernel (no fix-up
    evaluations), with the same bits; below the limit the fix-up kernel runs."""
    mesh = sliver_mesh(2, 1e-3)
    dm = S.DeviceMesh(mesh)
    lo, hi = mesh.bbox()
    grid = W.Grid((32, 32, 32), tuple(lo - 0.3), tuple(hi + 0.3))
    outs = []
    for limit in (0.2, None):
        out = torch.empty(grid.size, dtype=torch.float64, device="cuda")
        kw = dict(SSDF_B200_COUNT=1) if limit is None else dict(SSDF_B200_COUNT=1, SSDF_B200_ILL_MAX=limit)
        with env(**kw):
            dm.query_grid(grid, out, None, precision=S.PREC_F32_FIXUP, output=S.OUT_SDF)
            torch.cuda.synchronize()
        outs.append(out.cpu().numpy())
        c = S.last_query_counts()["fixup_evaluations"]
        assert (c == 0) if limit is not None else (c > 0)
    dm.close()
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("arity", [2, 4])
@pytest.mark.parametrize("budget", [8, 64, 0])
def test_packet_budget_hands_queries_to_second_stage(budget, arity):
    """A warp packet that has tested more triangle records than SSDF_B200_WARP_BUDGET stops and hands
    its queries, with their current windows, to the warp-per-query stage: the result stays the FP64
    one at every node (single launch and batch), and small budgets do send queries there. Both the
    binary and the 4-wide packet walks."""
    mesh = W.icosphere(4)
    lo, hi = mesh.bbox()
    grid = W.Grid((48, 40, 36), tuple(lo - 0.3), tuple(hi + 0.3))
    dm = S.DeviceMesh(mesh)
    ref = torch.empty(grid.size, dtype=torch.float64, device="cuda")
    rtri = torch.empty(grid.size, dtype=torch.int32, device="cuda")
    dm.query_grid(grid, ref, rtri, precision=S.PREC_F64)
    out = torch.empty_like(ref)
    tri = torch.empty_like(rtri)
    with env(SSDF_B200_WARP_BUDGET=budget, SSDF_B200_COUNT=1, SSDF_B200_ARITY=arity):
        dm.query_grid(grid, out, tri, precision=S.PREC_F32_FIXUP)
        torch.cuda.synchronize()
        fb = S.last_query_counts()["fallback_queries"]
    assert torch.equal(out, ref) and torch.equal(tri, rtri)
    assert (fb > grid.size // 10) if budget == 8 else True
    bout = torch.empty_like(ref)
    with env(SSDF_B200_WARP_BUDGET=budget, SSDF_B200_ARITY=arity):
        b = S.Batch(4, S.PREC_F32_FIXUP)
        b.add_grid(dm, grid, bout)
        b.run(use_graph=False)
        torch.cuda.synchronize()
        b.close()
    assert torch.equal(bout, ref)
    dm.close()
