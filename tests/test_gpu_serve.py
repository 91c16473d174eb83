"""GPU: the serving loop (ssdf_server_*): continuous batching, LRU admission under a memory budget.

Each request's result is the same alone and in the mix -- bitwise, since a batched job runs the
same kernel as an alone query -- while requests from several threads arrive during other batches,
meshes are evicted and rebuilt, and batches hold requests of very different sizes.
"""

import threading
import time

import numpy as np
import pytest

import ssdf_b200 as S
from ssdf_b200 import workloads as W

pytestmark = pytest.mark.gpu


def meshes():
    out = []
    for k in range(6):
        c = (0.3 * k, -0.2 * k, 0.1 * k)
        if k % 2 == 0:
            out.append(W.icosphere(2 + k // 2, radius=0.6, seed=k, center=c))
        else:
            out.append(W.torus(0.7, 0.2, nu=24 + 16 * k, nv=12 + 4 * k, jitter=0.01, seed=k, center=c))
    return out


def requests(ms, seed=0):
    rng = np.random.default_rng(seed)
    reqs = []
    for r in range(36):
        mid = int(rng.integers(len(ms)))
        m = ms[mid]
        lo, hi = m.bbox()
        if rng.uniform() < 0.5:
            side = int(rng.integers(8, 40))
            reqs.append(("grid", mid, W.Grid.padded_nodes(m, side, 0.1)))
        else:
            n = int(np.exp(rng.uniform(np.log(50), np.log(60000))))
            reqs.append(("points", mid, W.uniform_points(n, lo - 0.1, hi + 0.1, seed=1000 + r)))
    return reqs


def alone(ms, req):
    kind, mid, q = req
    if kind == "grid":
        return S.sample_sdf_bvh(ms[mid], q, with_index=True)
    return S.sdf_points(q, ms[mid])


def test_results_same_alone_and_in_the_mix():
    ms = meshes()
    reqs = requests(ms)
    want = [alone(ms, r) for r in reqs]
    sizes = []
    for m in ms:
        dm = S.DeviceMesh(m)
        sizes.append(dm.stats()["bytes"])
        dm.close()
    # a budget of about two meshes forces evictions and rebuilds
    srv = S.Server(memory_budget=int(sorted(sizes)[-1] * 2.2), max_batch_queries=1 << 20, max_batch_jobs=16)
    ids = [srv.add_mesh(m) for m in ms]
    got = [None] * len(reqs)
    errors = []

    def client(part):
        try:
            rng = np.random.default_rng(part)
            tickets = []
            for i in range(part, len(reqs), 4):
                kind, mid, q = reqs[i]
                t = srv.submit_grid(ids[mid], q) if kind == "grid" else srv.submit_points(ids[mid], q)
                tickets.append((i, t))
                time.sleep(float(rng.uniform(0, 0.004)))
            for i, t in tickets:
                got[i] = srv.wait(t)
        except Exception as ex:  # surfaced below
            errors.append(ex)

    threads = [threading.Thread(target=client, args=(p,)) for p in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for (d, tri), (wd, wtri) in zip(got, want):
        assert np.array_equal(d, wd)
        assert np.array_equal(tri, wtri)
    st = srv.stats()
    assert st["completed"] == len(reqs)
    assert st["evictions"] > 0 and st["builds"] > len(ms)
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    # a burst is packed: requests waiting while a batch runs share the next one
    srv.reset_stats()
    burst = [srv.submit_points(ids[1], reqs[i][2]) for i in range(len(reqs)) if reqs[i][0] == "points"]
    for t in burst:
        srv.wait(t)
    st = srv.stats()
    assert st["completed"] == len(burst) and st["batches"] < len(burst)
    srv.close()


def test_rejects_oversized_and_unknown():
    """A grid whose z-plane alone exceeds a batch cannot be split into slabs and is refused; larger
    requests are otherwise answered in parts (8,000 nodes through 1,000-query batches here)."""
    mesh = W.icosphere(1)
    srv = S.Server(max_batch_queries=1000, max_batch_jobs=4)
    mid = srv.add_mesh(mesh)
    with pytest.raises(S.SsdfError):
        srv.submit_grid(mid, W.Grid((40, 40, 3), (0, 0, 0), (1, 1, 1)))  # 1,600 nodes a plane
    g = W.Grid((20, 20, 20), (-1, -1, -1), (1, 1, 1))
    d, tri = srv.wait(srv.submit_grid(mid, g))
    wd, wt = S.sample_sdf_bvh(mesh, g, with_index=True)
    assert np.array_equal(d, wd) and np.array_equal(tri, wt)
    with pytest.raises(S.SsdfError):
        srv.submit_points(mid + 5, np.zeros((3, 10)))
    srv.close()
    with pytest.raises(S.SsdfError):
        S.Server(slots=17)


@pytest.mark.parametrize("slots", [1, 2, 6])
def test_slot_counts_give_the_same_results(slots):
    ms = meshes()[:3]
    reqs = requests(ms, seed=4)[:12]
    want = [alone(ms, r) for r in reqs]
    srv = S.Server(max_batch_queries=1 << 18, max_batch_jobs=4, slots=slots)
    ids = [srv.add_mesh(m) for m in ms]
    tickets = [srv.submit_grid(ids[mid], q) if kind == "grid" else srv.submit_points(ids[mid], q)
               for kind, mid, q in reqs]
    for t, (wd, wtri) in zip(tickets, want):
        d, tri = srv.wait(t)
        assert np.array_equal(d, wd) and np.array_equal(tri, wtri)
    assert srv.stats()["completed"] == len(reqs)
    srv.close()


def test_split_requests_equal_unsplit():
    """Requests larger than split_queries are answered in parts (z-slabs of a grid, runs of a point
    list) packed round-robin with other requests; every value equals the request alone, bit for bit."""
    ms = meshes()
    reqs = requests(ms, seed=4)
    big_grid = ("grid", 1, W.Grid.padded_nodes(ms[1], 53, 0.1))  # 148,877 nodes: 19 slabs of 2809 x 3 planes
    big_pts = ("points", 3, W.uniform_points(70001, *(np.array(ms[3].bbox()) + [[-0.1], [0.1]]), seed=77))
    reqs = [big_grid] + reqs[:10] + [big_pts] + reqs[10:20]
    want = [alone(ms, r) for r in reqs]
    srv = S.Server(memory_budget=1 << 30, max_batch_queries=1 << 17, max_batch_jobs=32, split_queries=9000, slots=3)
    ids = [srv.add_mesh(m) for m in ms]
    tickets = [srv.submit_grid(ids[mid], q) if kind == "grid" else srv.submit_points(ids[mid], q)
               for kind, mid, q in reqs]
    for t, (wd, wt) in zip(tickets, want):
        d, tri = srv.wait(t)
        assert np.array_equal(d, wd) and np.array_equal(tri, wt)
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["rejected"] == 0
    srv.close()


def test_admission_limit_refuses_with_busy():
    """Past the queued-query limit a submit returns SSDF_ERR_BUSY at once; the accepted requests are
    answered exactly, and the refusals are counted."""
    ms = meshes()
    srv = S.Server(memory_budget=1 << 30, max_batch_queries=1 << 16, max_batch_jobs=8, slots=1,
                   max_queued_queries=60000)
    ids = [srv.add_mesh(m) for m in ms]
    grid = W.Grid.padded_nodes(ms[0], 30, 0.1)  # 27,000 queries
    want = alone(ms, ("grid", 0, grid))
    accepted, busy = [], 0
    for _ in range(40):
        try:
            accepted.append(srv.submit_grid(ids[0], grid))
        except S.SsdfError as e:
            assert e.status == S.SSDF_ERR_BUSY
            busy += 1
    assert busy > 0 and accepted
    for t in accepted:
        d, tri = srv.wait(t)
        assert np.array_equal(d, want[0]) and np.array_equal(tri, want[1])
    st = srv.stats()
    assert st["rejected"] == busy and st["completed"] == len(accepted)
    # once the queue has drained, requests are accepted again
    t = srv.submit_grid(ids[0], grid)
    srv.wait(t)
    srv.close()
