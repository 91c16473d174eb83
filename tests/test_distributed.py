"""The exchange steps of pedf / pedf_update (ssdf_b200/distributed.py) with two and three gloo
ranks on CPU: the gathered surface (indices shifted by the vertex counts of the ranks before), the
parts broadcast in rank order, and the candidate triangles each rank receives for pedf_update
against a brute-force selection of every rank's triangles meeting its grown point box. The ranks have
no GPU, so the device selection steps (tests/test_gpu_distributed.py checks them) are replaced by
host stand-ins of the same contract; what runs here is the exchange."""

import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_data(rank, seed=5):
    """Rank r's points, current distances and surface part (its own vertex numbering); rank 1's
    surface part is empty when seed is odd."""
    rng = np.random.default_rng(seed * 100 + rank)
    npts = int(rng.integers(0, 40)) if rank == 2 else int(rng.integers(5, 40))
    pts = rng.uniform(-1, 1, size=(3, npts)) + 0.5 * rank
    out = rng.uniform(0.05, 0.4, size=npts)
    nv = 0 if (rank == 1 and seed % 2) else int(rng.integers(3, 30))
    verts = rng.uniform(-1, 1, size=(3, nv)) + 0.7 * rank
    nt = 0 if nv == 0 else int(rng.integers(1, 25))
    tris = rng.integers(0, max(nv, 1), size=(3, nt)).astype(np.int32)
    return pts, out, tris, verts


def host_grown_box(x, y, z, out):
    """Stand-in for ssdf_grown_box on CPU tensors (the exchange tests run gloo ranks without a GPU)."""
    import torch

    if x.numel() == 0:
        big = torch.finfo(x.dtype).max
        return torch.tensor([big, big, big, -big, -big, -big], dtype=x.dtype)
    r = out.to(x.dtype)
    return torch.stack([(x - r).min(), (y - r).min(), (z - r).min(), (x + r).max(), (y + r).max(), (z + r).max()])


def host_meeting(s0, s1, s2, sx, sy, sz, boxes):
    """Stand-in for ssdf_triangles_meeting_boxes on CPU tensors: corners of the triangles meeting each
    box, box after box, and the count per box."""
    import torch

    if s0.numel() == 0:
        return torch.zeros((0, 9), dtype=sx.dtype), [0] * boxes.shape[0]
    corners = torch.stack([sx[s0.long()], sy[s0.long()], sz[s0.long()], sx[s1.long()], sy[s1.long()], sz[s1.long()],
                           sx[s2.long()], sy[s2.long()], sz[s2.long()]], 1)
    tlo = torch.stack([corners[:, d::3].min(1).values for d in range(3)], 1)
    thi = torch.stack([corners[:, d::3].max(1).values for d in range(3)], 1)
    parts = [corners[~((thi < b[:3]) | (tlo > b[3:])).any(1)] for b in boxes]
    return torch.cat(parts), [p.shape[0] for p in parts]


def _rank(rank, world, port, seed, results):
    import torch
    import torch.distributed as dist

    from ssdf_b200 import distributed as D

    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}")
    try:
        pts, out, tris, verts = rank_data(rank, seed)
        t = [torch.from_numpy(np.ascontiguousarray(a)) for a in (*pts, *tris, *verts)]
        x, y, z, s0, s1, s2, sx, sy, sz = t
        g = D.gather_surface(s0, s1, s2, sx, sy, sz)
        parts = [(root, *[a.numpy().copy() for a in p]) for root, *p in D.surface_parts(s0, s1, s2, sx, sy, sz)]
        cand = D.update_candidates(x, y, z, torch.from_numpy(out), s0, s1, s2, sx, sy, sz,
                                   select=(host_grown_box, host_meeting))
        results[rank] = ([a.numpy().copy() for a in g], parts, cand.numpy().copy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,seed", [(2, 4), (2, 5), (3, 6), (3, 7)])
def test_exchanges(world, seed):
    import torch.multiprocessing as mp

    port = _free_port()
    manager = mp.get_context("spawn").Manager()
    results = manager.dict()
    mp.start_processes(_rank, args=(world, port, seed, results), nprocs=world, start_method="spawn", join=True)
    data = [rank_data(r, seed) for r in range(world)]
    # gathered surface: the same on every rank, parts concatenated with shifted indices
    shift = np.cumsum([0] + [d[3].shape[1] for d in data])
    want_idx = np.concatenate([d[2] + shift[r] for r, d in enumerate(data)], axis=1)
    want_v = np.concatenate([d[3] for d in data], axis=1)
    for r in range(world):
        g = results[r][0]
        assert np.array_equal(np.stack(g[:3]), want_idx) and np.array_equal(np.stack(g[3:]), want_v)
    # broadcast parts: every non-empty part, in rank order, in its owner's numbering
    for r in range(world):
        parts = results[r][1]
        owners = [p[0] for p in parts]
        assert owners == [o for o, d in enumerate(data) if d[2].shape[1] and d[3].shape[1]]
        for root, a0, a1, a2, vx, vy, vz in parts:
            assert np.array_equal(np.stack([a0, a1, a2]), data[root][2])
            assert np.array_equal(np.stack([vx, vy, vz]), data[root][3])
    # pedf_update candidates: every rank's triangles meeting this rank's grown point box, rank order
    for r in range(world):
        pts, out = data[r][0], data[r][1]
        if pts.shape[1]:
            lo, hi = (pts - out).min(1), (pts + out).max(1)
        else:
            big = np.finfo(np.float64).max
            lo, hi = np.full(3, big), np.full(3, -big)
        rows = []
        for src, (_, _, tris, verts) in enumerate(data):
            for t in range(tris.shape[1]):
                c = verts[:, tris[:, t]]  # 3 x 3 (axis, corner)
                if not ((c.max(1) < lo) | (c.min(1) > hi)).any():
                    rows.append(c.T.reshape(9))
        want = np.array(rows).reshape(-1, 9)
        assert np.array_equal(results[r][2], want)
