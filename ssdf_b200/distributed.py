"""ssdf's distributed point-to-surface distance over torch.distributed: ``pedf`` and
``pedf_update`` (distributed/psdf.hpp:149-302 and 303-482), one process per GPU, the exchanges as
NCCL collectives over NVLink and the distances on this library's device BVH.

Every rank holds a part of the query points and a part of the surface (triangles indexing its own
vertices). ``out`` is in/out, as in ``ssdf::edf``: on entry the current best unsigned distance of
each local point, on exit the smaller of that and the distance to the union of all ranks' surface
parts.

* ``pedf`` with ``use_allgather`` (the reference's default, ``SSDF_USE_ALLGATHER=1``): the surface
  parts are gathered on every rank, each part's vertex indices shifted by the vertex counts of the
  ranks before it (psdf.hpp:181-245), and the local points are queried once against the whole
  surface.
* ``pedf`` without it (``SSDF_USE_ALLGATHER=0``): each rank's part in turn is broadcast and queried,
  the in/out value carrying the minimum from one part to the next (psdf.hpp:246-298).
* ``pedf_update``: every rank publishes the box of its points grown by their current distances
  (psdf.hpp:323-385) and receives from every rank the triangles whose box meets it, sent as unindexed
  corner triples; the local points are then queried in/out against those. Only triangles that could
  improve a distance travel.

The query is the library's edf dispatch: double outputs on the FP32-with-FP64-fix-up path (bitwise
the double result), float outputs in the reference's float arithmetic. Tensors live on the rank's
GPU (``torch.cuda.current_device()``); with the gloo backend the collectives also take CPU tensors,
which is how the exchange steps are tested without GPUs.
"""

from __future__ import annotations

import os

from . import capi


def _dist():
    import torch.distributed as dist

    return dist


def _world(group):
    dist = _dist()
    return dist.get_world_size(group), dist.get_rank(group)


def _gather_sizes(n: int, device, group) -> list:
    """Every rank's count (all-gather of one int64)."""
    import torch

    world, _ = _world(group)
    mine = torch.tensor([int(n)], dtype=torch.int64, device=device)
    got = [torch.zeros(1, dtype=torch.int64, device=device) for _ in range(world)]
    _dist().all_gather(got, mine, group=group)
    return [int(t.item()) for t in got]


def _gather_var(t, sizes, group):
    """All-gather of a tensor whose first dimension differs between ranks (padded to the largest,
    then trimmed), concatenated in rank order."""
    import torch

    m = max(sizes) if sizes else 0
    pad = torch.zeros((m,) + tuple(t.shape[1:]), dtype=t.dtype, device=t.device)
    pad[: t.shape[0]] = t
    parts = [torch.empty_like(pad) for _ in sizes]
    _dist().all_gather(parts, pad, group=group)
    return torch.cat([p[:n] for p, n in zip(parts, sizes)])


def gather_surface(s0, s1, s2, sx, sy, sz, group=None):
    """The union of every rank's surface part on every rank: (s0, s1, s2, sx, sy, sz), indices shifted
    by the vertex counts of the ranks before (psdf.hpp:181-240)."""
    import torch

    device = sx.device
    nv = _gather_sizes(sx.numel(), device, group)
    nt = _gather_sizes(s0.numel(), device, group)
    _, rank = _world(group)
    shift = int(sum(nv[:rank]))
    idx = torch.stack([s0, s1, s2], 1).to(torch.int32) + shift
    gidx = _gather_var(idx, nt, group)
    gv = _gather_var(torch.stack([sx, sy, sz], 1), nv, group)
    return (gidx[:, 0].contiguous(), gidx[:, 1].contiguous(), gidx[:, 2].contiguous(), gv[:, 0].contiguous(),
            gv[:, 1].contiguous(), gv[:, 2].contiguous())


def surface_parts(s0, s1, s2, sx, sy, sz, group=None):
    """Every rank's surface part in rank order, broadcast by its owner (psdf.hpp:254-283): yields
    (root, s0, s1, s2, sx, sy, sz) with the root's own numbering; empty parts are skipped."""
    import torch

    dist = _dist()
    world, rank = _world(group)
    device = sx.device
    for root in range(world):
        sizes = torch.tensor([s0.numel(), sx.numel()] if rank == root else [0, 0], dtype=torch.int64, device=device)
        dist.broadcast(sizes, dist.get_global_rank(group, root) if group is not None else root, group=group)
        nt, nv = int(sizes[0].item()), int(sizes[1].item())
        if nt == 0 or nv == 0:
            continue
        src = dist.get_global_rank(group, root) if group is not None else root
        if rank == root:
            idx = torch.stack([s0, s1, s2], 1).to(torch.int32).contiguous()
            v = torch.stack([sx, sy, sz], 1).contiguous()
        else:
            idx = torch.empty((nt, 3), dtype=torch.int32, device=device)
            v = torch.empty((nv, 3), dtype=sx.dtype, device=device)
        dist.broadcast(idx, src, group=group)
        dist.broadcast(v, src, group=group)
        yield (root, idx[:, 0].contiguous(), idx[:, 1].contiguous(), idx[:, 2].contiguous(), v[:, 0].contiguous(),
               v[:, 1].contiguous(), v[:, 2].contiguous())


def _precision(out) -> int:
    import torch

    v = os.environ.get("SSDF_B200_PRECISION")
    if v in ("f64",):
        return capi.PREC_F64
    if v in ("f32",):
        return capi.PREC_F32
    if v in ("f32x", "fixup"):
        return capi.PREC_F32_FIXUP
    return capi.PREC_F32_FIXUP if out.dtype == torch.float64 else capi.PREC_F32


def edf_inout(x, y, z, out, s0, s1, s2, sx, sy, sz, stream=None):
    """out = min(out, unsigned distance of (x, y, z) to the triangles (s0, s1, s2) over (sx, sy, sz)),
    all device tensors, on this library's BVH (the drop-in edf's arithmetic for out's dtype)."""
    if s0.numel() == 0 or sx.numel() == 0 or x.numel() == 0:
        return out
    prec = _precision(out)
    dm = capi.DeviceMesh.from_device(s0.to(dtype=_i32()).contiguous(), s1.to(dtype=_i32()).contiguous(),
                                     s2.to(dtype=_i32()).contiguous(), sx.contiguous(), sy.contiguous(),
                                     sz.contiguous(), keep_fp64=prec != capi.PREC_F32, normals=False, stream=stream)
    try:
        dm.query_points(x, y, z, out, precision=prec, output=capi.OUT_EDF, coord_type=capi._dtype_code(x),
                        out_type=capi._dtype_code(out), stream=stream)
    finally:
        _sync(stream)
        dm.close()
    return out


def _i32():
    import torch

    return torch.int32


def _sync(stream):
    import torch

    if stream is None:
        torch.cuda.synchronize()
    else:
        stream.synchronize()


def _use_allgather(flag) -> bool:
    if flag is not None:
        return bool(flag)
    return int(os.environ.get("SSDF_USE_ALLGATHER", "1")) != 0


def pedf(x, y, z, s0, s1, s2, sx, sy, sz, out, group=None, use_allgather=None, stream=None):
    """ssdf::pedf (distributed/psdf.hpp:149-302): out = min(out, distance of this rank's points to the
    union of every rank's surface part). Device tensors; every rank calls it (collective)."""
    if _use_allgather(use_allgather):
        g = gather_surface(s0, s1, s2, sx, sy, sz, group)
        return edf_inout(x, y, z, out, *g, stream=stream)
    for _root, *part in surface_parts(s0, s1, s2, sx, sy, sz, group):
        edf_inout(x, y, z, out, *part, stream=stream)
    return out


def update_candidates(x, y, z, out, s0, s1, s2, sx, sy, sz, group=None, select=None):
    """The triangles every rank sends this one for pedf_update: each rank's local triangles whose box
    meets this rank's grown point box (psdf.hpp:327-470), as corner triples [m, 9] (x0 y0 z0 x1 ... z2)
    in the coordinates' type, in rank order. The grown box and the selection run on the device
    (ssdf_grown_box, ssdf_triangles_meeting_boxes); `select` = (grown_box, meeting) replaces them with
    host functions of the same contract, for exchange tests on CPU process groups."""
    import torch

    from . import capi

    grown, meeting = select if select is not None else (capi.grown_box, capi.triangles_meeting_boxes)
    dist = _dist()
    world, rank = _world(group)
    box = grown(x, y, z, out)
    boxes = [torch.empty_like(box) for _ in range(world)]
    dist.all_gather(boxes, box, group=group)
    corners, per_rank = meeting(s0, s1, s2, sx, sy, sz, torch.stack(boxes))
    counts = torch.tensor(per_rank, dtype=torch.int64, device=sx.device)
    recv = torch.empty_like(counts)
    dist.all_to_all_single(recv, counts, group=group)
    out_sizes, in_sizes = [int(v) for v in recv.tolist()], [int(v) for v in counts.tolist()]
    got = torch.empty((sum(out_sizes), 9), dtype=sx.dtype, device=sx.device)
    dist.all_to_all_single(got, corners.contiguous(), output_split_sizes=out_sizes, input_split_sizes=in_sizes,
                           group=group)
    return got


def pedf_update(x, y, z, s0, s1, s2, sx, sy, sz, out, group=None, stream=None):
    """ssdf::pedf_update (distributed/psdf.hpp:303-482): like pedf, but each rank receives only the
    triangles that can improve its points' current distances (those meeting the box of its points
    grown by `out`); `out` must hold upper bounds (for instance a previous pedf result)."""
    import torch

    tri = update_candidates(x, y, z, out, s0, s1, s2, sx, sy, sz, group)
    if tri.shape[0] == 0:
        return out
    m = tri.shape[0]
    v = tri.reshape(m * 3, 3)
    ids = torch.arange(3 * m, dtype=torch.int32, device=tri.device).reshape(m, 3)
    return edf_inout(x, y, z, out, ids[:, 0].contiguous(), ids[:, 1].contiguous(), ids[:, 2].contiguous(),
                     v[:, 0].contiguous(), v[:, 1].contiguous(), v[:, 2].contiguous(), stream=stream)
