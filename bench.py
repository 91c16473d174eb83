#!/usr/bin/env python
"""bench.py -- grid signed-distance queries/s on B200, against the reference's CPU cell list.

Workload (one "step"): the signed distance of a 256^3 node grid (16,777,216 queries) over the
bounding box padded by 0.25 of a closed tube swept along a (2,3) torus knot (131,072 triangles,
coordinates jittered by N(0, 1e-4)), with the closest triangle's pseudo-normal sign, in double,
computed with the FP32 traversal + FP64 fix-up kernel. Synthetic, seeded inputs (no dataset).

* ``value``: queries/s with the mesh and its BVH resident in HBM (device time of each step, CUDA
  events on the launching stream, L2 flushed between steps);
* ``fp64_plain``: the same with the plain FP64 kernel (the reference point of the 3x target);
* ``e2e``: queries/s through the drop-in C ABI (``ssdf_b200_sample_sdf_bvh_dd``) from host
  arrays, i.e. mesh upload, BVH + pseudo-normal build, query and the download of the distances
  into pinned host memory, per call, as the reference's sample_sdf_bvh does per call;
* ``roofline``: the query kernel against the measured FP32 FMA peak of this GPU (the path is
  FP32-pipe bound; its HBM traffic is the output stream), flops counted by an instrumented launch;
  ``roofline.traffic`` and ``roofline.issue`` (the share of issue slots the kernel keeps busy, the
  limit it actually meets) come from the committed ncu summary ``profiles/traffic.json``;
* ``cpu_baseline``: the reference's own OpenMP ``edf_celllist<double>`` (compiled from its sources
  into oracle/_ref) on a seeded sample of the same grid nodes, all host threads;
* ``error``: the fix-up result against the plain FP64 one at every node (distance bits and closest
  triangle), and, in the cpu_baseline leg, max / RMS error against the reference's FP64 distance on its
  sample and value / sign / index mismatches against the oracle's signed distance on part of it;
* ``e2e_pageable``: ``e2e`` into ordinary (pageable) host memory, as the reference's drivers allocate;
* ``dense`` (``--workload icosphere``): the GPU ``edf`` and ``edf_celllist`` over device arrays with
  their counted work against the measured FP64 peak (the reference's ``edf`` is timed beside
  ``edf_celllist`` in cpu_baseline).

``--impl reference`` times that reference CPU code alone. With torchrun (N > 1) every rank runs
an independent replica (the path does not shard across GPUs here: "replicas only"), the step time
is the max over ranks and ``value`` the total over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "grid SDF queries/s (FP32+FP64 fixup vs plain FP64 GPU); served p50/p99 latency"
BEAMS_METRIC = "unsigned edf queries/s (FP32, reference float arithmetic) + closest triangle"
WORKLOAD = "torus-knot tube (2,3), 131072 triangles, 256^3 node grid over bbox+0.25, signed, double"
REF_SAMPLE = 262144       # reference arm: grid nodes per step
CPU_SAMPLE = 1048576      # cpu_baseline leg of our arm


def parse_args():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", choices=["knot", "icosphere", "beams"], default="knot",
                   help="knot (default): the headline line; icosphere / beams: the other single-mesh "
                        "configurations, one line each, without the batched and serving legs")
    p.add_argument("--grid", type=int, default=None, help="grid side (default 256 knot, 64 icosphere, 512 beams)")
    p.add_argument("--cpu-sample", type=int, default=CPU_SAMPLE)
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-batch", action="store_true", help="skip the 256-mesh batched leg")
    p.add_argument("--no-dense", action="store_true", help="skip the edf / edf_celllist leg (icosphere workload)")
    p.add_argument("--no-serve", action="store_true", help="skip the serving leg")
    p.add_argument("--batch-meshes", type=int, default=256)
    p.add_argument("--serve-meshes", type=int, default=512)
    p.add_argument("--serve-seconds", type=float, default=3.0)
    p.add_argument("--serve-batch-queries", type=int, default=1 << 22, help="serving: queries per batch")
    p.add_argument("--serve-split", type=int, default=0, help="serving: parts of larger requests (0: default)")
    p.add_argument("--serve-queue", type=int, default=8 << 20, help="serving: admission limit, queued queries")
    p.add_argument("--serve-slots", type=int, default=16, help="serving: batches in flight (0: the library default, 8)")
    a = p.parse_args()
    if a.grid is None:
        a.grid = DEFAULT_GRID[a.workload]
    return a


def max_over_ranks(value, dist, device):
    """The slowest rank's time: every rank takes the same collective step (MAX all-reduce)."""
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(queries_per_rank, steps, max_ms, world):
    """Whole-job queries/s of `world` replicas, each doing `steps` steps, timed by the slowest."""
    return world * queries_per_rank * steps / (max_ms * 1e-3)


WORKLOADS = {
    "knot": WORKLOAD,
    "icosphere": "icosphere r=1 subdivided 4x (5120 triangles, 0.02 radial jitter), 64^3 cell-centred grid over "
                 "bbox+0.2, signed, double, closest triangle",
    "beams": "beam lattice (20000 beams, 240000 triangles), 8e6 uniform points in [-0.1,1.1]^3 + 512^3 grid over "
             "the same cube, unsigned float distance + int32 closest triangle",
}
DEFAULT_GRID = {"knot": 256, "icosphere": 64, "beams": 512}


def workload(n=256, name="knot"):
    from ssdf_b200 import workloads as W

    if name == "icosphere":
        mesh = W.icosphere(4)
        return mesh, W.Grid.cell_centred(mesh, n, 0.2)
    mesh = W.torus_knot_tube()
    grid = W.Grid.padded_nodes(mesh, n, 0.25)
    return mesh, grid


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(device_index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"error": "nvidia-smi unavailable"}
        time.sleep(0.3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [s.strip() for s in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"error": "no samples"}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def cpu_reference_rate(mesh, grid, nsample, seed=17, steps=1):
    """The reference's edf_celllist<double> (oracle/_ref) on a seeded sample of the grid nodes."""
    import oracle

    if not oracle.ref_available():
        raise RuntimeError("reference CPU library (oracle/_ref) is not built")
    rng = np.random.default_rng(seed)
    ids = np.sort(rng.choice(grid.size, size=min(nsample, grid.size), replace=False))
    q = oracle.grid_points(grid)[:, ids].copy()
    times = []
    vals = None
    for _ in range(steps):
        t0 = time.perf_counter()
        vals = oracle.ref_edf(q, mesh, which="celllist")
        times.append(time.perf_counter() - t0)
    return len(ids), times, ids, vals


def error_stats(got, want, diag):
    """Max / RMS absolute error of got against want and the max relative to the bbox diagonal."""
    err = np.abs(np.asarray(got, dtype=np.float64) - np.asarray(want, dtype=np.float64))
    return {"max_abs": float(err.max()) if err.size else 0.0, "rms": float(np.sqrt(np.mean(err ** 2))) if err.size else 0.0,
            "max_rel_to_bbox_diagonal": float(err.max() / diag) if err.size else 0.0}


def signed_check(S, oracle, grid, mesh, ids, gd, gt, diag):
    """Signed distances and closest triangles against the oracle at grid nodes ids (its double restatement
    of ssdf's signed sampler): value, sign and index mismatches."""
    want, wtri = oracle.sdf_points(oracle.grid_points(grid)[:, ids], mesh)
    res = error_stats(gd, want, diag)
    res.update({"nodes": int(len(ids)), "value_mismatches": int(np.sum(gd != want)),
                "sign_mismatches": int(np.sum(np.signbit(gd) != np.signbit(want))),
                "index_mismatches": int(np.sum(gt != wtri))})
    return res


def beams_workload(n=512, npoints=8_000_000):
    """Config 3: the beam lattice, seeded uniform points in [-0.1, 1.1]^3 and an n^3 node grid there."""
    from ssdf_b200 import workloads as W

    mesh = W.beam_lattice()
    pts = W.uniform_points(npoints, -0.1, 1.1, seed=23).astype(np.float32)
    grid = W.Grid((n, n, n), (-0.1, -0.1, -0.1), (1.1, 1.1, 1.1))
    return mesh, (pts, grid)


def cpu_reference_points(mesh, pts_grid, nsample, dtype, seed=17, steps=1):
    """The reference's edf_celllist<float> (oracle/_ref) on a seeded sample of the beam-lattice queries."""
    import oracle

    if not oracle.ref_available():
        raise RuntimeError("reference CPU library (oracle/_ref) is not built")
    pts, grid = pts_grid
    rng = np.random.default_rng(seed)
    half = nsample // 2
    pt_ids = np.sort(rng.choice(pts.shape[1], size=half, replace=False))
    a = pts[:, pt_ids]
    ids = np.sort(rng.choice(grid.size, size=nsample - half, replace=False))
    b = oracle.grid_points(grid, dtype=dtype)[:, ids]  # the nodes in G's arithmetic, as the GPU grid
    q = np.concatenate([a, b], axis=1).astype(dtype)
    times = []
    vals = None
    for _ in range(steps):
        t0 = time.perf_counter()
        vals = oracle.ref_edf(q, mesh, dtype=dtype, which="celllist")
        times.append(time.perf_counter() - t0)
    return q.shape[1], times, (pt_ids, ids, q, vals)


def run_beams(S, args, rank, world, dist):
    """Config 3 line: unsigned float distance + closest triangle (the reference's float arithmetic,
    SSDF_PREC_F32) at 8e6 scattered points and a 512^3 grid, one step = both sets."""
    import torch

    mesh, (pts, grid) = beams_workload(args.grid)
    dm = S.DeviceMesh(mesh, keep_fp64=False, normals=False)
    x, y, z = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in pts)
    npts, ng = x.numel(), grid.size
    nq = npts + ng
    out = torch.empty(nq, dtype=torch.float32, device="cuda")
    tri = torch.empty(nq, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    big = float(np.finfo(np.float32).max)

    def step():
        out.fill_(big)  # the in/out start value of edf (drivers/sdf.exe.cpp:330-333)
        dm.query_points(x, y, z, out[:npts], tri[:npts], precision=S.PREC_F32, output=S.OUT_EDF, coord_type=S.F32,
                        out_type=S.F32, stream=stream)
        dm.query_grid(grid, out[npts:], tri[npts:], precision=S.PREC_F32, output=S.OUT_EDF, coord_type=S.F32,
                      out_type=S.F32, stream=stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for e0, e1 in ev:
        flush.zero_()
        e0.record(stream)
        step()
        e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = [e0.elapsed_time(e1) for e0, e1 in ev]
    t = max_over_ranks(sum(ms), dist, "cuda")
    value = job_rate(nq, args.steps, t, world)
    os.environ["SSDF_B200_COUNT"] = "1"
    dm.query_points(x, y, z, out[:npts], tri[:npts], precision=S.PREC_F32, output=S.OUT_EDF, coord_type=S.F32,
                    out_type=S.F32, stream=stream)
    torch.cuda.synchronize()
    c1 = S.last_query_counts()
    dm.query_grid(grid, out[npts:], tri[npts:], precision=S.PREC_F32, output=S.OUT_EDF, coord_type=S.F32,
                  out_type=S.F32, stream=stream)
    torch.cuda.synchronize()
    c2 = S.last_query_counts()
    del os.environ["SSDF_B200_COUNT"]
    counts = {k: c1[k] + c2[k] for k in c1}
    out_keep = out.cpu().numpy()
    flops = 79.0 * counts["triangle_tests"] + 8.0 * counts["box_tests"]
    step_s = statistics.median(ms) * 1e-3
    peak = S.fma_peak_tflops(False)
    stats = dm.stats()
    alg_bytes = npts * 12 + nq * 8 + stats["bytes"]
    line = {
        "metric": BEAMS_METRIC, "value": value,
        "unit": "queries/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOADS["beams"], "queries_per_step": nq, "points": npts, "grid_nodes": ng,
                   "triangles": mesh.nt, "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                   "l2": "flushed between steps (256 MiB write); outputs 1.1 GB exceed L2"},
        "gpu_launches": 3 * args.steps,
        "roofline": {"bound": "fp32", "achieved": flops / step_s / 1e12, "peak": peak, "unit": "TFLOP/s",
                     "frac": flops / step_s / 1e12 / peak, "traffic": None,
                     "peak_source": "measured FP32 FMA microbenchmark on this GPU (ssdf_b200_fma_peak)",
                     "flops_per_step": flops, "counts": counts,
                     "hbm": {"algorithmic_bytes": alg_bytes, "achieved_gbs": alg_bytes / step_s / 1e9,
                             "peak_gbs": _hbm_peak()}},
        "clocks": clk,
        "mesh": stats,
    }
    if not args.no_e2e:
        # the drop-in host-array entry point on the scattered points (mesh upload + build + query + download),
        # the points and results in page-locked host memory
        hx, hy, hz = (torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy() for a in pts)
        hm = S.capi._HostMesh(mesh, np.float32)
        hout = torch.empty(npts, dtype=torch.float32, pin_memory=True).numpy()
        htri = torch.empty(npts, dtype=torch.int32, pin_memory=True).numpy()
        import ctypes as C

        def call():
            hout.fill(big)
            st = S.lib.ssdf_b200_edf_index_ff(npts, S.capi._p(hx), S.capi._p(hy), S.capi._p(hz), *hm.args(),
                                              S.capi._p(hout), htri.ctypes.data_as(C.POINTER(C.c_int)))
            if st != 0:
                raise RuntimeError(S.last_error())

        call()
        t0 = time.perf_counter()
        for _ in range(max(2, args.steps)):
            call()
        dt = (time.perf_counter() - t0) / max(2, args.steps)
        line["e2e"] = {"value": npts / dt, "unit": "queries/s", "h2d_bytes_per_step": int(3 * 4 * npts),
                       "d2h_bytes_per_step": int(8 * npts), "ms_per_call": dt * 1e3,
                       "api": "ssdf_b200_edf_index_ff on the 8e6 points (page-locked host arrays, blocking; wall clock)"}
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            n, times, (pt_ids, g_ids, q, ref_f) = cpu_reference_points(mesh, (pts, grid),
                                                                       min(args.cpu_sample, REF_SAMPLE), np.float32)
            line["cpu_baseline"] = {"value": n / times[0], "unit": "queries/s", "cores": os.cpu_count(),
                                    "kind": "reference",
                                    "sample": f"{n} seeded queries (half points, half grid nodes), "
                                              f"ssdf::edf_celllist<float>, oracle/_ref built from the reference's sources"}
            # error of this line's float arithmetic (the reference's own, bitwise) against double
            import oracle

            got = np.concatenate([out_keep[:npts][pt_ids], out_keep[npts:][g_ids]])
            ref_d = oracle.ref_edf(q.astype(np.float64), mesh, which="celllist")
            lo, hi = mesh.bbox()
            err = error_stats(got, ref_d, float(np.linalg.norm(hi - lo)))
            err.update({"vs": "the reference's edf_celllist<double> at the same float queries (FP64)",
                        "sample": int(n), "mismatches_vs_reference_float": int(np.sum(got != ref_f))})
            line["error"] = err
        except Exception as ex:
            line["cpu_baseline"] = {"error": repr(ex)}
    dm.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_reference(args, rank, world):
    if rank != 0:
        return
    cores = os.cpu_count()
    if args.workload == "beams":
        mesh, pts = beams_workload(args.grid)
        n, times, _ = cpu_reference_points(mesh, pts, REF_SAMPLE, np.float32, steps=args.warmup + args.steps)
        sample = f"{n} seeded queries of the beam-lattice set per step, ssdf::edf_celllist<float,float,int>"
    else:
        mesh, grid = workload(args.grid, args.workload)
        n, times, _, _ = cpu_reference_rate(mesh, grid, REF_SAMPLE, steps=args.warmup + args.steps)
        sample = (f"{n} seeded nodes of the {args.grid}^3 grid per step, ssdf::edf_celllist<double,double,int> "
                  f"(unsigned; the reference has no CPU signed grid sampler without cuBQL)")
    timed = times[args.warmup:]
    t = sum(timed)
    value = n * len(timed) / t
    line = {"impl": "reference", "metric": BEAMS_METRIC if args.workload == "beams" else METRIC, "value": value, "unit": "queries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / len(timed),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.workload == "beams" else "f64", "data": "synthetic",
            "config": {"workload": WORKLOADS[args.workload], "queries_per_step": n, "parallelism": "host threads"},
            "cpu_baseline": {"value": value, "unit": "queries/s", "cores": cores, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    import ssdf_b200 as S

    if args.workload == "beams":
        run_beams(S, args, rank, world, dist)
        return
    mesh, grid = workload(args.grid, args.workload)
    nq = grid.size
    dm = S.DeviceMesh(mesh)
    stream = torch.cuda.current_stream()
    out = torch.empty(nq, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def step(prec):
        dm.query_grid(grid, out, None, precision=prec, output=S.OUT_SDF, stream=stream)

    def barrier():
        if dist is not None:
            dist.barrier()

    def timed(prec, k, w):
        for _ in range(w):
            step(prec)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]
        for e0, e1 in ev:
            flush.zero_()  # L2 flush between steps, outside the timed events
            e0.record(stream)
            step(prec)
            e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms = [e0.elapsed_time(e1) for e0, e1 in ev]
        return max_over_ranks(sum(ms), dist, "cuda"), ms

    clocks = Clocks(local)
    t_x, ms_x = timed(S.PREC_F32_FIXUP, args.steps, args.warmup)
    clk = clocks.stop()
    value = job_rate(nq, args.steps, t_x, world)
    t_64, ms_64 = timed(S.PREC_F64, max(2, args.steps // 2), 1)
    fp64_value = world * nq * max(2, args.steps // 2) / (t_64 * 1e-3)

    # instrumented (untimed) launch: triangle / box / fix-up counts for the flop count
    os.environ["SSDF_B200_COUNT"] = "1"
    step(S.PREC_F32_FIXUP)
    torch.cuda.synchronize()
    counts = S.last_query_counts()
    del os.environ["SSDF_B200_COUNT"]
    flops = 79.0 * counts["triangle_tests"] + 8.0 * counts["box_tests"] + 79.0 * counts["fixup_evaluations"] \
        + 25.0 * nq
    step_s = statistics.median(ms_x) * 1e-3
    achieved = flops / step_s / 1e12
    peak = S.fma_peak_tflops(False)
    stats = dm.stats()
    alg_bytes = nq * 8 + stats["bytes"]
    # untimed: the fix-up result against the plain FP64 one at every node (distance bits, triangle)
    tri_x = torch.empty(nq, dtype=torch.int32, device="cuda")
    out_64 = torch.empty(nq, dtype=torch.float64, device="cuda")
    tri_64 = torch.empty(nq, dtype=torch.int32, device="cuda")
    dm.query_grid(grid, out, tri_x, precision=S.PREC_F32_FIXUP, output=S.OUT_SDF, stream=stream)
    dm.query_grid(grid, out_64, tri_64, precision=S.PREC_F64, output=S.OUT_SDF, stream=stream)
    torch.cuda.synchronize()
    vs_fp64 = {"nodes": nq, "distance_mismatches": int((out.view(torch.int64) != out_64.view(torch.int64)).sum()),
               "index_mismatches": int((tri_x != tri_64).sum())}
    del out_64, tri_64
    line = {
        "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_x / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload], "queries_per_step": nq, "triangles": mesh.nt, "parallelism":
                   f"replicas x{world}" if world > 1 else "1 GPU", "l2": "flushed between steps (256 MiB write)",
                   "precision": "FP32 traversal + FP64 fix-up (bitwise the FP64 result)"},
        "fp64_plain": {"value": fp64_value, "unit": "queries/s", "ms_per_step": t_64 / max(2, args.steps // 2),
                       "speedup_fixup_vs_fp64": value / fp64_value},
        "gpu_launches": 2 * args.steps,
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "peak_source": "measured FP32 FMA microbenchmark on this GPU (ssdf_b200_fma_peak)",
                     "traffic": None, "flops_per_launch": flops, "counts": counts,
                     "hbm": {"algorithmic_bytes": alg_bytes, "achieved_gbs": alg_bytes / step_s / 1e9,
                             "peak_gbs": _hbm_peak()}},
        "clocks": clk,
        "mesh": stats,
        "error": {"fixup_vs_fp64_every_node": vs_fp64},
    }
    if args.workload == "knot":
        _attach_traffic(line)
    if args.workload == "icosphere" and not args.no_dense:
        try:
            line["dense"] = dense_leg(S, mesh, grid, args)
        except Exception as ex:  # pragma: no cover - reported, not fatal
            line["dense"] = {"error": repr(ex)}

    if args.workload != "knot":
        args.no_batch = args.no_serve = True
    if not args.no_batch and rank == 0:
        try:
            line["batched"] = batched_leg(S, args)
        except Exception as ex:  # pragma: no cover - reported, not fatal
            line["batched"] = {"error": repr(ex)}
    if not args.no_serve and rank == 0:
        try:
            line["serving"] = serving_leg(S, args)
        except Exception as ex:  # pragma: no cover - reported, not fatal
            line["serving"] = {"error": repr(ex)}
    if not args.no_e2e:
        try:
            line["e2e"] = e2e(S, mesh, grid, args)
            line["e2e_pageable"] = e2e(S, mesh, grid, args, pageable=True)
        except Exception as ex:  # pragma: no cover - reported, not fatal
            line["e2e"] = {"error": repr(ex)}
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            n, times, ids, ref_d = cpu_reference_rate(mesh, grid, args.cpu_sample)
            line["cpu_baseline"] = {"value": n / times[0], "unit": "queries/s", "cores": os.cpu_count(),
                                    "kind": "reference",
                                    "sample": f"{n} seeded grid nodes, ssdf::edf_celllist<double> (unsigned), "
                                              f"oracle/_ref built from the reference's sources"}
            # this line's error: |distance| against the reference's own edf_celllist<double> on that
            # sample, and signs, values and triangles against the oracle on part of it
            import oracle

            gd = out.cpu().numpy()
            gt = tri_x.cpu().numpy()
            diag = mesh.diagonal()
            err = error_stats(np.abs(gd[ids]), ref_d, diag)
            err.update({"vs": "the reference's edf_celllist<double> (unsigned) at the sampled nodes", "sample": int(n),
                        "mismatches_vs_reference": int(np.sum(np.abs(gd[ids]) != ref_d))})
            sub = ids[:: max(1, len(ids) // 4096)]
            err["signed_vs_oracle"] = signed_check(S, oracle, grid, mesh, sub, gd[sub], gt[sub], diag)
            line["error"].update(err)
            if args.workload == "icosphere":  # config 1 names the reference's edf beside edf_celllist
                q = oracle.grid_points(grid)[:, ids].copy()
                t0 = time.perf_counter()
                oracle.ref_edf(q, mesh, which="edf")
                line["cpu_baseline"]["edf"] = {"value": len(ids) / (time.perf_counter() - t0), "unit": "queries/s",
                                               "sample": f"the same {len(ids)} nodes, ssdf::edf<double,double,int>"}
        except Exception as ex:
            line["cpu_baseline"] = {"error": repr(ex)}
    dm.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def batched_leg(S, args):
    """Config 4: uneven meshes (seeded icospheres / tori, 1e3..2e5 triangles, grid sides 32..160),
    signed, FP32 + FP64 fix-up: one persistent launch (CUDA graph replay) against one launch per mesh."""
    import torch

    from ssdf_b200 import workloads as W

    sets = W.multi_mesh_set(count=args.batch_meshes)
    # autotune on representative meshes across the size range; each mesh takes the leaf size of the
    # representative nearest in triangle count, the batch the query-weighted majority traversal/arity
    order = sorted(range(len(sets)), key=lambda i: sets[i][0].nt)
    reps = [order[int(k)] for k in np.linspace(0, len(order) - 1, 8)]
    tuned = {i: S.autotune_grid(sets[i][0], sets[i][1]) for i in reps}
    votes = {}
    for i, t in tuned.items():
        key = (t["traversal"], t["arity"])
        votes[key] = votes.get(key, 0) + sets[i][1].size
    trav, arity = max(votes, key=votes.get)
    leaf_of = lambda m: tuned[min(reps, key=lambda i: abs(np.log(sets[i][0].nt) - np.log(m.nt)))]["leaf_size"]  # noqa
    dms = [S.DeviceMesh(m, leaf_size=leaf_of(m)) for m, _ in sets]
    outs = [torch.empty(g.size, dtype=torch.float64, device="cuda") for _, g in sets]
    nq = sum(g.size for _, g in sets)
    ntri = sum(m.nt for m, _ in sets)
    stream = torch.cuda.current_stream()
    res = {"meshes": len(sets), "queries": nq, "triangles": ntri,
           "tuning": {"traversal": "warp" if trav == 1 else "thread", "arity": arity,
                      "leaf_sizes": sorted({t["leaf_size"] for t in tuned.values()})}}
    for prec, name in ((S.PREC_F32_FIXUP, "fixup"), (S.PREC_F64, "fp64")):
        b = S.Batch(len(sets), prec, traversal=trav, arity=arity)
        for dm, (m, g), out in zip(dms, sets, outs):
            b.add_grid(dm, g, out)
        ms = []
        for rep in range(4):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.run(use_graph=True, stream=stream)
            e1.record(stream)
            torch.cuda.synchronize()
            if rep:
                ms.append(e0.elapsed_time(e1))
        res[name] = {"queries_per_s": nq / (statistics.median(ms) * 1e-3), "ms": statistics.median(ms)}
        b.close()
    ms = []
    for rep in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for dm, (m, g), out in zip(dms, sets, outs):
            dm.query_grid(g, out, None, precision=S.PREC_F32_FIXUP, output=S.OUT_SDF, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        if rep:
            ms.append(e0.elapsed_time(e1))
    res["one_launch_per_mesh"] = {"queries_per_s": nq / (statistics.median(ms) * 1e-3), "ms": statistics.median(ms)}
    res["speedup_fixup_vs_fp64"] = res["fixup"]["queries_per_s"] / res["fp64"]["queries_per_s"]
    for dm in dms:
        dm.close()
    res["mixed_arithmetic"] = mixed_batch(S)
    return res


def mixed_batch(S):
    """A sliver-heavy mesh (the beam lattice, 160^3 grid) in a fix-up batch with 16 tori: its job runs in
    the batch's FP64 table. Reports the mixed batch's time against the tori's fix-up batch alone plus
    the beam job alone in FP64 (the arithmetic it gets alone)."""
    import torch

    from ssdf_b200 import workloads as W

    beams = W.beam_lattice()
    jobs = [(S.DeviceMesh(beams), W.Grid((160, 160, 160), (-0.1, -0.1, -0.1), (1.1, 1.1, 1.1)))]
    for k in range(16):
        m = W.torus(0.6, 0.2, nu=64 + 32 * k, nv=24 + 8 * k, jitter=0.01, seed=50 + k, center=(2.0 * k, 0.0, 0.0))
        jobs.append((S.DeviceMesh(m), W.Grid.padded_nodes(m, 96, 0.1)))
    outs = [torch.empty(g.size, dtype=torch.float64, device="cuda") for _, g in jobs]
    stream = torch.cuda.current_stream()

    def timed(fn, reps=4):
        ms = []
        for r in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            if r:
                ms.append(e0.elapsed_time(e1))
        return statistics.median(ms)

    def batch_of(sel):
        b = S.Batch(len(sel), S.PREC_F32_FIXUP)
        for i in sel:
            b.add_grid(jobs[i][0], jobs[i][1], outs[i])
        return b

    mixed = batch_of(range(len(jobs)))
    tori = batch_of(range(1, len(jobs)))
    t_mixed = timed(lambda: mixed.run(use_graph=True, stream=stream))
    t_tori = timed(lambda: tori.run(use_graph=True, stream=stream))
    t_beam = timed(lambda: jobs[0][0].query_grid(jobs[0][1], outs[0], None, precision=S.PREC_F64, output=S.OUT_SDF,
                                                 stream=stream))
    for b in (mixed, tori):
        b.close()
    for dm, _ in jobs:
        dm.close()
    return {"beam_lattice_grid": 160 ** 3, "tori": 16, "mixed_ms": t_mixed, "tori_fixup_alone_ms": t_tori,
            "beam_fp64_alone_ms": t_beam, "beam_share_in_mix_over_alone": (t_mixed - t_tori) / t_beam}


def serving_leg(S, args):
    """Config 5 (reduced): resident meshes drawn as config 4, Poisson arrivals at swept rates; each
    request a point list (log-uniform 1e3..1e6, uniform in the padded bbox) or a grid (32^3..128^3)."""
    import threading

    from ssdf_b200 import workloads as W

    sets = W.multi_mesh_set(count=args.serve_meshes, seed=11)
    rng = np.random.default_rng(5)
    payloads = []
    for k in range(48):
        mid = int(rng.integers(len(sets)))
        m, _ = sets[mid]
        if rng.uniform() < 0.5:
            side = int(np.exp(rng.uniform(np.log(32), np.log(128))))
            payloads.append(("grid", mid, W.Grid.padded_nodes(m, side, 0.1 * m.diagonal()), side ** 3))
        else:
            n = int(np.exp(rng.uniform(np.log(1e3), np.log(1e6))))
            lo, hi = m.bbox()
            pad = 0.1 * m.diagonal()
            payloads.append(("points", mid, W.uniform_points(n, lo - pad, hi + pad, seed=k), n))
    # admission limit: at most 8M queries waiting to be packed (about two batches' worth); past it a
    # submit is refused (SSDF_ERR_BUSY) and counted, so overload shows as rejections, not as latency
    srv = S.Server(memory_budget=120 << 30, max_batch_queries=args.serve_batch_queries, max_batch_jobs=64,
                   max_queued_queries=args.serve_queue, split_queries=args.serve_split, slots=args.serve_slots)
    ids = [srv.add_mesh(m) for m, _ in sets]
    # admit every mesh once (building is not part of the latency being measured)
    for mid in range(len(sets)):
        srv.wait(srv.submit_points(ids[mid], np.zeros((3, 1))))
    out = {"meshes": len(sets), "payloads": len(payloads), "seconds_per_rate": args.serve_seconds, "rates": [],
           "server": {"max_batch_queries": args.serve_batch_queries, "split_queries": args.serve_split or "default",
                      "max_queued_queries": args.serve_queue, "slots": args.serve_slots or "default"}}
    # the latency floor: every payload submitted alone (the median of three), and the p50 / p99 of
    # those over the uniform draw the arrivals make -- what a request costs with no queue in front
    alone = []
    for kind, mid, q, n in payloads:
        t = []
        for _ in range(3):
            t0 = time.perf_counter()
            srv.wait(srv.submit_grid(ids[mid], q) if kind == "grid" else srv.submit_points(ids[mid], q))
            t.append((time.perf_counter() - t0) * 1e3)
        alone.append(sorted(t)[1])
    heavy = int(np.argmax(alone))
    out["alone"] = {"p50_ms": float(np.percentile(alone, 50)), "p99_ms": float(np.percentile(alone, 99)),
                    "max_ms": alone[heavy], "heaviest": {"kind": payloads[heavy][0], "queries": payloads[heavy][3],
                                                         "triangles": int(sets[payloads[heavy][1]][0].nt)}}
    for lam in (50.0, 200.0, 800.0, 3200.0):
        srv.reset_stats()
        tickets = []
        t_end = time.perf_counter() + args.serve_seconds
        arrivals = np.random.default_rng(int(lam))
        offered = 0
        while time.perf_counter() < t_end:
            kind, mid, q, n = payloads[int(arrivals.integers(len(payloads)))]
            offered += 1
            try:
                tickets.append(srv.submit_grid(ids[mid], q) if kind == "grid" else srv.submit_points(ids[mid], q))
            except S.SsdfError as ex:
                if ex.status != S.SSDF_ERR_BUSY:
                    raise
            time.sleep(float(arrivals.exponential(1.0 / lam)))
        for t in tickets:
            srv.wait(t, timeout=300)
        st = srv.stats()
        out["rates"].append({"lambda_per_s": lam, "offered": offered, "requests": st["completed"],
                             "rejected": st["rejected"], "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
                             "queries_per_s": st["queries"] / max(st["seconds"], 1e-9), "batches": st["batches"]})
    srv.close()
    return out


def e2e(S, mesh, grid, args, pageable=False):
    """Through the drop-in C ABI from host arrays: upload, build, query, download (into page-locked
    memory, or ordinary pageable numpy memory as the reference's drivers allocate)."""
    import torch

    nq = grid.size
    host_out = np.empty(nq) if pageable else torch.empty(nq, dtype=torch.float64, pin_memory=True).numpy()
    hm = S.capi._HostMesh(mesh, np.float64)
    nx, ny, nz = grid.n
    import ctypes as C

    def call():
        st = S.lib.ssdf_b200_sample_sdf_bvh_dd(*hm.args(), nx, ny, nz, *[C.c_double(v) for v in grid.lo],
                                               *[C.c_double(v) for v in grid.hi], C.c_void_p(host_out.ctypes.data))
        if st != 0:
            raise RuntimeError(S.last_error())

    for _ in range(max(1, args.warmup)):
        call()
    torch.cuda.synchronize()
    k = max(2, args.steps)
    t0 = time.perf_counter()
    for _ in range(k):
        call()
    dt = (time.perf_counter() - t0) / k
    h2d = sum(a.nbytes for a in (hm.sx, hm.sy, hm.sz, hm.s0, hm.s1, hm.s2))
    return {"value": nq / dt, "unit": "queries/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": nq * 8,
            "ms_per_call": dt * 1e3, "api": "ssdf_b200_sample_sdf_bvh_dd (host arrays, blocking; wall clock)",
            "output_memory": "pageable" if pageable else "page-locked"}


def dense_leg(S, mesh, grid, args):
    """Config 1's plain methods on the GPU: ssdf::edf (brute force) and ssdf::edf_celllist over device
    arrays at the grid's nodes (ssdf_edf_device, FP64), timed with CUDA events, each with its counted
    work against the measured FP64 FMA peak; the reference's own edf and edf_celllist<double> on the
    host cores are timed on a sample in the cpu_baseline leg."""
    import torch

    nx, ny, nz = grid.n
    h = [(grid.hi[d] - grid.lo[d]) / (grid.n[d] - 1) for d in range(3)]
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    pts = [grid.lo[d] + (ii, jj, kk)[d].transpose(2, 1, 0).ravel() * h[d] for d in range(3)]
    x, y, z = (torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda") for a in pts)
    sx, sy, sz = (torch.tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda") for a in mesh.coords())
    s0, s1, s2 = (torch.tensor(np.ascontiguousarray(a, dtype=np.int32), device="cuda") for a in mesh.indices())
    n = x.numel()
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    big = float(np.finfo(np.float64).max)
    stream = torch.cuda.current_stream()
    peak64 = S.fma_peak_tflops(True)
    res = {"points": n, "triangles": mesh.nt, "dtype": "f64"}
    for method, name in ((0, "edf"), (1, "edf_celllist")):
        ms = []
        for rep in range(3 + args.steps):
            out.fill_(big)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            S.edf_device(method, x, y, z, s0, s1, s2, sx, sy, sz, out, stream=stream)
            e1.record(stream)
            torch.cuda.synchronize()
            if rep >= 3:
                ms.append(e0.elapsed_time(e1))
        os.environ["SSDF_B200_COUNT"] = "1"
        out.fill_(big)
        S.edf_device(method, x, y, z, s0, s1, s2, sx, sy, sz, out, stream=stream)
        counts = S.last_query_counts()
        del os.environ["SSDF_B200_COUNT"]
        t = statistics.median(ms) * 1e-3
        flops = 79.0 * counts["triangle_tests"] + 8.0 * counts["box_tests"]
        res[name] = {"queries_per_s": n / t, "ms": t * 1e3, "triangle_tests": counts["triangle_tests"],
                     "box_tests": counts["box_tests"],
                     "roofline": {"bound": "fp64", "achieved": flops / t / 1e12, "peak": peak64, "unit": "TFLOP/s",
                                  "frac": flops / t / 1e12 / peak64,
                                  "peak_source": "measured FP64 FMA microbenchmark on this GPU (ssdf_b200_fma_peak)",
                                  "note": "the whole call (record build, launch, flag read-back) in the time"}}
    return res


def _hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)["hbm_gbs"]
    except Exception:
        return 6650.0


def _attach_traffic(line):
    """DRAM bytes per launch of the query kernel, and the share of issue slots it keeps busy, from the
    committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            t = json.load(f)
        line["roofline"]["traffic"] = t["dram_bytes_per_launch"]
        line["roofline"]["traffic_source"] = t.get("source")
        if "issue" in t:  # the bound that binds: instruction issue (flops counted per test undercount it)
            line["roofline"]["issue"] = t["issue"]
    except Exception:
        pass


if __name__ == "__main__":
    main()
