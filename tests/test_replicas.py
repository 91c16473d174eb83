"""The N > 1 path of bench.py on CPU: two gloo ranks, the step time reduced as the max over ranks
and the whole-job rate of independent replicas (the path does not shard: replicas only)."""

import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, results):
    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}")
    try:
        mine = 10.0 + 5.0 * rank  # rank 1 is the slow one
        t = bench.max_over_ranks(mine, dist, "cpu")
        results[rank] = (t, bench.job_rate(1000, 4, t, world))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_rate():
    import torch.multiprocessing as mp

    world = 2
    port = _free_port()
    manager = mp.get_context("spawn").Manager()
    results = manager.dict()
    mp.start_processes(_rank, args=(world, port, results), nprocs=world, start_method="spawn", join=True)
    assert results[0][0] == results[1][0] == 15.0
    # 2 replicas x 1000 queries x 4 steps in 15 ms
    assert results[0][1] == pytest.approx(2 * 1000 * 4 / 0.015)
