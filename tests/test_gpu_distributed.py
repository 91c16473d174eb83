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
