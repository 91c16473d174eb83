"""GPU: the autotuner picks a (leaf size, traversal, arity) and caches it per size class."""

import json

import numpy as np
import pytest

import ssdf_b200 as S
from ssdf_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_autotune_and_cache(tmp_path):
    mesh = W.torus_knot_tube(nu=256, nv=32)
    grid = W.Grid.padded_nodes(mesh, 96, 0.25)
    cache = str(tmp_path / "tuning.json")
    t = S.autotune_grid(mesh, grid, cache_path=cache)
    assert t["leaf_size"] in (2, 4, 8) and t["traversal"] in (1, 2) and t["arity"] in (2, 4) and t["ms"] > 0
    data = json.load(open(cache))
    assert len(data) == 1 and list(data.values())[0][:3] == [t["leaf_size"], t["traversal"], t["arity"]]
    # same size class: answered from the cache, identical
    again = S.autotune_grid(mesh, W.Grid.padded_nodes(mesh, 97, 0.3), cache_path=cache)
    assert [again[k] for k in ("leaf_size", "traversal", "arity")] == [t[k] for k in ("leaf_size", "traversal", "arity")]
    assert abs(again["ms"] - t["ms"]) < 1e-5
    # the tuned configuration gives the default configuration's values
    want = S.sample_sdf_bvh(mesh, grid)
    dm = S.DeviceMesh(mesh, leaf_size=t["leaf_size"])
    import torch

    out = torch.empty(grid.size, dtype=torch.float64, device="cuda")
    b = S.Batch(1, S.PREC_F32_FIXUP, traversal=t["traversal"], arity=t["arity"])
    b.add_grid(dm, grid, out)
    b.run()
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), want)
    b.close()
    dm.close()
