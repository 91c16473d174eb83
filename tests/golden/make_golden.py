"""Regenerates the committed golden fixtures in tests/golden/ from the reference itself.

Run in a checkout where zulianp/ssdf's sources are available (default /root/reference; override
with SSDF_REFERENCE_SRC). Two kinds of fixture:

* reference_tests.json -- the inputs of ssdf's own CPU tests for this path, regenerated exactly
  (gen_golden.cpp, compiled against the reference's serial/ssdf.hpp), with its outputs;
* <workload>_sample.npz -- the reference's own edf / edf_celllist (oracle/_ref, compiled from its
  sources by oracle/Makefile) on a seeded sample of each workload's query points.

    python tests/golden/make_golden.py
"""

from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from ssdf_b200 import workloads as W  # noqa: E402

REF = os.environ.get("SSDF_REFERENCE_SRC", "/root/reference")


def reference_tests() -> None:
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "gen_golden")
        subprocess.run(["g++", "-std=c++17", "-O3", "-fopenmp", "-c", "-o", exe + ".o",
                        f"-I{ROOT}/oracle/ref_config", f"-I{REF}/serial", os.path.join(HERE, "gen_golden.cpp")],
                       check=True)
        subprocess.run(["g++", "-o", exe, exe + ".o", "-l:libgomp.so.1"], check=True)
        subprocess.run([exe, os.path.join(HERE, "reference_tests.json")], check=True, stdout=subprocess.DEVNULL)


def sample(name, mesh, points, nsample, seed, dtypes=(np.float64, np.float32), which=("edf", "celllist")):
    rng = np.random.default_rng(seed)
    ids = np.sort(rng.choice(points.shape[1], size=nsample, replace=False))
    q = points[:, ids]
    data = {"ids": ids.astype(np.int64), "points": q}
    for dt in dtypes:
        tag = "d" if dt == np.float64 else "f"
        qd = q.astype(dt)
        for w in which:
            data[f"{w}_{tag}"] = oracle.ref_edf(qd, mesh, dtype=dt, which=w)
    np.savez_compressed(os.path.join(HERE, f"{name}_sample.npz"), **data)


def main() -> None:
    oracle.build(REF)
    reference_tests()
    ico = W.icosphere()
    g1 = W.Grid.cell_centred(ico, 64, 0.2)
    sample("icosphere", ico, oracle.grid_points(g1), 4096, 11)
    knot = W.torus_knot_tube()
    g2 = W.Grid.padded_nodes(knot, 256, 0.25)
    sample("torus_knot", knot, oracle.grid_points(g2), 512, 12, which=("celllist",))
    beams = W.beam_lattice()
    pts = W.uniform_points(200000, -0.1, 1.1, seed=13)
    sample("beam_lattice", beams, pts, 512, 14, dtypes=(np.float32,), which=("celllist",))


if __name__ == "__main__":
    main()
