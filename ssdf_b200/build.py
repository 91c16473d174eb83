"""Builds libssdf_b200.so in-tree with nvcc for sm_100a (B200).

Every .cu under csrc/ is compiled to an object in parallel and linked into one shared library
with a static CUDA runtime. -fmad=false keeps every multiply and add separately rounded, as the
reference's C++17 build does (so the exact routines are bitwise its arithmetic); code that wants a
fused multiply-add calls fmaf() explicitly.

    python -m ssdf_b200.build [-v]
"""

from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libssdf_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xcompiler", "-Wall"]


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(OUT_DIR, os.path.basename(src) + ".o")
    deps = [src] + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        [os.path.join(HERE, "..", "include", "ssdf_b200.h")]
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return obj
    cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{res.stderr}")
    if verbose and res.stderr:
        sys.stderr.write(res.stderr)
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-Xlinker", "--exclude-libs,ALL"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stderr}")
    _build_cli(verbose)
    return LIB


CLI_SRC = os.path.join(HERE, "cli", "ssdf_sdf.cpp")
CLI = os.path.join(OUT_DIR, "ssdf_sdf")


def _build_cli(verbose: bool) -> str:
    """The command-line driver (drivers/sdf.exe.cpp's arguments and files) over the library."""
    deps = [CLI_SRC, LIB, os.path.join(HERE, "..", "include", "ssdf_b200.h")]
    if os.path.exists(CLI) and all(os.path.getmtime(CLI) >= os.path.getmtime(d) for d in deps):
        return CLI
    cmd = [NVCC, "-O2", "-std=c++17", "-I", os.path.join(HERE, "..", "include"), CLI_SRC, "-o", CLI,
           "-L", OUT_DIR, "-lssdf_b200", "-Xlinker", "-rpath,$ORIGIN"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {CLI_SRC}:\n{res.stderr}")
    if verbose and res.stderr:
        sys.stderr.write(res.stderr)
    return CLI


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
