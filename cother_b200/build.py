"""Build recipes for the native libraries of the package.

* ``libcother_b200.so`` -- the search path: hand-written sm_100a CUDA
  kernels plus the C++ host driver behind the C ABI of
  ``include/cother_b200.h``. Compiled with ``nvcc -gencode
  arch=compute_100a,code=sm_100a``; ``--fmad=false`` keeps every
  multiply-add where the source writes one (``__fmaf_rn``), so results are
  reproducible operation by operation.
* ``libcbsynth.so`` -- the seeded synthetic profile generator (host C++).

Both land next to this file (in-tree) so that they travel with the
repository snapshot.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")

LIB_MAIN = os.path.join(HERE, "libcother_b200.so")
LIB_SYNTH = os.path.join(HERE, "libcbsynth.so")

CUDA_SOURCES = [
    "api.cu",
    "score_kernel.cu",
    "dp1_kernel.cu",
    "stats_kernel.cu",
    "map_kernel.cu",
    "dp1_noalloc.cu",
    "tc_kernel.cu",
    "hits_kernel.cu",
    "format.cpp",
    "server.cpp",
    "dbfile.cpp",
]
CUDA_HEADERS = [
    "map_kernel.cuh",
    "stats_kernel.cuh",
    "common.cuh",
    "cbmath.cuh",
    "layout.h",
    "score_kernel.cuh",
    "dp1_kernel.cuh",
    "tc_kernel.cuh",
    "hits_kernel.cuh",
    "bulkcopy.cuh",
]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def nvcc_flags(verbose_ptxas: bool = False):
    flags = [
        "-gencode", "arch=compute_100a,code=sm_100a",
        "-O3", "-lineinfo", "--fmad=false", "-std=c++17",
        "-Xcompiler", "-fPIC,-O2,-ffp-contract=off",
        "-I" + INCLUDE, "-I" + CSRC,
    ]
    if verbose_ptxas:
        flags += ["-Xptxas", "-v"]
    return flags


def build_main(force: bool = False, verbose_ptxas: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in CUDA_SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in CUDA_HEADERS] + \
        [os.path.join(INCLUDE, "cother_b200.h"), os.path.abspath(__file__)]
    if not force and _newer(LIB_MAIN, deps):
        return LIB_MAIN
    tmp = LIB_MAIN + ".tmp"
    cmd = [_nvcc(), "-shared", "-o", tmp] + nvcc_flags(verbose_ptxas) + srcs + ["-lpthread"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB_MAIN)
    return LIB_MAIN


def build_synth(force: bool = False) -> str:
    src = os.path.join(CSRC, "synth.cpp")
    if not force and _newer(LIB_SYNTH, [src]):
        return LIB_SYNTH
    tmp = LIB_SYNTH + ".tmp"
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", tmp, src, "-lpthread"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB_SYNTH)
    return LIB_SYNTH


def build_all(force: bool = False) -> None:
    build_synth(force)
    build_main(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
