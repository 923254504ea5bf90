"""Build recipe for the native library ``libhgx.so`` (sm_100a), in-tree.

    python -m hypergraphrewritingengine_b200.build      # or build() from Python

Compiles the CUDA step kernels, the host engine and the C-ABI with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` into ``hypergraphrewritingengine_b200/libhgx.so``.
No torch types or headers are involved: the library is a plain C-ABI shared object.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libhgx.so")
SOURCES = ["engine.cu", "capi.cpp"]
DEPS = ["engine.cu", "capi.cpp", "engine.hpp", "step_kernels.cu", "step_kernels.cuh", "common.cuh",
        "lane_wl.cuh",
        os.path.join("..", "..", "include", "hgx.h")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(os.path.join(CSRC, d)) > t for d in DEPS)


def build(force: bool = False, verbose: bool = False, extra_flags=()) -> str:
    if not force and not _stale():
        return LIB
    tmp = LIB + ".tmp"
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3",
           "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
           "--expt-relaxed-constexpr", "-I", os.path.join(HERE, "..", "include"),
           *extra_flags, *[os.path.join(CSRC, s) for s in SOURCES], "-o", tmp]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True,
                extra_flags=["-Xptxas", "-v"] if "--ptxas" in sys.argv else []))
