"""Compile the CUDA builder into ``marigold_b200/libmgbvh.so`` (sm_100a).

Build rule: nvcc, one translation unit, -fmad=false (the reference's f32
arithmetic has no fused multiply-adds), static CUDA runtime so the library
does not depend on which libcudart a host process already loaded.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmgbvh.so")
SOURCES = ["mgbvh_build.cu", "mgbvh_trace.cu", "mgbvh_mlp.cu"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-shared", "-cudart", "static",
]


def nvcc_path() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA builder cannot be compiled")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    # every header under csrc/: a header left out of the list would not trigger a rebuild
    headers = sorted(f for f in os.listdir(CSRC) if f.endswith((".cuh", ".h")))
    deps = [os.path.join(CSRC, f) for f in SOURCES + headers]
    deps.append(os.path.join(HERE, "..", "include", "mgbvh.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    cmd = [nvcc_path(), *NVCC_FLAGS, "-o", LIB + ".tmp",
           *[os.path.join(CSRC, s) for s in SOURCES]]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
