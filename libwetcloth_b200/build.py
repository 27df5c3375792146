"""Build recipe for libwcgpu.so (sm_100a), in-tree.

    python -m libwetcloth_b200.build
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libwcgpu.so")
SOURCES = ["wcg_step.cu", "wcg_capi.cu", "wcg_noalloc.cu", "wcg_batch.cu"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3",
              "-std=c++17", "-Xcompiler", "-fPIC", "-shared"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def newest_source_mtime() -> float:
    t = 0.0
    for f in os.listdir(CSRC):
        t = max(t, os.path.getmtime(os.path.join(CSRC, f)))
    hdr = os.path.join(os.path.dirname(HERE), "include", "wetcloth_gpu.h")
    if os.path.exists(hdr):
        t = max(t, os.path.getmtime(hdr))
    return t


def build(force: bool = False, verbose: bool = True) -> str:
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= newest_source_mtime():
        return OUT
    cmd = [nvcc(), *NVCC_FLAGS, "-o", OUT] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv)
