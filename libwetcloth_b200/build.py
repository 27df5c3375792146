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
SOURCES = ["wcg_step.cu", "wcg_capi.cu", "wcg_noalloc.cu", "wcg_batch.cu", "wcg_csr.cu"]
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


OBJDIR = os.path.join(os.path.dirname(HERE), "_build", "wcgpu")


def build(force: bool = False, verbose: bool = True) -> str:
    """Compiles every translation unit to an object in parallel, then links."""
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= newest_source_mtime():
        return OUT
    os.makedirs(OBJDIR, exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]
    objs, procs = [], []
    for src in SOURCES:
        obj = os.path.join(OBJDIR, os.path.splitext(src)[0] + ".o")
        cmd = [nvcc(), *compile_flags, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((cmd, subprocess.Popen(cmd)))
        objs.append(obj)
    failed = [cmd for cmd, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", OUT, *objs]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv)
