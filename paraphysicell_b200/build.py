"""Builds libppc.so (the CUDA library behind include/ppc.h) in-tree.

    python -m paraphysicell_b200.build

Compiles every .cu under csrc/ for sm_100a with nvcc into
paraphysicell_b200/libppc.so. -fmad=false keeps FP64 arithmetic free of FMA
contraction, so the FP64 path rounds exactly like the reference's baseline
x86-64 build.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libppc.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "--expt-relaxed-constexpr",
         "-Xcompiler", "-fPIC,-O2"]
OBJDIR = os.path.join(HERE, "_build")


def nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def headers():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + \
        sorted(glob.glob(os.path.join(os.path.dirname(HERE), "include", "*.h")))


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in sources() + headers())


def build(verbose=False, extra=()):
    """Compiles every source to an object in parallel, then links them."""
    os.makedirs(OBJDIR, exist_ok=True)
    jobs, objs = [], []
    for src in sources():
        obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
        cmd = [nvcc(), *ARCH, *FLAGS, *extra, "-c", "-o", obj, src]
        if verbose:
            print(" ".join(cmd))
        jobs.append((cmd, subprocess.Popen(cmd)))
        objs.append(obj)
    failed = [cmd for cmd, p in jobs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    link = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True)
    return LIB


def ensure_built():
    if stale():
        build()
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
