"""Build recipe of libefie_b200.so (sm_100a) -- in-tree, no JIT cache.

Run as ``python matlab-cuda-efief-vs-cpu_b200/build.py`` or through
``__graft_entry__.build()``.  nvcc cross-compiles for sm_100a without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libefie_b200.so")
SOURCES = ["capi.cu", "assemble.cu", "solve.cu", "trsv.cu", "gemm_tc.cu", "noalloc.cu", "surrogate.cu", "gmres.cu", "precompute.cu", "mesh.cu", "geom.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    deps = [os.path.join(CSRC, s) for s in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "efie_b200.h"))
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(objdir, s + ".o")
        cmd = [NVCC, "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
               "-I", os.path.join(HERE, "..", "include"), "-c", src, "-o", obj] + ARCH
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.check_call(cmd)
        objs.append(obj)
    tmp = LIB + ".tmp"
    subprocess.check_call([NVCC, "-shared", "-o", tmp] + objs + ARCH +
                          ["-lcusolver", "-lcublas", "-lcudart"])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
