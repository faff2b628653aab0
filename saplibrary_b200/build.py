"""Build recipe of the sap_b200 CUDA library (sm_100a) and its CPU oracle.

`python saplibrary_b200/build.py` compiles every CUDA/C++ source of
saplibrary_b200/csrc into saplibrary_b200/libsap_b200.so with nvcc, in tree,
so the shared object travels with the repository snapshot.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsap_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp", "--expt-relaxed-constexpr",
         "-Xptxas", "-warn-spills"]
SOURCES = ["sap_impl.cu", "dots_noalloc.cu", "mlp.cu", "gen.cpp", "reorder.cpp", "mmio.cpp"]


def _newest_source_mtime() -> float:
    t = 0.0
    for f in os.listdir(CSRC):
        t = max(t, os.path.getmtime(os.path.join(CSRC, f)))
    t = max(t, os.path.getmtime(os.path.join(HERE, "..", "include", "sap_b200.h")))
    return t


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest_source_mtime():
        return LIB
    objs = []
    for src in SOURCES:
        obj = os.path.join(CSRC, os.path.splitext(src)[0] + ".o")
        cmd = [NVCC, *ARCH, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cpp"):
            cmd = [NVCC, *FLAGS, "-Wno-deprecated-gpu-targets", "-x", "c++", "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC,-fopenmp", "-o", LIB, *objs, "-lgomp", "-lcublas",
           "-Xlinker", "-rpath,/usr/local/cuda/lib64"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
