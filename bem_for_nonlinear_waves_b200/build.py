"""Builds the in-tree CUDA library lib/libbem_b200.so (sm_100a) from csrc/.

CUDA sources go through nvcc for sm_100a; the host-side plan builder goes through
g++ with the same flags as the reference build (-O2 -march=x86-64-v3, no fast-math) so
that the octree placement arithmetic rounds the same way.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(OUT_DIR, "libbem_b200.so")
BUILD = os.path.join(HERE, "_build")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
CXXFLAGS = ["-O2", "-march=x86-64-v3", "-std=c++17", "-fPIC", "-Wall", "-fopenmp", "-pthread"]

CU_SOURCES = ["kernels.cu", "m2l_tc.cu", "gmres.cu", "capi.cu", "mel.cu", "tree.cu"]
CXX_SOURCES = ["plan.cpp", "batch.cpp", "poly.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + os.path.basename(cmd[-1]))
    return r


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "bem_b200.h"))
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers) or ptxas_info:
            cmd = [NVCC] + ARCH + NVFLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", "-o", o, s]
            r = _run(cmd)
            if verbose or ptxas_info:
                sys.stderr.write(r.stderr)
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers):
            _run(["g++"] + CXXFLAGS + ["-c", "-o", o, s])
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart=static", "-o", LIB] + objs + ["-lstdc++", "-lgomp", "-lpthread"])
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))
