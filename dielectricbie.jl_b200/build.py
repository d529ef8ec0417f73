"""Builds libbie_b200.so in-tree for sm_100a (nvcc cross-compiles without a GPU).

    python dielectricbie.jl_b200/build.py [--force]

The shared library lands next to this file so that it travels with the source
tree; CUDA runtime is linked statically (libcuda.so and the toolkit's libcublas.so, found
through the rpath, are needed at run time).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbie_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["bie_b200.cu", "solver.cu", "blocktc.cu", "dt64mma.cu", "noalloc.cu", "server.cu", "near_gpu.cu", "peaks.cu", "combine_bulk.cu", "probe.cu"]
CPP_SOURCES = ["host_setup.cpp", "probe_setup.cpp"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _hostcxx() -> str:
    # a g++ whose OpenMP runtime is installed (the system one)
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("g++ not found")


def _deps():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    files.append(os.path.join(INCLUDE, "bie_b200.h"))
    files.append(os.path.abspath(__file__))
    return files


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _deps())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    nvcc, cxx = _nvcc(), _hostcxx()
    common = ["-O3", "-std=c++17", "-I", INCLUDE, "-I", CSRC]
    objs = []
    for src in CU_SOURCES:
        if not os.path.exists(os.path.join(CSRC, src)):
            continue
        obj = os.path.join(BUILD, src + ".o")
        cmd = [nvcc, "-ccbin", cxx, *ARCH, "-lineinfo", *common, "-Xcompiler", "-fPIC,-fopenmp",
               "--expt-relaxed-constexpr", "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
        objs.append(obj)
    for src in CPP_SOURCES:
        obj = os.path.join(BUILD, src + ".o")
        subprocess.run([cxx, *common, "-fPIC", "-fopenmp", "-Wall", "-c", os.path.join(CSRC, src), "-o", obj],
                       check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    # cuBLAS (the block GMRES basis products) from the CUDA toolkit, found through the rpath
    cudalib = os.path.join(os.path.dirname(os.path.dirname(nvcc)), "lib64")
    subprocess.run([nvcc, "-ccbin", cxx, *ARCH, "-shared", "-o", tmp, *objs, "-Xcompiler", "-fopenmp", "-lgomp",
                    "-L", cudalib, "-lcublas", "-Xlinker", "-rpath," + cudalib, "-Xlinker", "--no-undefined"],
                   check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
