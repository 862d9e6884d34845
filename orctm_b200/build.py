"""Builds liborctm_gpu.so (sm_100a) in-tree with nvcc.

The library is plain CUDA C++ behind an extern "C" ABI (include/orctm_gpu.h);
it does not link against torch.  Device code is compiled with --fmad=false
and IEEE division/square root so that the FP64 path reproduces the
operation order of the reference's Fortran arithmetic.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
SO = os.path.join(HERE, "liborctm_gpu.so")
SOURCES = ["advect.cu", "diffuse.cu", "nh.cu", "poisson.cu", "handle.cu", "grid.cpp", "serve.cpp", "extra.cpp",
           "noalloc.cu", "obc.cu", "barotropic.cu", "baroclinic.cu"]
HEADERS = ["common.cuh", "ops.h", "tma.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.exists(c) or c == "nvcc"):
            return c
    raise RuntimeError("nvcc not found")


def needs_build() -> bool:
    if not os.path.exists(SO):
        return True
    t = os.path.getmtime(SO)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "orctm_gpu.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return SO
    cmd = [nvcc(), *ARCH, "-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-prec-div=true",
           "-prec-sqrt=true", "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared",
           "-I", os.path.join(ROOT, "include"), "-o", SO + ".tmp",
           *[os.path.join(CSRC, f) for f in SOURCES], "-lcudart"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, cwd=CSRC, env={**os.environ, "CC": "gcc", "CXX": "g++"})
    os.replace(SO + ".tmp", SO)
    return SO


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(SO)
