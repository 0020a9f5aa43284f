"""Build the sm_100a library in-tree: hipft_b200/libhipft_gpu.so and the
standalone executable hipft_b200/bin/hipft.

nvcc compiles the CUDA translation unit for sm_100a only, with --fmad=false so
that a*b+c is rounded twice, as in the reference's operation order; g++
compiles the host-only sources.  Run `python -m hipft_b200.build`.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libhipft_gpu.so")
EXE = os.path.join(PKG, "bin", "hipft")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["hipft_gpu.cu"]
CXX_SOURCES = ["namelist.cpp", "h5lite.cpp", "h5write.cpp", "driver.cpp"]
HEADERS = sorted(f for f in os.listdir(CSRC) if f.endswith((".cuh", ".h")))


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build hipft_b200")


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    nvcc = _nvcc()
    objdir = os.path.join(PKG, "_build")
    os.makedirs(objdir, exist_ok=True)
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    include = os.path.join(os.path.dirname(PKG), "include", "hipft_gpu.h")
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [include]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(objdir, src + ".o")
        if force or _newer(o, [s] + hdrs):
            cmd = [nvcc, "-std=c++17", *ARCH, "-O3", "--fmad=false", "-lineinfo", "-Xcompiler", "-fPIC",
                   "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
        objs.append(o)
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(objdir, src + ".o")
        if force or _newer(o, [s] + hdrs):
            cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-Wall", "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
        objs.append(o)
    if force or _newer(LIB, objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart_static", "-lrt", "-lpthread", "-ldl"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    main = os.path.join(CSRC, "main.cpp")
    if force or _newer(EXE, [main, LIB]):
        cmd = ["g++", "-std=c++17", "-O2", main, "-o", EXE, "-L" + PKG, "-lhipft_gpu",
               "-Wl,-rpath,$ORIGIN/.."]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
