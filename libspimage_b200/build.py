"""Builds libspimage_b200.so in-tree (sm_100a CUDA kernels + host C library).

    python -m libspimage_b200.build [--force]

CUDA sources are compiled by nvcc for sm_100a only; host C sources by gcc.
Floating-point contraction is disabled everywhere on the phasing path
(-fmad=false / -ffp-contract=off): the kernels spell out every rounding so the
iterates reproduce the reference CPU engine's arithmetic.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libspimage_b200.so")

CU_SOURCES = ["spb_kernels.cu", "spb_fast.cu", "spb_split.cu", "spb_capi.cu"]
C_SOURCES = ["host/image.c", "host/phasing.c", "host/support_update.c", "host/fft.c", "host/prtf.c"]
CXX_SOURCES = ["host/serve.cpp"]
HEADERS = ["spb_fft.cuh", "spb_internal.h", "spb_pointwise.cuh", "spb_passes.cuh", "host/host_internal.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC", "-Xptxas", "-O3"]
CC_FLAGS = ["-O2", "-fPIC", "-std=gnu11", "-ffp-contract=off", "-fno-fast-math", "-Wall", "-Wno-unused-function"]
CXX_FLAGS = ["-O2", "-fPIC", "-std=c++17", "-ffp-contract=off", "-Wall", "-Wno-unused-function", "-pthread"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libspimage_b200")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles the stale objects (in parallel) and links the library."""
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(INCLUDE, "spimage", f) for f in os.listdir(os.path.join(INCLUDE, "spimage"))
    ]
    cuda_inc = os.path.join(os.path.dirname(os.path.dirname(nvcc)), "include")
    objs, jobs = [], []
    for srcs, compiler in ((CU_SOURCES, "nvcc"), (C_SOURCES, "gcc"), (CXX_SOURCES, "g++")):
        for src in srcs:
            s = os.path.join(CSRC, src)
            o = os.path.join(BUILD, os.path.basename(src) + ".o")
            objs.append(o)
            if not (force or _newer(o, [s] + headers)):
                continue
            if compiler == "nvcc":
                cmd = [nvcc] + ARCH + NVCC_FLAGS + ["-I", INCLUDE, "-I", CSRC, "-c", s, "-o", o]
            elif compiler == "gcc":
                cmd = ["gcc"] + CC_FLAGS + ["-I", INCLUDE, "-c", s, "-o", o]
            else:
                cmd = ["g++"] + CXX_FLAGS + ["-I", INCLUDE, "-I", cuda_inc, "-c", s, "-o", o]
            jobs.append(cmd)
    if verbose:
        for cmd in jobs:
            print(" ".join(cmd))
    if jobs:
        with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1)) as ex:
            list(ex.map(_run, jobs))
    if force or _newer(LIB, objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lm", "-lpthread"]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
