"""Build libflexrt_b200.so in-tree (sm_100a).

nvcc compiles the CUDA sources for compute_100a / sm_100a; the geometry translation unit uses
-fmad=false (its float arithmetic must round exactly like the reference's g++ build; the adjoint
recomputes the same ray walk and is compiled the same way), the host
set-up arithmetic is compiled by g++ with -ffp-contract=off for the same reason.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libflexrt_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
               "--expt-relaxed-constexpr"]

SOURCES = [
    # (file, extra flags)
    ("frt_geom.cu", ["-fmad=false"]),
    ("frt_phys.cu", []),
    ("frt_adjoint.cu", ["-fmad=false"]),
    ("frt_subgrid.cu", ["-fmad=false"]),
    ("frt_ctx.cu", []),
]
HEADERS = ["frt_internal.cuh", "frt_physics.cuh", "frt_params.h", "hp_nest.h", "frt_hostmath.h", "frt_dda.cuh", "frt_tune.h",
           os.path.join("..", "..", "include", "flexrt.h")]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(p) > t for p in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS]
    objs = []
    for src, extra in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src.replace(".cu", ".o"))
        if force or _newer(o, [s] + hdrs + [__file__]):
            _run(["nvcc"] + ARCH + NVCC_COMMON + extra + ["-c", s, "-o", o], verbose)
        objs.append(o)
    for src in ("frt_hostmath.cc", "frt_tune.cc"):
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src.replace(".cc", ".o"))
        if force or _newer(o, [s] + hdrs + [__file__]):
            _run(["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-c", s, "-o", o], verbose)
        objs.append(o)
    if force or _newer(LIB, objs):
        _run(["nvcc"] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"], verbose)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
