"""Build the engine's shared library in-tree: libgrpp_b200/libgrpp_b200.so.

nvcc compiles for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``);
no GPU is needed to build. Usage: ``python -m libgrpp_b200.build [-v]``.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libgrpp_b200.so")
BUILD = os.path.join(HERE, "_build")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden"]

SOURCES = ["engine.cu", "nofma.cu", "tables.cpp", "capi.cpp", "fortran_abi.cpp", "noalloc.cu"]
# libgrpp is built without floating-point contraction; the angular sums round as its do
EXTRA = {"nofma.cu": ["-fmad=false"]}
HEADERS = ["grpp_common.cuh", "specfunc.cuh", "mmd.cuh", "radial.cuh", "angular.cuh", "level_model.cuh", "gradient.cuh", "tables.h",
           "engine.h", "onee.cuh", "nucmodel.h", "nofma_launch.h", "exp_rn.h"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", h)
                                                       for h in ("libgrpp.h", "libgrpp_b200.h", "libgrpp_f90.h")]
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            cmd = [NVCC] + ARCH + COMMON + EXTRA.get(src, []) + ["-c", s, "-o", o]
            if src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"] if verbose else []
            else:
                cmd = [NVCC] + COMMON + ["-x", "c++", "-c", s, "-o", o]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if verbose or r.returncode:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode:
                raise RuntimeError(f"nvcc failed on {src}")
    if force or _newer(OUT, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart_static", "-lrt", "-lpthread", "-ldl",
                                                              "-Xlinker", "-Bsymbolic"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
