"""Compile the CUDA library in-tree: penguin_b200/libpenguin_b200.so (sm_100a).

    python -m penguin_b200.build [--force]

nvcc cross-compiles without a GPU.  The CUDA runtime is linked statically so
the library does not depend on which libcudart the host process loaded first.
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
LIB = os.path.join(PKG, "libpenguin_b200.so")
OBJ = os.path.join(PKG, "_build")

SOURCES = ["pg_kernels.cu", "pg_engine.cu", "pg_noalloc.cu", "pg_f32.cu", "pg_ensemble.cu", "pg_dust.cu", "pg_adjoint.cu", "pg_3d.cu"]
HEADERS = ["pg_common.cuh", "pg_hydro.cuh", "pg_internal.h", "pg_planet.cuh", "pg_f32.cuh", "pg_dust.cuh", "pg_dual.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INCLUDE]
# The FP32-mixed kernels take the approximate FP32 division and square root
# (a few ulp); FP64 arithmetic, the FP64 kernels and denormals are unaffected.
EXTRA = {"pg_f32.cu": ["-prec-div=false", "-prec-sqrt=false"]}


def _nvcc() -> str:
    for c in (os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc"), shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise FileNotFoundError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    nvcc = _nvcc()
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "penguin_b200.h")]
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            cmd = [nvcc] + ARCH + FLAGS + EXTRA.get(src, []) + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-cudart", "static"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
