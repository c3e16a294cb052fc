"""Relink PEnGUIn's own main.cu against libpenguin_b200 through the shim.

    python -m penguin_b200.shim.build_dropin <objdir> <parameters.h> <out>

<objdir> holds the reference's object files compiled with --device-c against
<parameters.h> (oracle/ref_build.py produces them under oracle/_ref/<case>/obj).
The new executable keeps main.o and the reference's initialisation, I/O and
planet objects, drops solver.o, timestep.o and orbit.o (plus the boundary,
killwave and viscosity objects only they use) and resolves global_dt, solve and
init_OrbAdv from penguin_shim.cu, which forwards to the C ABI.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
KEEP = ["main", "util", "geom", "EOS", "output", "init", "planet"]


def build(objdir: str, header: str, out: str, reference_include: str) -> str:
    from penguin_b200 import build as pb

    lib = pb.build()
    os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
    shim_o = os.path.join(os.path.dirname(os.path.abspath(out)), "penguin_shim.o")
    base = ["nvcc", "-arch=sm_100a", "-O3", "-std=c++11"]
    subprocess.run(base + ["--device-c", "-include", header, "-I" + os.path.dirname(header),
                           "-I" + reference_include, "-I" + os.path.join(ROOT, "include"),
                           "-o", shim_o, os.path.join(HERE, "penguin_shim.cu")], check=True)
    objs = [os.path.join(objdir, k + ".o") for k in KEEP] + [shim_o]
    subprocess.run(base + ["-o", out] + objs + ["-L" + PKG, "-lpenguin_b200", "-Xlinker", "-rpath=" + PKG],
                   check=True)
    return out


if __name__ == "__main__":
    sys.path.insert(0, ROOT)
    from oracle.ref_build import REFERENCE_ROOT  # where the recipe reads the reference's sources

    print(build(sys.argv[1], sys.argv[2], sys.argv[3], os.path.join(REFERENCE_ROOT, "include")))
