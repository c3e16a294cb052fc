"""The C-ABI library: it loads, exports every entry point include/penguin_b200.h
declares, validates parameters and builds the reference's grid bit for bit.
CPU only (no kernel launches)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from oracle.oracle import Oracle
from penguin_b200 import _lib
from penguin_b200 import params as P
from penguin_b200.disk import make_grid

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "penguin_b200.h")


def _declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"\b(pg_[a-z_0-9]+)\s*\(", src)))


def test_header_and_binding_agree():
    assert _declared() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (pg_\w+)", out))
    for name in _declared():
        assert name in exported, name
        assert hasattr(L, name)
    assert b"sm_100a" in L.pg_version()


def test_params_struct_layout_matches_header(tmp_path):
    """Every field offset of the ctypes mirrors equals the C compiler's."""
    structs = {"pg_params": P.PGParams, "pg_body": _lib.PGBody}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "penguin_b200.h"', "int main(void){"]
    for cname, cls in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    for cname, cls in structs.items():
        assert int(got[cname]) == ctypes.sizeof(cls)
        for fname, _ in cls._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(cls, fname).offset, (cname, fname)


@pytest.mark.parametrize("bad", [
    dict(ndim=3), dict(EOS_flag=1), dict(xres=31), dict(bound_lft=3), dict(geomx=2), dict(n_planet=2),
    dict(dust_flag=1, Stokes=0.0), dict(dust_flag=1, init_flag=1), dict(yres=4),
    dict(cool_flag=3), dict(cool_flag=1, beta_cool=0.0),
    dict(twobd_flag=2), dict(twobd_flag=1, n_planet=0), dict(twobd_flag=1, geomx=0, geomy=0),
])
def test_check_params_rejects(bad):
    p = P.planet_disk(64, 192).replace(**bad)
    st = _lib.lib().pg_check_params(ctypes.byref(_raw(p)))
    assert st == _lib.PG_ERR_CONFIG
    assert _lib.lib().pg_last_error()


def _raw(p):
    # bypass the Python-side validation to exercise the C checks
    return P.PGParams(
        p.ndim, p.xres, p.yres, p.geomx, p.geomy, p.gridx, p.gridy, p.xmin, p.xmax, p.ymin, p.ymax,
        p.EOS_flag, p.internal_e_flag, p.gam, p.CFL, p.bound_lft, p.bound_rgh, p.init_flag, p.frame_omega,
        p.p_alpha, p.p_beta, p.ss_alpha, p.sc_h, p.planet_radius, p.visc_flag, p.OrbAdv_flag, p.kill_flag,
        p.kill_width, p.kill_width_out, p.n_planet, p.planet_mass, p.planet_ecc, p.rs_fac, p.ramp_time,
        p.zmin, p.zmax, p.dust_flag, p.Stokes, p.D_G_ratio, p.cool_flag, p.beta_cool, p.twobd_flag)


def test_check_params_accepts_workloads():
    for p in (P.sod_tube(1024), P.planet_disk(1024, 3072), P.reference_disk(64, 192),
              P.reference_disk(64, 192).replace(EOS_flag=2, gam=1.4, cool_flag=2, beta_cool=0.05),
              P.reference_disk(64, 192).replace(twobd_flag=1)):
        assert _lib.lib().pg_check_params(ctypes.byref(_raw(p))) == _lib.PG_OK


@pytest.mark.parametrize("p", [P.sod_tube(1024), P.planet_disk(1024, 3072), P.reference_disk(32, 96)],
                         ids=["sod", "disk1024", "disk32"])
def test_grid_is_bitwise_the_references(p):
    """Faces and volumes with ghosts (src/init/init.cu:472-500) from the library
    equal the oracle's restatement exactly (both use the host libm)."""
    xa, xv, ya, yv = make_grid(p)
    o = Oracle(p)
    oxa, oxv, oya, oyv = o.grid()
    for a, b in ((xa, oxa), (xv, oxv), (ya, oya), (yv, oyv)):
        assert np.array_equal(a, b)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "missing.so"))
    with pytest.raises(RuntimeError, match="missing"):
        _lib.lib()
