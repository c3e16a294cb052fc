"""pg_global_dt_noalloc: the CFL step size for callers that cannot allocate
device memory (an application whose own pool or fixed budget owns the GPU).
It must return what the allocating entry points return on the same state,
call after call, while keeping its scratch in the library's fixed file-scope
device array: on a gas disk, on a gas + dust disk (the dust speeds bound dt)
and on the 1D tube (no azimuthal faces).  This file is collected last so that a
run stopping at the first failure has already run every other test."""
import ctypes

import numpy as np
import pytest

import cases as C
from penguin_b200 import params as P
from penguin_b200._lib import PG_ERR_ARG, PG_ERR_CONFIG, PG_OK, check, lib

pytestmark = pytest.mark.gpu

# the CFL rate is evaluated with divisions here and with reciprocal tables in
# the allocating entry points: a few ulp apart
REL_TOL = 1e-13


def _noalloc_dt(PP, C_ptr, CD_ptr, xa, ya, rot, dt_prev, stream=None):
    out = ctypes.c_double()
    st = lib().pg_global_dt_noalloc(ctypes.byref(PP), C_ptr, CD_ptr, xa, ya, rot, dt_prev, ctypes.byref(out),
                                    stream)
    check(st)
    return out.value


def _grid_dt(loop, dt_prev):
    out = ctypes.c_double()
    check(lib().pg_grid_global_dt(None, ctypes.byref(loop.G), dt_prev, ctypes.byref(out)))
    return out.value


def _vp(p):
    return ctypes.cast(p, ctypes.c_void_p)


def _case(name):
    return [c for c in C.cases() + C.dust_cases() if c["name"] == name][0]


@pytest.mark.parametrize("name", ["disk64_n10", "sod_n10"])
def test_noalloc_dt_matches_allocating_entry_point_on_two_calls(name):
    from penguin_b200.grid import ReferenceLoop

    case = _case(name)
    loop = ReferenceLoop(case["params"], case["t0"], C.initial_state(case))
    try:
        G = loop.G
        ya = _vp(G.ya) if case["params"].ndim > 1 else None  # unused in 1D
        rot = _vp(G.orb_rot) if case["params"].OrbAdv_flag else None
        for call in range(2):  # the second call sees the array as the first one left it
            dt_prev = 1.0e30 if call == 0 else loop.dt
            a = _noalloc_dt(loop.P, G.C, None, _vp(G.xa), ya, rot, dt_prev, G.stream)
            b = _grid_dt(loop, dt_prev)
            assert np.isfinite(a) and a > 0.0
            assert a == pytest.approx(b, rel=REL_TOL), (call, a, b)
            loop.step(1)
    finally:
        loop.close()


def _aos(p, fields, names):
    """Interior host fields into a device AoS array of xarr*yarr records (ghosts zero)."""
    import torch

    a = np.zeros((p.yarr, p.xarr, len(names)))
    for k, n in enumerate(names):
        if n in fields:
            a[p.ypad:p.ypad + p.yres, P.NPAD:P.NPAD + p.xres, k] = fields[n]
    return torch.tensor(a, device="cuda")


def test_noalloc_dt_includes_the_dust_speeds_on_two_calls():
    """A gas + dust disk whose dust moves faster than the gas signal speed in
    some cells: the step must be the allocating path's, which bounds the rate
    by the dust speeds as well (src/timestep/timestep.cu:64-75)."""
    import torch

    from penguin_b200.disk import Disk, make_grid
    from penguin_b200.grid import ReferenceLoop

    case = _case("dust64_st01_n10")
    p = case["params"]
    st = C.initial_state(case)
    # orb_rot of this disk, as init_OrbAdv fills it (the gas disk alone sets it)
    gas = ReferenceLoop(p.replace(dust_flag=0), case["t0"], st)
    d = Disk(p)
    try:
        d.set_state(case["t0"], st)
        dust = d.get_dust()
        # radial dust velocities ten times the gas's largest signal rate in a band
        # of radii, so that they set the step
        dust["u"] = dust["u"].copy()
        dust["u"][:, 20:24] += 20.0
        d.set_dust(dust)
        xa, _, ya, _ = make_grid(p)
        xa_d = torch.tensor(np.asarray(xa), device="cuda")
        ya_d = torch.tensor(np.asarray(ya), device="cuda")
        PP = P.PGParams.from_params(p)
        PG = P.PGParams.from_params(p.replace(dust_flag=0))
        dt_prev = 1.0e30
        for call in range(2):
            g, dd = d.get_state(), d.get_dust()
            Cg = _aos(p, g, "rpuvw")
            Cd = _aos(p, dd, "ruvw")
            torch.cuda.synchronize()
            a = _noalloc_dt(PP, Cg.data_ptr(), Cd.data_ptr(), xa_d.data_ptr(), ya_d.data_ptr(),
                            _vp(gas.G.orb_rot), dt_prev)
            # the gas alone, without the 1.1 dt_prev cap
            gas_only = _noalloc_dt(PG, Cg.data_ptr(), None, xa_d.data_ptr(), ya_d.data_ptr(),
                                   _vp(gas.G.orb_rot), 1.0e30)
            b = d.global_dt(dt_prev)
            assert a == pytest.approx(b, rel=REL_TOL), (call, a, b)
            assert a < 0.5 * gas_only, (a, gas_only)  # the dust speeds set the step
            d.solve(d.t, b)
            d.t += b
            dt_prev = b
    finally:
        d.close()
        gas.close()


def test_noalloc_rejects_bad_arguments():
    out = ctypes.c_double()
    dummy = ctypes.c_void_p(16)  # never dereferenced: the argument checks come first
    # a grid beyond the fixed scratch
    PP = P.PGParams.from_params(P.planet_disk(8192, 8192))  # 67M interior cells > 8192 * 4096
    st = lib().pg_global_dt_noalloc(ctypes.byref(PP), dummy, None, dummy, dummy, None, 1.0, ctypes.byref(out), None)
    assert st == PG_ERR_CONFIG
    assert b"scratch limit" in lib().pg_last_error()
    # dust_flag without the dust state
    PD = P.PGParams.from_params(P.dust_disk(64, 192))
    st = lib().pg_global_dt_noalloc(ctypes.byref(PD), dummy, None, dummy, dummy, None, 1.0, ctypes.byref(out), None)
    assert st == PG_ERR_ARG
    # a 1D grid with more than one row
    PS = P.PGParams.from_params(P.sod_tube(64))
    PS.yres = 4
    st = lib().pg_global_dt_noalloc(ctypes.byref(PS), dummy, None, dummy, None, None, 1.0, ctypes.byref(out), None)
    assert st == PG_ERR_CONFIG
    # a 2D grid without its azimuthal faces
    PP = P.PGParams.from_params(P.planet_disk(64, 192))
    st = lib().pg_global_dt_noalloc(ctypes.byref(PP), dummy, None, dummy, None, None, 1.0, ctypes.byref(out), None)
    assert st == PG_ERR_ARG
    assert st != PG_OK
