"""pg_global_dt_noalloc: the CFL step size for callers that cannot allocate
device memory (an application whose own pool or fixed budget owns the GPU).
It must return what the allocating entry point pg_grid_global_dt returns on the
same caller-owned buffers, call after call, while keeping its scratch in the
library's fixed file-scope device array.  This file is collected last so that a
run stopping at the first failure has already run every other test."""
import ctypes

import numpy as np
import pytest

import cases as C
from penguin_b200 import params as P
from penguin_b200._lib import PG_ERR_CONFIG, PG_OK, check, lib

pytestmark = pytest.mark.gpu

# the CFL rate is evaluated with divisions here and with reciprocal tables in
# pg_grid_global_dt: a few ulp apart
REL_TOL = 1e-13


def _noalloc_dt(loop, dt_prev):
    out = ctypes.c_double()
    G = loop.G
    st = lib().pg_global_dt_noalloc(ctypes.byref(loop.P), G.C, ctypes.cast(G.xa, ctypes.c_void_p),
                                    ctypes.cast(G.ya, ctypes.c_void_p), ctypes.cast(G.orb_rot, ctypes.c_void_p),
                                    dt_prev, ctypes.byref(out), G.stream)
    check(st)
    return out.value


def _grid_dt(loop, dt_prev):
    out = ctypes.c_double()
    check(lib().pg_grid_global_dt(None, ctypes.byref(loop.G), dt_prev, ctypes.byref(out)))
    return out.value


def test_noalloc_dt_matches_allocating_entry_point_on_two_calls():
    from penguin_b200.grid import ReferenceLoop

    case = [c for c in C.cases() if c["name"] == "disk64_n10"][0]
    loop = ReferenceLoop(case["params"], case["t0"], C.initial_state(case))
    try:
        for call in range(2):  # the second call sees the array as the first one left it
            dt_prev = 1.0e30 if call == 0 else loop.dt
            a = _noalloc_dt(loop, dt_prev)
            b = _grid_dt(loop, dt_prev)
            assert np.isfinite(a) and a > 0.0
            assert a == pytest.approx(b, rel=REL_TOL), (call, a, b)
            loop.step(1)
    finally:
        loop.close()


def test_noalloc_rejects_grids_beyond_its_scratch():
    p = P.planet_disk(8192, 8192)  # 67M interior cells > 8192 * 4096
    PP = P.PGParams.from_params(p)
    out = ctypes.c_double()
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    st = lib().pg_global_dt_noalloc(ctypes.byref(PP), dummy, dummy, dummy, None, 1.0, ctypes.byref(out), None)
    assert st == PG_ERR_CONFIG
    assert b"scratch limit" in lib().pg_last_error()
    assert st != PG_OK
