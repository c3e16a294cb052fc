"""Ensembles of planet-disks advanced by the FP32-mixed step (pg_ens_* C ABI).

Each member is a 2D polar, isothermal disk with its own parameters (size,
planet mass, alpha, h/r ...).  All members step together, one persistent
kernel launch per pass for the whole ensemble, the step captured in a CUDA
graph; each member keeps its own clock and CFL step size.  An ensemble of one
is the FP32-mixed form of a single disk.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np

from ._lib import PGBody, check, lib
from .params import Params, PGParams


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def check_params(params: Sequence[Params]) -> None:
    """Raises PGError if a member is outside the FP32 form (no GPU needed)."""
    arr = (PGParams * len(params))(*[PGParams.from_params(p) for p in params])
    check(lib().pg_ens_check_params(arr, len(params)))


class Ensemble:
    STAGES = ("time", "kick1", "sweep_x", "sweep_y", "advect", "kick2")

    def __init__(self, params: Sequence[Params], device: int = 0, stream: int | None = None):
        self.params = list(params)
        self._P = (PGParams * len(self.params))(*[PGParams.from_params(p) for p in self.params])
        h = ctypes.c_void_p()
        check(lib().pg_ens_create(self._P, len(self.params), device, ctypes.c_void_p(stream or 0), ctypes.byref(h)))
        self._h = h

    def __len__(self) -> int:
        return len(self.params)

    def set_state(self, k: int, t: float, state: dict) -> None:
        """Interior fields (yres, xres) of member k: r, u and optionally v (p is cs^2 r)."""
        r = np.ascontiguousarray(state["r"], dtype=np.float64)
        u = np.ascontiguousarray(state["u"], dtype=np.float64)
        v = state.get("v")
        vv = np.ascontiguousarray(v, dtype=np.float64) if v is not None else None
        check(lib().pg_ens_set_state(self._h, k, t, _dp(r), _dp(u), _dp(vv) if vv is not None else None))

    def set_dust(self, k: int, dust: dict) -> None:
        """Interior dust r, u, v (yres, xres) of dust_flag member k."""
        f = {n: np.ascontiguousarray(dust[n], dtype=np.float64) for n in ("r", "u", "v")}
        check(lib().pg_ens_set_dust(self._h, k, _dp(f["r"]), _dp(f["u"]), _dp(f["v"])))

    def get_dust(self, k: int) -> dict:
        p = self.params[k]
        out = {n: np.empty((p.yres, p.xres)) for n in ("r", "u", "v")}
        check(lib().pg_ens_get_dust(self._h, k, _dp(out["r"]), _dp(out["u"]), _dp(out["v"])))
        return out

    def get_state(self, k: int) -> dict:
        p = self.params[k]
        out = {n: np.empty((p.yres, p.xres)) for n in ("r", "p", "u", "v")}
        t = ctypes.c_double()
        check(lib().pg_ens_get_state(self._h, k, _dp(out["r"]), _dp(out["p"]), _dp(out["u"]), _dp(out["v"]),
                                     ctypes.byref(t)))
        out["t"] = t.value
        return out

    def run(self, nsteps: int, end_time: float = 1.0e30) -> None:
        """nsteps of every member (stream-ordered; call sync())."""
        check(lib().pg_ens_run(self._h, nsteps, end_time))

    def sync(self) -> None:
        check(lib().pg_ens_sync(self._h))

    def clock(self, k: int):
        t, dt, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_longlong()
        check(lib().pg_ens_clock(self._h, k, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(n)))
        return t.value, dt.value, n.value

    def planet(self, k: int) -> dict:
        b = PGBody()
        check(lib().pg_ens_planet(self._h, k, ctypes.byref(b)))
        return {n: getattr(b, n) for n, _ in PGBody._fields_}

    def check(self) -> None:
        check(lib().pg_ens_check(self._h))

    def totals(self, k: int):
        """(mass, angular momentum) of member k, FP64 compensated sums."""
        m, l = ctypes.c_double(), ctypes.c_double()
        check(lib().pg_ens_totals(self._h, k, ctypes.byref(m), ctypes.byref(l)))
        return m.value, l.value

    def torque(self, k: int) -> float:
        """Torque of the planet on member k (unnormalised, as Disk.torque)."""
        out = ctypes.c_double()
        check(lib().pg_ens_torque(self._h, k, ctypes.byref(out)))
        return out.value

    TUNING = ("v_kick1", "v_sweep_x", "v_sweep_y", "v_advect", "v_kick2",
              "cps_kick1", "cps_sweep_x", "cps_sweep_y", "cps_advect", "cps_kick2")

    def autotune(self, reps: int = 5) -> dict:
        """Times the compiled occupancy variants and CTAs-per-SM caps of each pass
        on the current state and keeps the fastest (results are unchanged)."""
        out = (ctypes.c_int * 10)()
        check(lib().pg_ens_autotune(self._h, reps, out))
        return {k: int(out[n]) for n, k in enumerate(self.TUNING)}

    def set_tuning(self, choice: dict) -> None:
        arr = (ctypes.c_int * 10)(*[int(choice[k]) for k in self.TUNING])
        check(lib().pg_ens_set_tuning(self._h, arr))

    def profile(self, nsteps: int, end_time: float = 1.0e30) -> dict:
        ms = (ctypes.c_float * 6)()
        check(lib().pg_ens_profile(self._h, nsteps, end_time, ms, 6))
        return {k: float(ms[n]) for n, k in enumerate(self.STAGES)}

    @property
    def kernels_per_step(self) -> int:
        return lib().pg_ens_kernels_per_step(self._h)

    @property
    def cells(self) -> int:
        return sum(p.xres * p.yres for p in self.params)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().pg_ens_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
