"""One disk (or tube) on one B200, driven through the C ABI.

``Disk`` owns its device state.  Its methods mirror the reference's host loop
(main.cu:320-360): ``global_dt`` (src/timestep/timestep.cu:113) and ``solve``
(src/solver/solve.cu:279) with host-side t and dt, or ``run`` which keeps t, dt
and the planet on the device and replays the step as a CUDA graph.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import PGBody, check, lib
from .params import NPAD, Params, PGParams


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Disk:
    def __init__(self, params: Params, device: int = 0, stream: int | None = None):
        self.params = params
        self._P = PGParams.from_params(params)
        h = ctypes.c_void_p()
        check(lib().pg_disk_create(ctypes.byref(self._P), device, ctypes.c_void_p(stream or 0), ctypes.byref(h)))
        self._h = h
        self.t = 0.0
        self.dt = None

    # --------------------------------------------------------------- state
    def set_state(self, t: float, state: dict) -> None:
        """Restart injection: interior fields (yres, xres), like load_grid."""
        f = {k: np.ascontiguousarray(state[k], dtype=np.float64) for k in ("r", "p", "u")}
        v = state.get("v")
        vv = np.ascontiguousarray(v, dtype=np.float64) if v is not None else None
        check(lib().pg_disk_set_state(self._h, t, _dp(f["r"]), _dp(f["p"]), _dp(f["u"]),
                                      _dp(vv) if vv is not None else None))
        self.t = t
        self.dt = None

    def get_state(self) -> dict:
        shape = (self.params.yres, self.params.xres)
        out = {k: np.empty(shape) for k in ("r", "p", "u", "v")}
        t = ctypes.c_double()
        check(lib().pg_disk_get_state(self._h, _dp(out["r"]), _dp(out["p"]), _dp(out["u"]), _dp(out["v"]),
                                      ctypes.byref(t)))
        out["t"] = t.value
        return out

    def set_dust(self, dust: dict) -> None:
        """Interior dust fields r, u, v (yres, xres) of a dust_flag disk; set_state
        resets the dust to init_CD first, like the reference's restart."""
        f = {k: np.ascontiguousarray(dust[k], dtype=np.float64) for k in ("r", "u", "v")}
        check(lib().pg_disk_set_dust(self._h, _dp(f["r"]), _dp(f["u"]), _dp(f["v"])))

    def get_dust(self) -> dict:
        shape = (self.params.yres, self.params.xres)
        out = {k: np.empty(shape) for k in ("r", "u", "v")}
        check(lib().pg_disk_get_dust(self._h, _dp(out["r"]), _dp(out["u"]), _dp(out["v"])))
        return out

    def state_ptr(self) -> int:
        p = ctypes.c_void_p()
        check(lib().pg_disk_state_ptr(self._h, ctypes.byref(p)))
        return p.value

    @property
    def dims(self):
        xa, ya, npad = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib().pg_disk_dims(self._h, ctypes.byref(xa), ctypes.byref(ya), ctypes.byref(npad)))
        return xa.value, ya.value, npad.value

    # ------------------------------------------------------------ stepping
    def global_dt(self, dt_prev: float) -> float:
        out = ctypes.c_double()
        check(lib().pg_disk_global_dt(self._h, dt_prev, ctypes.byref(out)))
        return out.value

    def solve(self, t: float, dt: float) -> None:
        check(lib().pg_disk_solve(self._h, t, dt))

    def step_host(self, max_step: int, end_time: float = 1.0e30) -> int:
        """main.cu:320-360 driven from the host: dt from global_dt (read back every
        step), clipped at end_time, then solve; the loop runs in the library
        (pg_disk_step_host)."""
        t, dt, n = ctypes.c_double(self.t), ctypes.c_double(self.dt or 0.0), ctypes.c_int(0)
        s = lib().pg_disk_step_host(self._h, max_step, end_time, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(n))
        self.t, self.dt = t.value, dt.value
        check(s)
        return n.value

    def run(self, nsteps: int, end_time: float = 1.0e30) -> None:
        """nsteps of the device-resident loop (stream-ordered; call sync())."""
        check(lib().pg_disk_run(self._h, nsteps, end_time))

    def sync(self) -> None:
        check(lib().pg_disk_sync(self._h))

    def clock(self):
        t, dt, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_longlong()
        check(lib().pg_disk_clock(self._h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(n)))
        return t.value, dt.value, n.value

    def planet(self) -> dict:
        b = PGBody()
        check(lib().pg_disk_planet(self._h, ctypes.byref(b)))
        return {k: getattr(b, k) for k, _ in PGBody._fields_}

    def check(self) -> None:
        check(lib().pg_disk_check(self._h))

    def torque(self) -> float:
        """Torque of the planet on the disk (unnormalised; the reference prints it / (q^2/h^2))."""
        out = ctypes.c_double()
        check(lib().pg_disk_torque(self._h, ctypes.byref(out)))
        return out.value

    # ---------------------------------------------------- snapshots, averages
    def write_snapshot(self, path: str, average: bool = False) -> None:
        """The newest state (or the time average) in the reference's checkpoint format."""
        check(lib().pg_disk_write_snapshot(self._h, str(path).encode(), int(average)))

    def read_snapshot(self, path: str) -> float:
        """Restart from a checkpoint file (t and the gas fields, like load_grid)."""
        t = ctypes.c_double()
        check(lib().pg_disk_read_snapshot(self._h, str(path).encode(), ctypes.byref(t)))
        self.t = t.value
        self.dt = None
        return t.value

    def set_average(self, interval: float) -> None:
        """ave_flag: average the gas over a save interval (0 switches it off)."""
        check(lib().pg_disk_set_average(self._h, interval))

    def reset_average(self) -> None:
        check(lib().pg_disk_reset_average(self._h))

    def get_average(self) -> dict:
        shape = (self.params.yres, self.params.xres)
        out = {k: np.empty(shape) for k in ("r", "p", "u", "v")}
        check(lib().pg_disk_get_average(self._h, _dp(out["r"]), _dp(out["p"]), _dp(out["u"]), _dp(out["v"])))
        return out

    TUNING = ("v_sweep_x", "v_sweep_y", "v_advect", "cps_kick1", "cps_sweep_x", "cps_sweep_y", "cps_advect",
              "cps_kick2")

    def autotune(self, reps: int = 10) -> dict:
        """Times every launch configuration of each pass on the current state and
        keeps the fastest (results stay bit for bit the same).  Returns the raw
        choice (TUNING keys) and, under "passes", every pass's knobs."""
        out = (ctypes.c_int * 8)()
        check(lib().pg_disk_autotune(self._h, reps, out))
        choice = {k: int(out[n]) for n, k in enumerate(self.TUNING)}
        return dict(choice, passes=describe_tuning(choice))

    def set_tuning(self, choice: dict) -> None:
        arr = (ctypes.c_int * 8)(*[int(choice[k]) for k in self.TUNING])
        check(lib().pg_disk_set_tuning(self._h, arr))

    STAGES = ("time", "kick1", "sweep_x", "sweep_y", "advect", "kick2")

    def profile(self, nsteps: int, end_time: float = 1.0e30) -> dict:
        """Average ms per step of each stage (CUDA events between the launches)."""
        ms = (ctypes.c_float * 6)()
        check(lib().pg_disk_profile(self._h, nsteps, end_time, ms, 6))
        return {k: float(ms[n]) for n, k in enumerate(self.STAGES)}

    @property
    def kernels_per_step(self) -> int:
        return lib().pg_kernels_per_step(self._h)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().pg_disk_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sweep_variant(v: int) -> dict:
    """Knobs of tile variant v of the sweeps and the residual advection."""
    out = (ctypes.c_int * 6)()
    check(lib().pg_sweep_variant(v, out))
    return {"pencils_per_tile": out[0], "pencil_length": out[1], "cells_per_thread": out[2],
            "tma_stages": out[3], "threads": out[4], "ctas_per_sm_compiled": out[5]}


def describe_tuning(choice: dict) -> dict:
    """Every pass's launch knobs from an autotuner choice (Disk.TUNING keys)."""
    out = {}
    for p in ("kick1", "sweep_x", "sweep_y", "advect", "kick2"):
        k = {"ctas_per_sm": choice["cps_" + p] or "all that fit"}
        if p in ("sweep_x", "sweep_y", "advect"):
            k.update(sweep_variant(choice["v_" + p]))
        else:  # the stencil passes: 32 x 8 cells per tile, one cell per thread, two TMA stages
            k.update({"tile": "32x8", "cells_per_thread": 1, "tma_stages": 2})
        out[p] = k
    return out


def make_grid(params: Params):
    """The library's host grid (faces and volumes with ghosts)."""
    P = PGParams.from_params(params)
    xarr, yarr = params.xres + 2 * NPAD, params.yres + 2 * params.ypad
    xa, xv, ya, yv = np.zeros(xarr + 1), np.zeros(xarr), np.zeros(yarr + 1), np.zeros(yarr)
    check(lib().pg_make_grid(ctypes.byref(P), _dp(xa), _dp(xv), _dp(ya), _dp(yv)))
    return xa, xv, ya, yv
