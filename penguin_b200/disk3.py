"""One 3D grid (ndim 3) on one B200, driven through the C ABI (pg_disk3_*).

The spherical (r, phi, theta) disk of the reference's 3D preset
(include/para_files/Adiabatic_CPD.h) or a cartesian box.  Fields are arrays of
shape (zres, yres, xres), x fastest.  The methods mirror the reference's host
loop (main.cu:320-360) like ``Disk``'s: ``global_dt`` and ``solve`` with host t
and dt, or ``run`` with t, dt and the planet on the device.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import check, lib
from .params import NPAD, Params, PGParams

FIELDS = ("r", "p", "u", "v", "w")


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Disk3:
    STAGES = ("time", "kick1", "sweep_x", "sweep_y", "sweep_z", "kick2")

    def __init__(self, params: Params, device: int = 0, stream: int | None = None):
        if params.ndim != 3:
            raise ValueError("Disk3 needs ndim 3")
        self.params = params
        self._P = PGParams.from_params(params)
        h = ctypes.c_void_p()
        check(lib().pg_disk3_create(ctypes.byref(self._P), device, ctypes.c_void_p(stream or 0), ctypes.byref(h)))
        self._h = h
        self.t = 0.0
        self.dt = None

    @property
    def shape(self):
        p = self.params
        return (p.zres, p.yres, p.xres)

    def set_state(self, t: float, state: dict) -> None:
        """Restart injection: interior fields (zres, yres, xres), like load_grid."""
        f = {k: np.ascontiguousarray(state[k], dtype=np.float64) for k in FIELDS}
        for k in FIELDS:
            if f[k].shape != self.shape:
                raise ValueError(f"{k}: shape {f[k].shape}, expected {self.shape}")
        check(lib().pg_disk3_set_state(self._h, t, *(_dp(f[k]) for k in FIELDS)))
        self.t = t
        self.dt = None

    def get_state(self) -> dict:
        out = {k: np.empty(self.shape) for k in FIELDS}
        t = ctypes.c_double()
        check(lib().pg_disk3_get_state(self._h, *(_dp(out[k]) for k in FIELDS), ctypes.byref(t)))
        out["t"] = t.value
        return out

    def global_dt(self, dt_prev: float) -> float:
        out = ctypes.c_double()
        check(lib().pg_disk3_global_dt(self._h, dt_prev, ctypes.byref(out)))
        return out.value

    def solve(self, t: float, dt: float) -> None:
        check(lib().pg_disk3_solve(self._h, t, dt))

    def step_host(self, max_step: int, end_time: float = 1.0e30) -> int:
        """main.cu:320-360 driven from the host: dt from global_dt, clipped at end_time."""
        dt = self.dt if self.dt else end_time - self.t
        n = 0
        while n < max_step:
            dt = self.global_dt(dt)
            last = False
            if self.t + dt > end_time:
                dt = end_time - self.t
                last = True
            self.solve(self.t, dt)
            self.t += dt
            n += 1
            if last:
                break
        self.dt = dt
        return n

    def run(self, nsteps: int, end_time: float = 1.0e30) -> None:
        """nsteps of the device-resident loop (stream-ordered; call check())."""
        check(lib().pg_disk3_run(self._h, nsteps, end_time))

    def clock(self):
        t, dt, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_longlong()
        check(lib().pg_disk3_clock(self._h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(n)))
        return t.value, dt.value, n.value

    def check(self) -> None:
        check(lib().pg_disk3_check(self._h))

    def pass_times(self, nsteps: int) -> dict:
        """Average ms of each pass over nsteps device-clocked steps (CUDA events)."""
        ms = (ctypes.c_double * 6)()
        check(lib().pg_disk3_pass_times(self._h, nsteps, ms))
        return {k: float(ms[n]) for n, k in enumerate(self.STAGES)}

    def write_snapshot(self, path: str) -> None:
        """The newest state in the reference's checkpoint format (ndim 3)."""
        check(lib().pg_disk3_write_snapshot(self._h, str(path).encode()))

    def read_snapshot(self, path: str) -> float:
        """Restart from a checkpoint file (t and the five fields, like load_grid)."""
        t = ctypes.c_double()
        check(lib().pg_disk3_read_snapshot(self._h, str(path).encode(), ctypes.byref(t)))
        self.t = t.value
        self.dt = None
        return t.value

    def stages(self, t: float, dt: float) -> np.ndarray:
        """One step with host t and dt; the cell array (zarr, yarr, xarr, 5) after
        each pass: kick1, sweep_x, sweep_y, sweep_z, kick2 (test support)."""
        p = self.params
        out = np.zeros((5, p.zarr, p.yarr, p.xarr, 5))
        check(lib().pg_disk3_stages(self._h, t, dt, _dp(out)))
        self.t = t + dt
        return out

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().pg_disk3_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_axis(params: Params, axis: int):
    """The library's host grid along one axis (faces and volumes with ghosts)."""
    P = PGParams.from_params(params)
    n = (params.xarr, params.yarr, params.zarr)[axis]
    a, v = np.zeros(n + 1), np.zeros(n)
    check(lib().pg_make_axis(ctypes.byref(P), axis, _dp(a), _dp(v)))
    return a, v


__all__ = ["Disk3", "make_axis", "NPAD"]
