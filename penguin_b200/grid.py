"""The drop-in path: the reference's ``Grid`` struct and main.cu's step loop on
the pg_grid_* entry points.

``ReferenceLoop`` allocates the device buffers the way main.cu does
(main.cu:165-258), fills them the way init()/load_grid()/init_planet() do,
and then calls pg_grid_global_dt / pg_grid_solve exactly where main.cu calls
global_dt / solve (main.cu:320-355).  It exists to exercise the C ABI that a
relinked main.cu uses; device memory comes from torch's allocator.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import PGBody, check, lib
from .disk import make_grid
from .params import NPAD, PI, HPI, Params, PGParams

_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int)
_v = ctypes.c_void_p


def _d2d(dst: int, src: int, nbytes: int) -> None:
    from cuda.bindings import runtime as rt

    (err,) = rt.cudaMemcpy(dst, src, nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToDevice)
    if int(err) != 0:
        raise RuntimeError(f"cudaMemcpy failed: {err}")


class PGGrid(ctypes.Structure):
    """Layout twin of pg_grid / the reference's Grid (include/structs.h:122-183)."""

    _fields_ = [
        ("stream", _v),
        ("xbgn", ctypes.c_int), ("xres", ctypes.c_int), ("xarr", ctypes.c_int),
        ("ybgn", ctypes.c_int), ("yres", ctypes.c_int), ("yarr", ctypes.c_int),
        ("zbgn", ctypes.c_int), ("zres", ctypes.c_int), ("zarr", ctypes.c_int),
        ("xa", _d), ("xv", _d), ("ya", _d), ("yv", _d), ("za", _d), ("zv", _d),
        ("dt", _d), ("sum", _d), ("Buff", _d),
        ("orb_rot", _d), ("orb_res", _d),
        ("orb_shf", _i), ("orb_inc", _i), ("shfL", _i), ("shfR", _i),
        ("C", _v), ("T", _v), ("A", _v),
        ("CD", _v), ("TD", _v),
        ("BuffL", _v), ("BuffR", _v),
        ("BuffLD", _v), ("BuffRD", _v),
        ("vis_tensor", _d), ("fx", _d), ("fy", _d), ("fz", _d), ("fx_d", _d), ("fy_d", _d), ("fz_d", _d),
        ("ext", _d),
        ("planets", _v),
    ]


def _orbit_solution(p: Params, t: float) -> PGBody:
    """init_planet for one planet on a circular orbit (src/planet/planet.cu:105-133, 319-402)."""
    import math

    a, e = p.planet_radius, p.planet_ecc
    if e != 0.0:
        raise NotImplementedError("host-side init of eccentric planets")
    n = math.sqrt(1.0 / a / a / a)
    f = math.fmod(n * t, 2.0 * PI)
    b = PGBody()
    b.m = p.planet_mass * math.sin(HPI * t / p.ramp_time) if t < p.ramp_time else p.planet_mass
    b.a, b.e = a, e
    b.x = a * 1.0 * 1.0 / (1.0 + 0.0)
    b.y = f - math.fmod(p.frame_omega * t, 2.0 * PI) + PI
    b.z = HPI
    b.vx, b.vy, b.vz = 0.0, n, 0.0
    b.rs = p.rs_fac * p.sc_h * a if p.ndim == 2 else p.rs_fac * (p.planet_mass / 3.0) ** (1.0 / 3.0) * a
    return b


class ReferenceLoop:
    def __init__(self, params: Params, t0: float, state: dict, device: int = 0):
        import torch

        self.torch = torch
        self.p = params
        dev = torch.device("cuda", device)
        self.stream = torch.cuda.Stream(device=dev)
        xarr, yarr = params.xarr, params.yarr
        n = xarr * yarr
        xa, xv, ya, yv = make_grid(params)
        self._keep = {}

        def dbuf(name, arr=None, size=None, dtype=torch.float64):
            t = torch.zeros(size if size is not None else arr.size, dtype=dtype, device=dev)
            if arr is not None:
                t.copy_(torch.from_numpy(np.array(arr, copy=True, order="C")))
            self._keep[name] = t
            return t.data_ptr()

        G = PGGrid()
        G.stream = self.stream.cuda_stream
        G.xbgn, G.xres, G.xarr = 0, params.xres, xarr
        G.ybgn, G.yres, G.yarr = 0, params.yres, yarr
        G.zbgn, G.zres, G.zarr = 0, 1, 1
        G.xa = ctypes.cast(dbuf("xa", xa), _d)
        G.xv = ctypes.cast(dbuf("xv", xv), _d)
        G.ya = ctypes.cast(dbuf("ya", ya), _d)
        G.yv = ctypes.cast(dbuf("yv", yv), _d)
        # fill_grid (init_C everywhere, ghosts included) then load_grid's interior fields
        cells = self._initial_cells(params, state)
        G.C = dbuf("C", cells.ravel())
        G.T = dbuf("T", size=5 * n)
        G.vis_tensor = ctypes.cast(dbuf("vis", size=2 * n), _d)
        G.orb_rot = ctypes.cast(dbuf("rot", size=xarr), _d)
        G.orb_res = ctypes.cast(dbuf("res", size=xarr), _d)
        G.orb_shf = ctypes.cast(dbuf("shf", size=xarr, dtype=torch.int32), _i)
        G.orb_inc = ctypes.cast(dbuf("inc", size=xarr, dtype=torch.int32), _i)
        body = _orbit_solution(params, t0)
        raw = np.frombuffer(bytes(body), dtype=np.float64)
        G.planets = dbuf("planets", raw)
        self.G = G
        torch.cuda.synchronize(dev)
        self.P = PGParams.from_params(params)
        check(lib().pg_configure(ctypes.byref(self.P)))
        check(lib().pg_grid_init_orbadv(ctypes.byref(G)))
        self.t = t0
        self.dt = None

    def _initial_cells(self, p: Params, state: dict) -> np.ndarray:
        """init_C at every cell from the library's analytic state, interior from ``state``."""
        from .disk import Disk

        d = Disk(p)
        d.set_state(0.0, state)
        ptr = d.state_ptr()
        a = self.torch.empty((p.yarr, p.xarr, 5), dtype=self.torch.float64, device="cuda")
        self.torch.cuda.synchronize()
        _d2d(a.data_ptr(), ptr, a.numel() * 8)
        self.torch.cuda.synchronize()
        out = a.cpu().numpy()
        d.close()
        return out

    def step(self, max_step: int, end_time: float = 1.0e30) -> int:
        """main.cu:320-355 on the drop-in entry points."""
        dt = self.dt if self.dt else end_time - self.t
        n = 0
        while n < max_step:
            out = ctypes.c_double()
            check(lib().pg_grid_global_dt(None, ctypes.byref(self.G), dt, ctypes.byref(out)))
            dt = out.value
            last = False
            if self.t + dt > end_time:
                dt = end_time - self.t
                last = True
            check(lib().pg_grid_solve(ctypes.byref(self.G), self.t, dt))
            self.t += dt
            n += 1
            if last:
                break
        self.dt = dt
        self.stream.synchronize()
        return n

    def interior(self) -> dict:
        """The newest state (the caller's C after the swaps) as interior fields."""
        p = self.p
        n = p.xarr * p.yarr
        a = self.torch.empty(5 * n, dtype=self.torch.float64, device="cuda")
        _d2d(a.data_ptr(), self.G.C, 5 * n * 8)
        self.torch.cuda.synchronize()
        c = a.cpu().numpy().reshape(p.yarr, p.xarr, 5)
        j0, i0 = p.ypad, NPAD
        sl = c[j0:j0 + p.yres, i0:i0 + p.xres]
        return {k: sl[..., n].copy() for n, k in enumerate("rpuvw")}

    def close(self):
        lib().pg_grid_release()
