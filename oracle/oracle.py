"""ctypes binding of the CPU oracle (oracle.c) -- TEST INFRASTRUCTURE ONLY.

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` load this module; the product never does.  ``Oracle`` drives the
restated reference step exactly like main.cu's loop drives solve()/global_dt().
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("ndim", ctypes.c_int), ("xres", ctypes.c_int), ("yres", ctypes.c_int),
        ("geomx", ctypes.c_int), ("geomy", ctypes.c_int), ("gridx", ctypes.c_int), ("gridy", ctypes.c_int),
        ("xmin", ctypes.c_double), ("xmax", ctypes.c_double), ("ymin", ctypes.c_double), ("ymax", ctypes.c_double),
        ("eos_flag", ctypes.c_int), ("internal_e_flag", ctypes.c_int),
        ("gam", ctypes.c_double), ("cfl", ctypes.c_double),
        ("bound_lft", ctypes.c_int), ("bound_rgh", ctypes.c_int), ("init_flag", ctypes.c_int),
        ("frame_omega", ctypes.c_double),
        ("p_alpha", ctypes.c_double), ("p_beta", ctypes.c_double), ("ss_alpha", ctypes.c_double),
        ("sc_h", ctypes.c_double), ("planet_radius", ctypes.c_double),
        ("visc_flag", ctypes.c_int), ("orbadv_flag", ctypes.c_int), ("kill_flag", ctypes.c_int),
        ("kill_width", ctypes.c_double), ("kill_width_out", ctypes.c_double),
        ("n_planet", ctypes.c_int),
        ("planet_mass", ctypes.c_double), ("planet_ecc", ctypes.c_double),
        ("rs_fac", ctypes.c_double), ("ramp_time", ctypes.c_double),
        ("zmin", ctypes.c_double), ("zmax", ctypes.c_double),
        ("dust_flag", ctypes.c_int), ("stokes", ctypes.c_double), ("d_g_ratio", ctypes.c_double),
        ("cool_flag", ctypes.c_int), ("beta_cool", ctypes.c_double),
        ("twobd_flag", ctypes.c_int),
        ("zres", ctypes.c_int), ("geomz", ctypes.c_int), ("gridz", ctypes.c_int),
        ("bound_bom", ctypes.c_int), ("bound_top", ctypes.c_int),
    ]

    @classmethod
    def from_params(cls, p) -> "OrcParams":
        return cls(
            p.ndim, p.xres, p.yres, p.geomx, p.geomy, p.gridx, p.gridy,
            p.xmin, p.xmax, p.ymin, p.ymax, p.EOS_flag, p.internal_e_flag, p.gam, p.CFL,
            p.bound_lft, p.bound_rgh, p.init_flag, p.frame_omega,
            p.p_alpha, p.p_beta, p.ss_alpha, p.sc_h, p.planet_radius,
            p.visc_flag, p.OrbAdv_flag, p.kill_flag, p.kill_width, p.kill_width_out,
            p.n_planet, p.planet_mass, p.planet_ecc, p.rs_fac, p.ramp_time, p.zmin, p.zmax,
            p.dust_flag, p.Stokes, p.D_G_ratio, p.cool_flag, p.beta_cool, p.twobd_flag,
            p.zres, p.geomz, p.gridz, p.bound_bom, p.bound_top,
        )


class OrcBody(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("m", "a", "e", "x", "y", "z", "vx", "vy", "vz", "rs")]


def build(force: bool = False) -> str:
    """Compile liboracle.so with the Makefile beside this file."""
    srcs = [os.path.join(HERE, f) for f in ("oracle.c", "oracle3d.c", "oracle.h")]
    if force or not os.path.exists(LIB_PATH) or any(os.path.getmtime(LIB_PATH) < os.path.getmtime(f) for f in srcs):
        subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [ctypes.POINTER(OrcParams)]
        L.orc_destroy.argtypes = [vp]
        L.orc_dims.argtypes = [vp, ip, ip]
        L.orc_get_grid.argtypes = [vp, dp, dp, dp, dp]
        L.orc_fill_init.argtypes = [vp]
        L.orc_set_interior.argtypes = [vp, dp, dp, dp, dp]
        L.orc_get_interior.argtypes = [vp, dp, dp, dp, dp]
        L.orc_get_cells.argtypes = [vp, dp]
        L.orc_init_planet.argtypes = [vp, ctypes.c_double]
        L.orc_init_orbadv.argtypes = [vp]
        L.orc_get_planet.argtypes = [vp, ctypes.POINTER(OrcBody)]
        L.orc_global_dt.restype = ctypes.c_double
        L.orc_global_dt.argtypes = [vp, ctypes.c_double]
        L.orc_torque.restype = ctypes.c_double
        L.orc_torque.argtypes = [vp]
        L.orc_set_dust.argtypes = [vp, dp, dp, dp]
        L.orc_get_dust.argtypes = [vp, dp, dp, dp]
        L.orc_solve.argtypes = [vp, ctypes.c_double, ctypes.c_double]
        L.orc_run.restype = ctypes.c_int
        L.orc_run.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double, dp, dp]
        for name in ("orc_boundx", "orc_boundy"):
            getattr(L, name).argtypes = [vp, ctypes.c_int]
        L.orc_viscous_forces.argtypes = [vp, ctypes.c_int, dp]
        L.orc_sweepx.argtypes = [vp, ctypes.c_double]
        L.orc_sweepy.argtypes = [vp, ctypes.c_double]
        L.orc_solve_stages.restype = ctypes.c_int
        L.orc_solve_stages.argtypes = [vp, ctypes.c_double, ctypes.c_double, dp, dp]
        L.orc3_create.restype = vp
        L.orc3_create.argtypes = [ctypes.POINTER(OrcParams)]
        L.orc3_destroy.argtypes = [vp]
        L.orc3_dims.restype = ctypes.c_int
        L.orc3_dims.argtypes = [vp, ip, ip, ip]
        L.orc3_get_axis.argtypes = [vp, ctypes.c_int, dp, dp]
        L.orc3_fill_init.argtypes = [vp]
        L.orc3_set_interior.argtypes = [vp, dp, dp, dp, dp, dp]
        L.orc3_get_interior.argtypes = [vp, dp, dp, dp, dp, dp]
        L.orc3_init_planet.argtypes = [vp, ctypes.c_double]
        L.orc3_get_planet.argtypes = [vp, ctypes.POINTER(OrcBody)]
        for name in ("orc3_boundx", "orc3_boundy", "orc3_boundz"):
            getattr(L, name).argtypes = [vp]
        for name in ("orc3_sweepx", "orc3_sweepy", "orc3_sweepz"):
            getattr(L, name).argtypes = [vp, ctypes.c_double]
        L.orc3_global_dt.restype = ctypes.c_double
        L.orc3_global_dt.argtypes = [vp, ctypes.c_double]
        L.orc3_solve.argtypes = [vp, ctypes.c_double, ctypes.c_double]
        L.orc3_solve_stages.restype = ctypes.c_int
        L.orc3_solve_stages.argtypes = [vp, ctypes.c_double, ctypes.c_double, dp]
        L.orc3_run.restype = ctypes.c_int
        L.orc3_run.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double, dp, dp]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Oracle:
    """One disk/tube on the CPU, stepping like the reference's main loop."""

    def __init__(self, params, state: dict | None = None, t0: float = 0.0):
        self.p = params
        self._P = OrcParams.from_params(params)
        self.h = lib().orc_create(ctypes.byref(self._P))
        xa, ya = ctypes.c_int(), ctypes.c_int()
        lib().orc_dims(self.h, ctypes.byref(xa), ctypes.byref(ya))
        self.xarr, self.yarr = xa.value, ya.value
        lib().orc_fill_init(self.h)
        if state is not None:
            self.set_interior(state)
        self.t = t0
        self.dt = None
        lib().orc_init_planet(self.h, t0)
        lib().orc_init_orbadv(self.h)

    def close(self) -> None:
        h = getattr(self, "h", None)
        if h:
            lib().orc_destroy(h)
            self.h = None

    def __del__(self):
        self.close()

    def grid(self):
        xa = np.zeros(self.xarr + 1); xv = np.zeros(self.xarr)
        ya = np.zeros(self.yarr + 1); yv = np.zeros(self.yarr)
        lib().orc_get_grid(self.h, _dp(xa), _dp(xv), _dp(ya), _dp(yv))
        return xa, xv, ya, yv

    def set_interior(self, s: dict) -> None:
        f = {k: np.ascontiguousarray(s[k], dtype=np.float64) for k in ("r", "p", "u")}
        v = np.ascontiguousarray(s.get("v", np.zeros_like(f["r"])), dtype=np.float64)
        lib().orc_set_interior(self.h, _dp(f["r"]), _dp(f["p"]), _dp(f["u"]), _dp(v))

    def interior(self) -> dict:
        shape = (self.p.yres, self.p.xres)
        out = {k: np.zeros(shape) for k in ("r", "p", "u", "v")}
        lib().orc_get_interior(self.h, _dp(out["r"]), _dp(out["p"]), _dp(out["u"]), _dp(out["v"]))
        return out

    def cells(self) -> np.ndarray:
        a = np.zeros((self.yarr, self.xarr, 5))
        lib().orc_get_cells(self.h, _dp(a))
        return a

    def planet(self) -> dict:
        b = OrcBody()
        lib().orc_get_planet(self.h, ctypes.byref(b))
        return {k: getattr(b, k) for k, _ in OrcBody._fields_}

    def global_dt(self, dt_prev: float) -> float:
        return lib().orc_global_dt(self.h, dt_prev)

    def dust(self) -> dict:
        """Dust interior (dust_flag): r, u, v arrays (yres, xres)."""
        shape = (self.p.yres, self.p.xres)
        out = {k: np.zeros(shape) for k in ("r", "u", "v")}
        lib().orc_get_dust(self.h, _dp(out["r"]), _dp(out["u"]), _dp(out["v"]))
        return out

    def set_dust(self, d: dict) -> None:
        f = {k: np.ascontiguousarray(d[k], dtype=np.float64) for k in ("r", "u", "v")}
        lib().orc_set_dust(self.h, _dp(f["r"]), _dp(f["u"]), _dp(f["v"]))

    def torque(self) -> float:
        """Torque of the planet on the disk (src/output/output.cu:336-412), unnormalised."""
        return lib().orc_torque(self.h)

    def solve(self, t: float, dt: float) -> None:
        lib().orc_solve(self.h, t, dt)

    def solve_stages(self, t: float, dt: float, dust: bool = False):
        """One step, returning the cell array after each stage (see oracle.c);
        with dust=True also the dust arrays after the same stages."""
        buf = np.zeros((12, self.yarr, self.xarr, 5))
        dbuf = np.zeros((12, self.yarr, self.xarr, 4)) if dust else None
        k = lib().orc_solve_stages(self.h, t, dt, _dp(buf), _dp(dbuf) if dust else None)
        return (buf[:k], dbuf[:k]) if dust else buf[:k]

    def run(self, max_step: int, end_time: float = 1.0e30) -> int:
        """main.cu:320-360: dt from global_dt (first call capped by end_time - t),
        clipped at end_time; stops after max_step steps."""
        t_out, dt_out = ctypes.c_double(), ctypes.c_double()
        n = lib().orc_run(self.h, self.t, self.dt if self.dt else -1.0, max_step, end_time,
                         ctypes.byref(t_out), ctypes.byref(dt_out))
        self.t, self.dt = t_out.value, dt_out.value
        return n


FIELDS3 = ("r", "p", "u", "v", "w")


class Oracle3:
    """One 3D grid (ndim 3) on the CPU, stepping like the reference's main loop.
    Fields are arrays of shape (zres, yres, xres)."""

    def __init__(self, params, state: dict | None = None, t0: float = 0.0):
        self.p = params
        self._P = OrcParams.from_params(params)
        self.h = lib().orc3_create(ctypes.byref(self._P))
        xa, ya, za = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        lib().orc3_dims(self.h, ctypes.byref(xa), ctypes.byref(ya), ctypes.byref(za))
        self.xarr, self.yarr, self.zarr = xa.value, ya.value, za.value
        lib().orc3_fill_init(self.h)
        if state is not None:
            self.set_interior(state)
        self.t = t0
        self.dt = None
        lib().orc3_init_planet(self.h, t0)

    def close(self) -> None:
        h = getattr(self, "h", None)
        if h:
            lib().orc3_destroy(h)
            self.h = None

    def __del__(self):
        self.close()

    def axis(self, axis: int):
        n = (self.xarr, self.yarr, self.zarr)[axis]
        a, v = np.zeros(n + 1), np.zeros(n)
        lib().orc3_get_axis(self.h, axis, _dp(a), _dp(v))
        return a, v

    def set_interior(self, s: dict) -> None:
        f = {k: np.ascontiguousarray(s[k], dtype=np.float64) for k in FIELDS3}
        lib().orc3_set_interior(self.h, *(_dp(f[k]) for k in FIELDS3))

    def interior(self) -> dict:
        shape = (self.p.zres, self.p.yres, self.p.xres)
        out = {k: np.zeros(shape) for k in FIELDS3}
        lib().orc3_get_interior(self.h, *(_dp(out[k]) for k in FIELDS3))
        return out

    def planet(self) -> dict:
        b = OrcBody()
        lib().orc3_get_planet(self.h, ctypes.byref(b))
        return {k: getattr(b, k) for k, _ in OrcBody._fields_}

    def global_dt(self, dt_prev: float) -> float:
        return lib().orc3_global_dt(self.h, dt_prev)

    def solve(self, t: float, dt: float) -> None:
        lib().orc3_solve(self.h, t, dt)

    def solve_stages(self, t: float, dt: float):
        """One step, returning the cell arrays (zarr, yarr, xarr, 5) after each stage."""
        buf = np.zeros((6, self.zarr, self.yarr, self.xarr, 5))
        k = lib().orc3_solve_stages(self.h, t, dt, _dp(buf))
        return buf[:k]

    def run(self, max_step: int, end_time: float = 1.0e30) -> int:
        """main.cu:320-360 (see Oracle.run)."""
        t_out, dt_out = ctypes.c_double(), ctypes.c_double()
        n = lib().orc3_run(self.h, self.t, self.dt if self.dt else -1.0, max_step, end_time,
                          ctypes.byref(t_out), ctypes.byref(dt_out))
        self.t, self.dt = t_out.value, dt_out.value
        return n
