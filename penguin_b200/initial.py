"""Seeded initial states for the benchmark and test workloads.

The reference has no Sod problem and no seeded noise (``srand(0)`` is called but
unused, src/init/init.cu:504); these states are injected into it through its
restart path (main.cu:265-274 -> load_grid, src/output/output.cu:182-248), which
loads the interior fields only.  Arrays are (yres, xres), x fastest, like the
snapshot files.
"""
from __future__ import annotations

import math

import numpy as np

from .params import Params, make_grid_np

_M64 = (1 << 64) - 1


def splitmix64_uniform(seed: int, n: int) -> np.ndarray:
    """n deterministic samples of U(-1,1) from the SplitMix64 sequence (Steele,
    Lea & Flood, OOPSLA 2014), identical on every platform."""
    with np.errstate(over="ignore"):
        k = np.arange(1, n + 1, dtype=np.uint64)
        z = (np.uint64(seed & _M64) + k * np.uint64(0x9E3779B97F4A7C15))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    u = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return 2.0 * u - 1.0


def cell_centres(p: Params):
    xa, _ = make_grid_np(p.xmin, p.xmax, p.xres, 3, p.geomx, p.gridx)
    xc = 0.5 * (xa[4:4 + p.xres] + xa[3:3 + p.xres])
    return xc


def _disk_profiles(p: Params, x: np.ndarray):
    """init_flag 2 profiles (src/init/init.cu:7-50, 72-82, 131-145, 240-252)."""
    coeff = p.sc_h * p.sc_h * (1.0 / p.planet_radius)

    def cs2(xx):
        return coeff * np.power(xx / p.planet_radius, -p.p_beta)

    def rho(xx):
        return np.power(xx / p.planet_radius, -p.p_alpha)

    def pres(xx):
        return cs2(xx) * rho(xx)

    dr = 1.1514178e-7
    dPdr = (pres(x + dr) - pres(x - dr)) / (2.0 * dr)
    v = np.sqrt(1.0 / x + (x / rho(x)) * dPdr)
    return rho(x), cs2(x), v


def disk_state(p: Params, seed: int = 1234, noise: float = 1.0e-4, vr: float = 0.0) -> dict:
    """Sigma = Sigma_0(r) (1 + noise U(-1,1)), p = cs^2 Sigma, v_r = ``vr``,
    v_phi = pressure-corrected Keplerian of the unperturbed profile."""
    x = cell_centres(p)
    s0, c2, v = _disk_profiles(p, x)
    shape = (p.yres, p.xres)
    u01 = splitmix64_uniform(seed, p.xres * p.yres).reshape(shape)
    r = s0[None, :] * (1.0 + noise * u01)
    return {
        "r": r,
        "p": c2[None, :] * r,
        "u": np.full(shape, vr),
        "v": np.broadcast_to(v[None, :], shape).copy(),
    }


def sod_state(p: Params, x0: float = 0.5, left=(1.0, 0.0, 1.0), right=(0.125, 0.0, 0.1)) -> dict:
    """Sod (1978) tube: (rho, u, p) = left for cell centres x < x0, right otherwise."""
    x = cell_centres(p)
    L = x < x0
    r = np.where(L, left[0], right[0])[None, :]
    u = np.where(L, left[1], right[1])[None, :]
    pr = np.where(L, left[2], right[2])[None, :]
    return {"r": r.astype(np.float64), "p": pr.astype(np.float64), "u": u.astype(np.float64),
            "v": np.zeros_like(r, dtype=np.float64)}


def orbit_time(orbits: float) -> float:
    return orbits * 2.0 * math.pi


# --------------------------------------------------------------------- 3D
def _centres(a):
    return 0.5 * (a[4:-3] + a[3:-4])


def spherical_state(p: Params, seed: int = 1234, noise: float = 1.0e-4, vnoise: float = 0.0) -> dict:
    """The spherical disk of init_flag 3 (src/init/init.cu:7-71, 90-91, 157-158,
    269-274): Sigma ~ (r sin(theta))^-p_alpha in vertical hydrostatic balance,
    p = cs^2 rho, pressure-corrected Keplerian v_phi; density times
    1 + noise U(-1,1) and, with ``vnoise``, radial and polar velocities of
    vnoise c_s U(-1,1).  Arrays (zres, yres, xres)."""
    from .params import axes_np

    (xa, _), _, (za, _) = axes_np(p)
    x = _centres(xa)[None, None, :]
    z = _centres(za)[:, None, None]
    coeff = p.sc_h * p.sc_h * (1.0 / p.planet_radius)

    def cs2(xx, zz):
        return coeff * np.power(xx * np.sin(zz) / p.planet_radius, -p.p_beta)

    def rho(xx, zz):
        r = xx * np.sin(zz)
        return np.power(r / p.planet_radius, -p.p_alpha) * np.exp((1.0 / xx - 1.0 / r) / cs2(xx, zz))

    def pres(xx, zz):
        return cs2(xx, zz) * rho(xx, zz)

    dr = 1.1514178e-7
    v0 = np.sqrt(1.0 / x + (x / rho(x, z)) * (pres(x + dr, z) - pres(x - dr, z)) / (2.0 * dr))
    shape = (p.zres, p.yres, p.xres)
    u = splitmix64_uniform(seed, 3 * p.cells).reshape((3,) + shape)
    r = rho(x, z) * (1.0 + noise * u[0])
    c2 = np.broadcast_to(cs2(x, z), shape)
    cs = np.sqrt(c2)
    return {"r": r, "p": c2 * r, "u": vnoise * cs * u[1], "v": np.broadcast_to(v0, shape).copy(),
            "w": vnoise * cs * u[2]}


def box_state(p: Params, seed: int = 4321) -> dict:
    """A cartesian box state with structure at every scale: density 1 + 0.2 U,
    pressure 1 + 0.2 U plus a Gaussian overpressure of 2 at (0.3, 0.6, 0.2),
    velocities 0.1 U per component.  Arrays (zres, yres, xres)."""
    from .params import axes_np

    (xa, _), (ya, _), (za, _) = axes_np(p)
    x, y, z = _centres(xa)[None, None, :], _centres(ya)[None, :, None], _centres(za)[:, None, None]
    shape = (p.zres, p.yres, p.xres)
    u = splitmix64_uniform(seed, 5 * p.cells).reshape((5,) + shape)
    blob = 2.0 * np.exp(-((x - 0.3) ** 2 + (y - 0.6) ** 2 + (z - 0.2) ** 2) / 0.02)
    return {"r": 1.0 + 0.2 * u[0], "p": 1.0 + 0.2 * u[1] + blob, "u": 0.1 * u[2], "v": 0.1 * u[3], "w": 0.1 * u[4]}
