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
