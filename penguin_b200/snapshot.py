"""Snapshot files in the reference's checkpoint format.

Layout (src/output/output.cu:125-180, parsed by read/read_penguin.py:136-202):
``[t][xa: xres+1][ya: yres+1 if ndim>1][za: zres+1 if ndim>2][rho][p][u]
[v if ndim>1][w if ndim>2]``, all float64, each field xres*yres(*zres) values
with x fastest, then y, then z.  File names follow
``binary_<label>_<5-digit frame>`` (output.cu:14-92, util.cu:25-36).
The same file restarts a run (load_grid reads t and the fields, skipping faces).
"""
from __future__ import annotations

import numpy as np


def write_snapshot(path: str, t: float, xa: np.ndarray, ya: np.ndarray | None, fields: dict, ndim: int,
                   za: np.ndarray | None = None) -> None:
    parts = [np.array([t], dtype=np.float64), np.asarray(xa, dtype=np.float64)]
    if ndim > 1:
        parts.append(np.asarray(ya, dtype=np.float64))
    if ndim > 2:
        parts.append(np.asarray(za, dtype=np.float64))
    names = ["r", "p", "u"] + (["v"] if ndim > 1 else []) + (["w"] if ndim > 2 else [])
    for k in names:
        parts.append(np.ascontiguousarray(fields[k], dtype=np.float64).ravel())
    np.concatenate(parts).tofile(path)


def read_snapshot(path: str, xres: int, yres: int, ndim: int, dust: bool = False, zres: int = 1) -> dict:
    """Fields come back as (yres, xres) arrays, (zres, yres, xres) when ndim is 3."""
    dat = np.fromfile(path, dtype=np.float64)
    o = 0
    t = float(dat[o]); o += 1
    xa = dat[o:o + xres + 1]; o += xres + 1
    ya = za = None
    if ndim > 1:
        ya = dat[o:o + yres + 1]; o += yres + 1
    if ndim > 2:
        za = dat[o:o + zres + 1]; o += zres + 1
    shape = (zres, yres, xres) if ndim > 2 else (yres, xres)
    n = xres * yres * (zres if ndim > 2 else 1)
    out = {"t": t, "xa": xa, "ya": ya, "za": za}
    for k in ["r", "p", "u"] + (["v"] if ndim > 1 else []) + (["w"] if ndim > 2 else []):
        out[k] = dat[o:o + n].reshape(shape)
        o += n
    if dust:  # dust_flag builds append the dust r, u (and v, w in 2D), src/output/output.cu:159-176
        for k in ["dust_r", "dust_u"] + (["dust_v", "dust_w"] if ndim > 1 else []):
            out[k] = dat[o:o + n].reshape(shape)
            o += n
    if o != dat.size:
        raise ValueError(f"{path}: {dat.size} values, expected {o}")
    return out


def frame_num(n: int) -> str:
    return f"{n:05d}"


# include/parameters.h:31,34
EARTH_MASS = 0.000003
JUPITER_MASS = 0.0009543


def _i(x: float) -> str:
    """int_to_string of a double argument (src/util/util.cu:18-23): truncation to int."""
    return str(int(x))


def label(p) -> str:
    """create_label (src/output/output.cu:14-92) for the configurations this library runs
    (recon_flag 6, alpha viscosity visc_flag 1, no cooling)."""
    import math

    if p.ndim == 1:
        s = _i(p.xres)
    elif p.ndim == 2:
        s = f"{_i(p.xres)}x{_i(p.yres)}"
    else:
        s = f"{_i(p.xres)}x{_i(p.yres)}x{_i(p.zres)}"
    s += "_h" + _i(1000.0 * p.sc_h)
    if p.n_planet > 0:
        if p.planet_mass >= JUPITER_MASS:
            s += f"_{_i(p.n_planet)}p{_i(p.planet_mass / JUPITER_MASS)}J"
        else:
            s += f"_{_i(p.n_planet)}p{_i(p.planet_mass / EARTH_MASS)}E"
        s += "_e" + _i(p.planet_ecc * 1000.0)
    if p.visc_flag == 1:
        s += "_a" + _i(math.log10(p.ss_alpha) * 10.0)
    if p.ndim > 1 and p.OrbAdv_flag:
        s += "_OA"
    if p.dust_flag:
        s += "_St" + _i(math.log10(p.Stokes) * 10.0)
    s += "_PPM4"
    return s


def file_name(p, frame: int, average: bool = False) -> str:
    """binary_<label>_<frame> (main.cu:403), binary_<label>_ave_<frame> for averages (main.cu:414)."""
    return "binary_" + label(p) + ("_ave_" if average else "_") + frame_num(frame)
