"""Snapshot files in the reference's checkpoint format.

Layout (src/output/output.cu:125-180, parsed by read/read_penguin.py:136-202):
``[t][xa: xres+1][ya: yres+1 if ndim>1][rho][p][u][v if ndim>1]``, all float64,
each field xres*yres values with x fastest.  File names follow
``binary_<label>_<5-digit frame>`` (output.cu:14-92, util.cu:25-36).
The same file restarts a run (load_grid reads t and the fields, skipping faces).
"""
from __future__ import annotations

import numpy as np


def write_snapshot(path: str, t: float, xa: np.ndarray, ya: np.ndarray | None, fields: dict, ndim: int) -> None:
    parts = [np.array([t], dtype=np.float64), np.asarray(xa, dtype=np.float64)]
    if ndim > 1:
        parts.append(np.asarray(ya, dtype=np.float64))
    names = ["r", "p", "u"] + (["v"] if ndim > 1 else [])
    for k in names:
        parts.append(np.ascontiguousarray(fields[k], dtype=np.float64).ravel())
    np.concatenate(parts).tofile(path)


def read_snapshot(path: str, xres: int, yres: int, ndim: int, dust: bool = False) -> dict:
    dat = np.fromfile(path, dtype=np.float64)
    o = 0
    t = float(dat[o]); o += 1
    xa = dat[o:o + xres + 1]; o += xres + 1
    ya = None
    if ndim > 1:
        ya = dat[o:o + yres + 1]; o += yres + 1
    n = xres * yres
    out = {"t": t, "xa": xa, "ya": ya}
    for k in ["r", "p", "u"] + (["v"] if ndim > 1 else []):
        out[k] = dat[o:o + n].reshape(yres, xres)
        o += n
    if dust:  # dust_flag builds append the dust r, u (and v, w in 2D), src/output/output.cu:159-176
        for k in ["dust_r", "dust_u"] + (["dust_v", "dust_w"] if ndim > 1 else []):
            out[k] = dat[o:o + n].reshape(yres, xres)
            o += n
    if o != dat.size:
        raise ValueError(f"{path}: {dat.size} values, expected {o}")
    return out


def frame_num(n: int) -> str:
    return f"{n:05d}"
