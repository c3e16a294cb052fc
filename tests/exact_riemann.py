"""Exact solution of the 1D Riemann problem for an ideal gas.

Restated from the published method of E. F. Toro, *Riemann Solvers and
Numerical Methods for Fluid Dynamics* (3rd ed., 2009), chapter 4: Newton
iteration on the star-region pressure function f(p) = f_L(p) + f_R(p) + du,
then sampling of the self-similar wave pattern at x/t.  The reference has no
exact solver; this one checks the Sod tube end to end.
"""
from __future__ import annotations

import math

import numpy as np


def _f_and_df(p, rk, pk, ck, g):
    if p > pk:  # shock
        A = 2.0 / ((g + 1.0) * rk)
        B = (g - 1.0) / (g + 1.0) * pk
        q = math.sqrt(A / (p + B))
        return (p - pk) * q, q * (1.0 - 0.5 * (p - pk) / (B + p))
    # rarefaction
    pr = p / pk
    f = 2.0 * ck / (g - 1.0) * (pr ** ((g - 1.0) / (2.0 * g)) - 1.0)
    df = 1.0 / (rk * ck) * pr ** (-(g + 1.0) / (2.0 * g))
    return f, df


def star_state(left, right, g=1.4):
    rl, ul, pl = left
    rr, ur, pr = right
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    p = max(1e-8, 0.5 * (pl + pr) - 0.125 * (ur - ul) * (rl + rr) * (cl + cr))
    for _ in range(100):
        fl, dfl = _f_and_df(p, rl, pl, cl, g)
        fr, dfr = _f_and_df(p, rr, pr, cr, g)
        dp = (fl + fr + (ur - ul)) / (dfl + dfr)
        p_new = max(1e-12, p - dp)
        if abs(p_new - p) / (0.5 * (p_new + p)) < 1e-14:
            p = p_new
            break
        p = p_new
    fl, _ = _f_and_df(p, rl, pl, cl, g)
    fr, _ = _f_and_df(p, rr, pr, cr, g)
    u = 0.5 * (ul + ur) + 0.5 * (fr - fl)
    return p, u


def sample(left, right, xi: np.ndarray, g=1.4):
    """(rho, u, p) at similarity coordinates xi = (x - x0)/t."""
    rl, ul, pl = left
    rr, ur, pr = right
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    ps, us = star_state(left, right, g)
    out = np.zeros((3, xi.size))
    gm = (g - 1.0) / (g + 1.0)
    for n, s in enumerate(xi):
        if s <= us:  # left of contact
            if ps > pl:  # left shock
                rsl = rl * ((ps / pl + gm) / (gm * ps / pl + 1.0))
                sl = ul - cl * math.sqrt((g + 1.0) / (2.0 * g) * ps / pl + (g - 1.0) / (2.0 * g))
                out[:, n] = (rl, ul, pl) if s <= sl else (rsl, us, ps)
            else:  # left rarefaction
                rsl = rl * (ps / pl) ** (1.0 / g)
                csl = cl * (ps / pl) ** ((g - 1.0) / (2.0 * g))
                sh, st = ul - cl, us - csl
                if s <= sh:
                    out[:, n] = (rl, ul, pl)
                elif s >= st:
                    out[:, n] = (rsl, us, ps)
                else:
                    c = 2.0 / (g + 1.0) * (cl + 0.5 * (g - 1.0) * (ul - s))
                    u = 2.0 / (g + 1.0) * (cl + 0.5 * (g - 1.0) * ul + s)
                    r = rl * (c / cl) ** (2.0 / (g - 1.0))
                    out[:, n] = (r, u, pl * (c / cl) ** (2.0 * g / (g - 1.0)))
        else:  # right of contact
            if ps > pr:  # right shock
                rsr = rr * ((ps / pr + gm) / (gm * ps / pr + 1.0))
                sr = ur + cr * math.sqrt((g + 1.0) / (2.0 * g) * ps / pr + (g - 1.0) / (2.0 * g))
                out[:, n] = (rr, ur, pr) if s >= sr else (rsr, us, ps)
            else:  # right rarefaction
                rsr = rr * (ps / pr) ** (1.0 / g)
                csr = cr * (ps / pr) ** ((g - 1.0) / (2.0 * g))
                sh, st = ur + cr, us + csr
                if s >= sh:
                    out[:, n] = (rr, ur, pr)
                elif s <= st:
                    out[:, n] = (rsr, us, ps)
                else:
                    c = 2.0 / (g + 1.0) * (cr - 0.5 * (g - 1.0) * (ur - s))
                    u = 2.0 / (g + 1.0) * (-cr + 0.5 * (g - 1.0) * ur + s)
                    r = rr * (c / cr) ** (2.0 / (g - 1.0))
                    out[:, n] = (r, u, pr * (c / cr) ** (2.0 * g / (g - 1.0)))
    return out
