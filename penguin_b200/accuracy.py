"""Accuracy of the FP32-mixed form against the FP64 form on one planet-disk.

    python -m penguin_b200.accuracy [--nr 1024 --nphi 3072 --orbits 100 --every 10]

Both forms start from the same seeded disk at t = 0 and are stopped at the
same times (every ``--every`` orbits, t = 2 pi k); each takes its own CFL
steps.  Reported per sample, one JSON line each:

  l1_sigma    sum |Sigma_32 - Sigma_64| / sum Sigma_64 over all cells
  l1_profile  the same for the azimuthally averaged profiles <Sigma>_phi(r)
  gap_depth   min over 0.8 <= r <= 1.2 of <Sigma>_phi(r) / Sigma_0(r), both forms
  torque      torque of the planet on the disk / (q^2 / h^2), both forms (the
              quantity main.cu writes, src/output/output.cu:336-412)
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import initial as I
from . import params as P
from .disk import Disk
from .ensemble import Ensemble


def gap_depth(sigma: np.ndarray, p) -> float:
    x = I.cell_centres(p)
    s0, _, _ = I._disk_profiles(p, x)
    prof = sigma.mean(axis=0) / s0
    sel = (x >= 0.8) & (x <= 1.2)
    return float(prof[sel].min())


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nr", type=int, default=1024)
    ap.add_argument("--nphi", type=int, default=3072)
    ap.add_argument("--orbits", type=float, default=100.0)
    ap.add_argument("--every", type=float, default=10.0)
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--q", type=float, default=1.0e-3, help="planet mass ratio (0: no planet, laminar disk)")
    ap.add_argument("--perturb", type=float, default=0.0,
                    help="instead of the FP32 form, compare with a second FP64 run whose initial Sigma is "
                         "multiplied by 1 + perturb U(-1,1) (the sensitivity floor of the flow)")
    args = ap.parse_args(argv)

    p = P.planet_disk(args.nr, args.nphi, q=args.q)
    st = I.disk_state(p, seed=args.seed)
    norm = (p.planet_mass ** 2 / p.sc_h ** 2) if p.planet_mass > 0 else 1.0
    d = Disk(p)
    d.set_state(0.0, st)
    if args.perturb > 0.0:
        st2 = dict(st)
        st2["r"] = st["r"] * (1.0 + args.perturb * I.splitmix64_uniform(args.seed + 1, st["r"].size).reshape(st["r"].shape))
        st2["p"] = st2["r"] * (st["p"] / st["r"])
        e = Disk(p)
        e.set_state(0.0, st2)
        other = "fp64-perturbed"
    else:
        e = Ensemble([p])
        e.set_state(0, 0.0, st)
        other = "fp32"
    k = 0
    wall = {"fp64": 0.0, "fp32": 0.0}  # "fp32": the compared run
    while True:
        k += 1
        orb = min(k * args.every, args.orbits)
        t_end = 2.0 * math.pi * orb
        t0 = time.perf_counter()
        d.run(10 ** 9, t_end)
        d.sync()
        wall["fp64"] += time.perf_counter() - t0
        t0 = time.perf_counter()
        e.run(10 ** 9, t_end)
        e.sync()
        wall["fp32"] += time.perf_counter() - t0
        d.check()
        e.check()
        two = isinstance(e, Disk)
        a, b = d.get_state(), (e.get_state() if two else e.get_state(0))
        pa, pb = a["r"].mean(axis=0), b["r"].mean(axis=0)
        tq = [d.torque() / norm, (e.torque() if two else e.torque(0)) / norm] if p.planet_mass > 0 else [0.0, 0.0]
        line = {
            "orbits": orb,
            "against": other,
            "t": [d.clock()[0], e.clock()[0] if two else e.clock(0)[0]],
            "steps": [d.clock()[2], e.clock()[2] if two else e.clock(0)[2]],
            "l1_sigma": float(np.abs(b["r"] - a["r"]).sum() / np.abs(a["r"]).sum()),
            "l1_profile": float(np.abs(pb - pa).sum() / np.abs(pa).sum()),
            "gap_depth": [gap_depth(a["r"], p), gap_depth(b["r"], p)],
            "torque": tq,
            "wall_s": dict(wall),
            "disk": f"planet_disk({args.nr}, {args.nphi}, q={args.q}), seed {args.seed}",
        }
        print(json.dumps(line), flush=True)
        if orb >= args.orbits:
            break
    d.close()
    e.close()


if __name__ == "__main__":
    main()
