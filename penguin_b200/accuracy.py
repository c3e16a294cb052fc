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

    python -m penguin_b200.accuracy --floor-runs 2 [--orbits 100 --torque-window 10]

runs the FP64 form, the FP32-mixed form and ``--floor-runs`` further FP64 runs
whose initial Sigma is multiplied by 1 + 1e-12 U(-1,1) (each its own seed) side
by side, and ends with one summary line: for the FP32 form and for each
perturbed FP64 run, against the FP64 form at the last sample, the L1 of Sigma
and of the azimuthally averaged profile, the gap depth difference, and the
difference of the torque averaged over the last ``--torque-window`` orbits
(sampled every 0.1 orbit).  The perturbed runs measure how far the flow itself
carries a rounding-level difference (its sensitivity floor); the FP32 error is
at the floor when it is no larger than theirs.
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


def _perturbed(st: dict, seed: int, eps: float) -> dict:
    out = dict(st)
    out["r"] = st["r"] * (1.0 + eps * I.splitmix64_uniform(seed, st["r"].size).reshape(st["r"].shape))
    out["p"] = out["r"] * (st["p"] / st["r"])
    return out


def floor_study(args) -> None:
    """FP64, FP32-mixed and perturbed FP64 runs of one disk, side by side."""
    p = P.planet_disk(args.nr, args.nphi, q=args.q)
    st = I.disk_state(p, seed=args.seed)
    norm = (p.planet_mass ** 2 / p.sc_h ** 2) if p.planet_mass > 0 else 1.0
    runs = {"fp64": Disk(p), "fp32": Ensemble([p])}
    runs["fp64"].set_state(0.0, st)
    runs["fp32"].set_state(0, 0.0, st)
    for k in range(args.floor_runs):
        d = Disk(p)
        d.set_state(0.0, _perturbed(st, args.seed + 1 + k, 1.0e-12))
        runs[f"fp64_perturbed_{k + 1}"] = d

    def state(name):
        r = runs[name]
        return r.get_state() if isinstance(r, Disk) else r.get_state(0)

    def torque(name):
        r = runs[name]
        return (r.torque() if isinstance(r, Disk) else r.torque(0)) / norm

    def advance(t_end):
        for r in runs.values():
            r.run(10 ** 9, t_end)
        for r in runs.values():
            r.sync()
            r.check()

    t_win0 = args.orbits - args.torque_window
    samples = [k * args.every for k in range(1, int(round(args.orbits / args.every)) + 1)]
    tq_times = [t_win0 + 0.1 * k for k in range(1, int(round(args.torque_window / 0.1)) + 1)]
    times = sorted(set(samples) | set(tq_times))
    tq = {k: [] for k in runs}
    t0 = time.perf_counter()
    for orb in times:
        advance(2.0 * math.pi * orb)
        if orb > t_win0 + 1e-9 and p.planet_mass > 0:
            for k in runs:
                tq[k].append(torque(k))
        if any(abs(orb - s_) < 1e-9 for s_ in samples):
            a = state("fp64")
            line = {"orbits": orb, "wall_s": time.perf_counter() - t0}
            for k in runs:
                if k == "fp64":
                    continue
                b = state(k)
                line[k] = {"l1_sigma": float(np.abs(b["r"] - a["r"]).sum() / np.abs(a["r"]).sum()),
                           "l1_profile": float(np.abs(b["r"].mean(0) - a["r"].mean(0)).sum()
                                               / np.abs(a["r"].mean(0)).sum())}
            print(json.dumps(line), flush=True)
    a = state("fp64")
    gd64 = gap_depth(a["r"], p)
    tq64 = float(np.mean(tq["fp64"])) if tq["fp64"] else 0.0
    summary = {"summary": True, "disk": f"planet_disk({args.nr}, {args.nphi}, q={args.q}), seed {args.seed}",
               "orbits": args.orbits, "torque_window_orbits": args.torque_window,
               "fp64": {"gap_depth": gd64, "torque_avg": tq64, "steps": runs["fp64"].clock()[2]}}
    for k in runs:
        if k == "fp64":
            continue
        b = state(k)
        gd = gap_depth(b["r"], p)
        tqa = float(np.mean(tq[k])) if tq[k] else 0.0
        summary[k] = {
            "l1_sigma": float(np.abs(b["r"] - a["r"]).sum() / np.abs(a["r"]).sum()),
            "l1_profile": float(np.abs(b["r"].mean(0) - a["r"].mean(0)).sum() / np.abs(a["r"].mean(0)).sum()),
            "gap_depth": gd, "gap_depth_diff": abs(gd - gd64),
            "torque_avg": tqa, "torque_avg_rel_diff": abs(tqa - tq64) / abs(tq64) if tq64 else 0.0,
        }
    print(json.dumps(summary), flush=True)
    for r in runs.values():
        r.close()


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nr", type=int, default=1024)
    ap.add_argument("--nphi", type=int, default=3072)
    ap.add_argument("--orbits", type=float, default=100.0)
    ap.add_argument("--every", type=float, default=10.0)
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--q", type=float, default=1.0e-3, help="planet mass ratio (0: no planet, laminar disk)")
    ap.add_argument("--floor-runs", type=int, default=0,
                    help="run the FP64 form, the FP32-mixed form and this many 1e-12-perturbed FP64 runs side "
                         "by side and summarise (see the module docstring)")
    ap.add_argument("--torque-window", type=float, default=10.0)
    ap.add_argument("--perturb", type=float, default=0.0,
                    help="instead of the FP32 form, compare with a second FP64 run whose initial Sigma is "
                         "multiplied by 1 + perturb U(-1,1) (the sensitivity floor of the flow)")
    args = ap.parse_args(argv)
    if args.floor_runs > 0:
        floor_study(args)
        return

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
