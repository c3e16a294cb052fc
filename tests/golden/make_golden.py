"""Generate the golden fixtures by running the unmodified reference.

Five phases:
  build    (here, where the reference sources are):  compile one reference binary
           per case into oracle/_ref/<case>/ with oracle/ref_build.py;
  run      (on a B200):  for each case write the restart file, run
           ``penguin init.bin 0`` in the case folder and save the reference's
           output snapshot plus the initial state as <out>/<case>.npz;
  floor    (on a B200):  the reference's own sensitivity to rounding: each case
           is run again from its restart file with every interior density moved
           by one ulp (up or down, seeded), and the relative L1 distance of that
           output from the unperturbed one (density, pressure, momentum; dust
           density and momentum) goes to <out>/floors.json.  The unperturbed
           run is repeated too and must equal the committed fixture bit for bit;
  fmafloor (on a B200):  the reference's sensitivity to its own operation order:
           each 3D case is run again by a build of the same sources compiled
           with -fmad=false (no FMA contraction, built by the build phase into
           oracle/_ref/<case>_nofma/), and its distance from the committed
           fixture goes to floors.json as "fma_floor";
  collect  (here):  copy the .npz files of the golden cases (and floors.json)
           into tests/golden/.

    python tests/golden/make_golden.py build
    python tests/golden/make_golden.py run --out <outdir> [--timing]
    python tests/golden/make_golden.py floor --out <outdir> [--only <regex>]
    python tests/golden/make_golden.py fmafloor --out <outdir>
    python tests/golden/make_golden.py collect --src <outdir>
"""
from __future__ import annotations

import argparse
import dataclasses
import glob
import json
import os
import re
import shutil
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import cases as C  # noqa: E402
from oracle import ref_build  # noqa: E402
from penguin_b200 import snapshot  # noqa: E402
from penguin_b200.params import axes_np, make_grid_np  # noqa: E402


def _all(timing: bool):
    return C.cases() + C.dust_cases() + C.ave_cases() + C.cases3d() + (C.timing_cases() if timing else [])


def build(timing: bool, jobs: int) -> None:
    for c in _all(timing):
        hdr = ref_build.case_header(c)
        t = time.time()
        exe = ref_build.build_case(c["name"], hdr, jobs=jobs, tools=tuple(c.get("tools", ())))
        print(f"{c['name']}: {exe} ({time.time() - t:.0f} s)", flush=True)
    for c in C.cases3d():  # the same sources without FMA contraction (fmafloor phase)
        exe = ref_build.build_case(c["name"] + "_nofma", ref_build.case_header(c), jobs=jobs,
                                   nvcc_flags=("-fmad=false",))
        print(f"{c['name']}_nofma: {exe}", flush=True)


def _run_dust(c: dict, d: str, out: str, st: dict, tag: str = "") -> int:
    """Dust cases: the reference's dust reconstruction reads a flattening coefficient
    from shared memory it never writes (src/solver/recon/PPM.cu:68-77 reached from
    src/solver/dust/dust.cu:105-147), so its snapshots depend on what earlier kernels
    left there.  These fixtures are produced by the reference's own kernels driven
    step by step by oracle/ref_stages.cu with that memory zeroed before each dust
    stage ("scrub"); the final stage of the last step is stored."""
    p = c["params"]
    t = time.time()
    r = subprocess.run(["./stages", "init.bin", str(c["max_step"]), "stages.bin", "scrub"], cwd=d,
                       capture_output=True, text=True, timeout=900)
    wall = time.time() - t
    with open(os.path.join(out, c["name"] + tag + ".log"), "w") as f:
        f.write(r.stdout + "\n--- stderr ---\n" + r.stderr)
    print(f"{c['name']}{tag}: rc={r.returncode} wall={wall:.2f}s (stage driver, scrub)", flush=True)
    if r.returncode != 0 or "CUDA error" in r.stdout:
        return 1
    xarr, yarr = p.xres + 6, p.yres + 6
    n = xarr * yarr
    rec = 32 + 16 + n * 40 + n * 32
    raw = np.fromfile(os.path.join(d, "stages.bin"), dtype=np.uint8)
    last = raw[(raw.size // rec - 1) * rec:]
    t_stage, dt_stage = np.frombuffer(last[32:48].tobytes())
    cells = np.frombuffer(last[48:48 + n * 40].tobytes()).reshape(yarr, xarr, 5)[3:-3, 3:-3]
    dust = np.frombuffer(last[48 + n * 40:].tobytes()).reshape(yarr, xarr, 4)[3:-3, 3:-3]
    os.remove(os.path.join(d, "stages.bin"))
    keys = ["r", "p", "u", "v"]
    res = {k: np.ascontiguousarray(cells[..., m]) for m, k in ((0, "r"), (1, "p"), (2, "u"), (3, "v"))}
    res.update({"dust_" + k: np.ascontiguousarray(dust[..., m]) for m, k in enumerate(("r", "u", "v", "w"))})
    np.savez_compressed(
        os.path.join(out, c["name"] + tag + ".npz"),
        t0=c["t0"], t=t_stage + dt_stage, max_step=c["max_step"], end_time=c["end_time"],
        params=json.dumps(dataclasses.asdict(p)), source="ref_stages scrub",
        **{"init_" + k: np.asarray(st[k], dtype=np.float64) for k in keys},
        **{"out_" + k: v for k, v in res.items()},
    )
    return 0


def _run_3d(c: dict, d: str, out: str, st: dict, tag: str = "") -> int:
    """3D cases: restart file with the faces of every axis (load_grid skips them,
    src/output/output.cu:190-195) and the five fields; the output snapshot's fields
    are stored (the initial state is regenerated from the case's seed)."""
    p = c["params"]
    (xa, _), (ya, _), (za, _) = axes_np(p)
    init = os.path.join(d, "init.bin")
    snapshot.write_snapshot(init, c["t0"], xa[3:3 + p.xres + 1], ya[3:3 + p.yres + 1], st, 3,
                            za=za[3:3 + p.zres + 1])
    t = time.time()
    r = subprocess.run(["./penguin", "init.bin", "0"], cwd=d, capture_output=True, text=True, timeout=900)
    wall = time.time() - t
    outs = sorted(f for f in glob.glob(os.path.join(d, "binary_*_00001")) if "_ave_" not in os.path.basename(f))
    print(f"{c['name']}{tag}: rc={r.returncode} wall={wall:.2f}s out={outs}", flush=True)
    with open(os.path.join(out, c["name"] + tag + ".log"), "w") as f:
        f.write(r.stdout + "\n--- stderr ---\n" + r.stderr)
    if r.returncode != 0 or not outs:
        print(f"{c['name']}: files {sorted(os.listdir(d))}\n{r.stdout[-1500:]}", flush=True)
        return 1
    res = snapshot.read_snapshot(outs[0], p.xres, p.yres, 3, zres=p.zres)
    os.remove(outs[0])
    np.savez_compressed(
        os.path.join(out, c["name"] + tag + ".npz"),
        t0=c["t0"], t=res["t"], max_step=c["max_step"], end_time=c["end_time"],
        params=json.dumps(dataclasses.asdict(p)), seed=c.get("seed", C.SEED),
        **{"out_" + k: res[k] for k in ("r", "p", "u", "v", "w")},
    )
    return 0


def perturb_ulp(st: dict, seed: int = 99) -> dict:
    """Every interior density one ulp up or down (the sign drawn per cell)."""
    r = np.asarray(st["r"], dtype=np.float64)
    up = np.random.default_rng(seed).integers(0, 2, size=r.shape).astype(bool)
    return dict(st, r=np.where(up, np.nextafter(r, np.inf), np.nextafter(r, -np.inf)))


def run(out: str, timing: bool, only: str | None, perturb: bool = False, tag: str = "") -> int:
    os.makedirs(out, exist_ok=True)
    bad = 0
    for c in _all(timing):
        if only and not re.search(only, c["name"]):
            continue
        p = c["params"]
        d = os.path.join(ref_build.REF_OUT, c["name"])
        exe = os.path.join(d, "penguin")
        if not os.path.exists(exe):
            print(f"{c['name']}: missing {exe}", flush=True)
            bad += 1
            continue
        for f in glob.glob(os.path.join(d, "binary_*")):
            os.remove(f)
        st = C.initial_state(c)
        st_run = perturb_ulp(st) if perturb else st
        if p.ndim == 3:
            bad += _run_3d(c, d, out, st_run, tag)
            continue
        xa, _ = make_grid_np(p.xmin, p.xmax, p.xres, 3, p.geomx, p.gridx)
        ya, _ = make_grid_np(p.ymin, p.ymax, p.yres, 3 if p.ndim > 1 else 0, p.geomy, p.gridy)
        init = os.path.join(d, "init.bin")
        snapshot.write_snapshot(init, c["t0"], xa[3:3 + p.xres + 1], ya[3:3 + p.yres + 1] if p.ndim > 1 else None,
                                st_run, p.ndim)
        if c.get("dust"):
            bad += _run_dust(c, d, out, st, tag)
            continue
        t = time.time()
        r = subprocess.run(["./penguin", "init.bin", "0"], cwd=d, capture_output=True, text=True, timeout=900)
        wall = time.time() - t
        outs = sorted(f for f in glob.glob(os.path.join(d, "binary_*_00001")) if "_ave_" not in os.path.basename(f))
        aves = sorted(glob.glob(os.path.join(d, "binary_*_ave_00001")))
        sps = re.findall(r"([0-9.eE+-]+) seconds per step", r.stdout)
        print(f"{c['name']}{tag}: rc={r.returncode} wall={wall:.2f}s s/step={sps[-1] if sps else '?'} out={outs}",
              flush=True)
        with open(os.path.join(out, c["name"] + tag + ".log"), "w") as f:
            f.write(r.stdout + "\n--- stderr ---\n" + r.stderr)
        if r.returncode != 0 or not outs:
            print(f"{c['name']}: files {sorted(os.listdir(d))}\n{r.stdout[-1500:]}", flush=True)
            bad += 1
            continue
        if c["name"].startswith("ref_"):
            os.remove(outs[0])
            with open(os.path.join(out, c["name"] + ".json"), "w") as f:
                json.dump({"seconds_per_step": float(sps[-1]) if sps else None, "wall_s": wall,
                           "steps": c["max_step"], "cells": p.xres * p.yres}, f)
            continue
        dust = bool(c.get("dust"))
        res = snapshot.read_snapshot(outs[0], p.xres, p.yres, p.ndim, dust=dust)
        keys = ["r", "p", "u"] + (["v"] if p.ndim > 1 else [])
        dkeys = ["dust_r", "dust_u", "dust_v", "dust_w"] if dust else []
        extra = {}
        if c.get("ave_interval"):  # the time average the reference wrote beside the state
            if not aves:
                bad += 1
                continue
            ave = snapshot.read_snapshot(aves[0], p.xres, p.yres, p.ndim)
            extra = {"ave_" + k: ave[k] for k in keys}
            extra["ave_interval"] = c["ave_interval"]
        np.savez_compressed(
            os.path.join(out, c["name"] + tag + ".npz"),
            t0=c["t0"], t=res["t"], max_step=c["max_step"], end_time=c["end_time"],
            params=json.dumps(dataclasses.asdict(p)),
            **{"init_" + k: np.asarray(st[k], dtype=np.float64) for k in keys},
            **{"out_" + k: res[k] for k in keys + dkeys},
            **extra,
        )
    return bad


def _rel_l1(a, b):
    den = float(np.abs(b).sum())
    return float(np.abs(a - b).sum()) / den if den > 0 else float(np.abs(a - b).sum())


def _distances(a: dict, b: dict, ndim: int, dust: bool) -> dict:
    """Relative L1 of density, pressure and the momentum vector of a against b
    (and of the dust density and momentum)."""
    def mom(z, pre=""):
        r = z[f"out_{pre}r"]
        comps = "uvw"[:max(ndim, 2) if pre == "" else 2]
        return [r * z[f"out_{pre}{k}"] if f"out_{pre}{k}" in z else 0 * r for k in comps]

    def l1(ma, mb):
        return float(sum(np.abs(x - y).sum() for x, y in zip(ma, mb)) / sum(np.abs(y).sum() for y in mb))

    out = {"r": _rel_l1(a["out_r"], b["out_r"]), "p": _rel_l1(a["out_p"], b["out_p"])}
    out["momentum"] = l1(mom(a), mom(b))
    if dust:
        out["dust_r"] = _rel_l1(a["out_dust_r"], b["out_dust_r"])
        out["dust_momentum"] = l1(mom(a, "dust_"), mom(b, "dust_"))
    return out


def floor(out: str, only: str | None) -> int:
    """The reference against itself: unperturbed (must equal the committed
    fixture) and with one-ulp density perturbations (the sensitivity floor)."""
    bad = run(out, False, only, perturb=False, tag=".rerun")
    bad += run(out, False, only, perturb=True, tag=".ulp")
    res = {}
    fl_path = os.path.join(out, "floors.json")
    if only and os.path.exists(os.path.join(HERE, "floors.json")):
        with open(os.path.join(HERE, "floors.json")) as f:
            res = json.load(f)  # a partial run updates the committed table
    for c in C.cases() + C.dust_cases() + C.cases3d():
        if only and not re.search(only, c["name"]):
            continue
        fx = os.path.join(HERE, c["name"] + ".npz")
        fr, fu = (os.path.join(out, c["name"] + t + ".npz") for t in (".rerun", ".ulp"))
        if not all(os.path.exists(f) for f in (fx, fr, fu)):
            print(f"{c['name']}: missing output", flush=True)
            bad += 1
            continue
        zx, zr, zu = np.load(fx), np.load(fr), np.load(fu)
        p, dust = c["params"], bool(c.get("dust"))
        rerun = _distances(zr, zx, p.ndim, dust)
        res[c["name"]] = {"steps": c["max_step"], "floor": _distances(zu, zr, p.ndim, dust),
                          "rerun_vs_fixture": rerun, "deterministic": all(v == 0.0 for v in rerun.values())}
        print(c["name"], json.dumps(res[c["name"]]), flush=True)
    with open(fl_path, "w") as f:
        json.dump(res, f, indent=1, sort_keys=True)
    return bad


def fmafloor(out: str) -> int:
    """Each 3D case by the -fmad=false build of the reference against the fixture."""
    os.makedirs(out, exist_ok=True)
    with open(os.path.join(HERE, "floors.json")) as f:
        res = json.load(f)
    bad = 0
    for c in C.cases3d():
        name = c["name"]
        d = os.path.join(ref_build.REF_OUT, name + "_nofma")
        fx = os.path.join(HERE, name + ".npz")
        if not os.path.exists(os.path.join(d, "penguin")) or not os.path.exists(fx):
            print(f"{name}: missing build or fixture", flush=True)
            bad += 1
            continue
        for f in glob.glob(os.path.join(d, "binary_*")):
            os.remove(f)
        bad += _run_3d(c, d, out, C.initial_state(c), ".nofma")
        z = os.path.join(out, name + ".nofma.npz")
        if not os.path.exists(z):
            continue
        dist = _distances(np.load(z), np.load(fx), 3, False)
        res.setdefault(name, {})["fma_floor"] = dist
        print(name, "fma_floor", json.dumps(dist), flush=True)
    with open(os.path.join(out, "floors.json"), "w") as f:
        json.dump(res, f, indent=1, sort_keys=True)
    return bad


def collect(src: str) -> None:
    for c in C.cases() + C.dust_cases() + C.ave_cases() + C.cases3d():
        f = os.path.join(src, c["name"] + ".npz")
        if os.path.exists(f):
            shutil.copy(f, os.path.join(HERE, c["name"] + ".npz"))
            print("collected", c["name"])
        else:
            print("missing", f)
    f = os.path.join(src, "floors.json")
    if os.path.exists(f):
        shutil.copy(f, os.path.join(HERE, "floors.json"))
        print("collected floors.json")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("phase", choices=["build", "run", "floor", "fmafloor", "collect"])
    ap.add_argument("--out", default="golden_out")
    ap.add_argument("--src", default="golden_out")
    ap.add_argument("--timing", action="store_true")
    ap.add_argument("--only", default=None)
    ap.add_argument("--jobs", type=int, default=6)
    a = ap.parse_args()
    if a.phase == "build":
        build(a.timing, a.jobs)
    elif a.phase == "run":
        sys.exit(1 if run(a.out, a.timing, a.only) else 0)
    elif a.phase == "floor":
        sys.exit(1 if floor(a.out, a.only) else 0)
    elif a.phase == "fmafloor":
        sys.exit(1 if fmafloor(a.out) else 0)
    else:
        collect(a.src)


if __name__ == "__main__":
    main()
