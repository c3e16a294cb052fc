#!/usr/bin/env python
"""Benchmark: zone-updates/s of the PEnGUIn Godunov timestep on B200.

Workload: the 2D polar planet-disk (Nr=1024 log-spaced on r in [0.4, 2.5],
Nphi=3072, locally isothermal h/r=0.05, Sigma ~ 1/r with seeded 1e-4 noise,
v_r = 0, alpha=1e-3, planet q=1e-3 at r=1 with 0.6 H smoothing and a 10-orbit
mass ramp, damping inside r=0.5 and outside r=2.2, orbital advection), FP64,
starting at t=0.  A step is main.cu's loop body: dt (CFL, 1.1x growth cap) and
one Godunov step (src/solver/solve.cu:279).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

N>1 runs under torchrun as N independent replicas (a single disk does not
shard: no domain decomposition), one process per GPU; the time is the max over
ranks and ``value`` counts all ranks' zone-updates.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "zone-updates/s on 2D planet-disk: FP32/batched/adjoint vs plain FP64; %HBM peak"
UNIT = "zone-updates/s"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
# algorithmic bytes per interior cell and launch: every pass keeps the drop-in
# AoS Cell (5 x FP64) and reads and writes it once; kick1 also writes the
# 2-component stress and kick2 reads it back.
ALGO_BYTES = {"time": 0, "kick1": 96, "sweep_x": 80, "sweep_y": 80, "advect": 80, "kick2": 96}
# FP32-mixed form: three FP32 residual planes (Sigma, v_r, v_phi) read and written
# once per pass, plus the 2-component FP32 stress written by kick1 and read by kick2
ALGO_BYTES_F32 = {"time": 0, "kick1": 32, "sweep_x": 24, "sweep_y": 24, "advect": 24, "kick2": 32}
ENSEMBLE_STEPS = 500
E2E_MIN_STEPS = 200


def workload(nr=1024, nphi=3072):
    from penguin_b200 import params as P

    return P.planet_disk(nr, nphi)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            j = json.load(f)
        return {"hbm_gbs": float(j["hbm_gbs"]), "bf16_tflops": float(j["bf16_tflops"]), "source": "measured"}
    except Exception:
        return dict(PEAKS_FALLBACK, source="fallback")


class Clocks:
    """SM clocks and clock-event reasons while the timed steps run.

    The profiling recipe's nvidia-smi clocks line samples every 200 ms and
    needs about as long to start, which is longer than a 20-step region of the
    headline workload (about 20 ms), so the samples are read through NVML
    instead: `wait(event)` polls the device's clocks from the host until the
    region's closing CUDA event has completed, i.e. only while the queued
    steps are running.  Without NVML (no pynvml) it falls back to nvidia-smi
    over the region."""

    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
    SMI = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
           "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
           "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []  # (sm MHz, max sm MHz, set of active reason names)
        self.nv = None
        self.h = None
        self.proc = None
        self.path = None

    def _handle(self):
        import pynvml as nv
        import torch

        nv.nvmlInit()
        self.nv = nv
        pr = torch.cuda.get_device_properties(self.gpu)
        bus = getattr(pr, "pci_bus_id", None)
        if bus is not None:
            bid = f"{getattr(pr, 'pci_domain_id', 0):08X}:{bus:02X}:{getattr(pr, 'pci_device_id', 0):02X}.0"
            try:
                return nv.nvmlDeviceGetHandleByPciBusId(bid)
            except Exception:
                pass
        return nv.nvmlDeviceGetHandleByIndex(self.gpu)

    def __enter__(self):
        try:
            self.h = self._handle()
            nv = self.nv
            self.bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                         "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                         "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                         "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM))
            return self
        except Exception:
            self.h = None
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.SMI}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def sample(self):
        if self.h is None:
            return
        nv = self.nv
        try:
            mhz = float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
            r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        except Exception:
            return
        self.rows.append((mhz, self.max_mhz, {n for n, b in self.bits.items() if r & b}))

    def wait(self, event):
        """Sample until `event` (recorded after the timed steps) has completed."""
        while not event.query():
            self.sample()
            time.sleep(0.0005)
        event.synchronize()

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.nv is not None:
            try:
                self.nv.nvmlShutdown()
            except Exception:
                pass

    def _smi_rows(self):
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9 and f[1].replace(".", "").isdigit():
                    act = {n for k, n in enumerate(self.NAMES) if f[5 + k].lower().startswith("active")}
                    self.rows.append((float(f[1]), float(f[2]), act))
        except Exception:
            pass
        finally:
            if os.path.exists(self.path):
                os.remove(self.path)

    def summary(self):
        if self.path:
            self._smi_rows()
        rows = self.rows
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [r[0] for r in rows]
        reasons = [n for n in self.NAMES if any(n in r[2] for r in rows)]
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": rows[0][1], "reasons": reasons,
                "samples": len(rows), "source": "nvml" if self.h is not None else "nvidia-smi"}


def cpu_baseline(p, state, t0, budget_s=15.0, keep=False):
    """The oracle (CPU restatement of the reference step, OpenMP over all host
    cores) on the same workload, for a bounded number of steps.  keep=True also
    returns the oracle, advanced by 1 + the timed steps, for a parity check."""
    from oracle.oracle import Oracle

    o = Oracle(p, state, t0)
    t = time.perf_counter()
    o.run(1)
    one = time.perf_counter() - t
    n = max(1, min(200, int(budget_s / max(one, 1e-3))))
    t = time.perf_counter()
    o.run(n)
    el = time.perf_counter() - t
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    cb = {"value": p.cells * n / el, "unit": UNIT, "cores": cores, "kind": "port",
          "sample": f"{n} steps of the full {p.xres}x{p.yres} workload after 1 warm-up step ({el:.1f} s)"}
    if keep:
        return cb, o, 1 + n
    o.close()
    return cb


def config_of(p, world):
    """The workload description both arms print."""
    return {"workload": f"planet-disk {p.xres}x{p.yres} FP64 (plain form), seeded 1e-4 Sigma noise, t0=0",
            "cells_per_gpu": p.cells, "state_bytes": 2 * 40 * (p.xres + 6) * (p.yres + 6),
            "l2": "inputs larger than L2 (two 127 MB AoS state buffers)",
            "parallelism": f"replicas x{world}" if world > 1 else "single device"}


REFERENCE_BUDGET_S = 150.0


def run_reference(args, rank, world):
    """Reference arm: the reference has no CPU implementation of the step (its
    only path is its CUDA build), so the CPU restatement (oracle/) stands in,
    on all host cores: W untimed warm-up steps, then K timed steps of the same
    workload (fewer only when K steps would exceed REFERENCE_BUDGET_S, and then
    the line says how many ran)."""
    if rank != 0:
        return
    from oracle.oracle import Oracle
    from penguin_b200 import initial as I

    p = workload()
    st = I.disk_state(p, seed=1234)
    o = Oracle(p, st, 0.0)
    t = time.perf_counter()
    o.run(1)
    one = time.perf_counter() - t
    W = max(1, min(args.warmup, int(0.2 * REFERENCE_BUDGET_S / max(one, 1e-3))))
    if W > 1:
        o.run(W - 1)
    K = max(1, min(args.steps, int(REFERENCE_BUDGET_S / max(one, 1e-3))))
    t = time.perf_counter()
    o.run(K)
    el = time.perf_counter() - t
    o.close()
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    value = p.cells * K / el
    cb = {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
          "sample": f"{K} timed steps of the full {p.xres}x{p.yres} workload after {W} warm-up steps ({el:.1f} s)"}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": K,
        "warmup": W, "ms_per_step": 1000.0 * el / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_of(p, args.gpus),
        "impl": "reference",
        "cpu_baseline": cb,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if K != args.steps or W != args.warmup:
        line["steps_requested"], line["warmup_requested"] = args.steps, args.warmup
    print(json.dumps(line), flush=True)


def timed(stream, fn):
    """Device time (ms) of fn() on `stream`, bracketed by synchronisation."""
    import torch

    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def roofline_of(prof, cells, algo, pk):
    stage = max((k for k in prof if algo.get(k)), key=lambda k: prof[k])
    achieved = algo[stage] * cells / (prof[stage] / 1000.0) / 1e9
    return {"bound": "hbm", "kernel": stage, "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / pk["hbm_gbs"], "peak_source": pk["source"], "algorithmic_bytes_per_cell": algo[stage]}


def measure_fp32(p, state, K, W, local, stream, pk):
    """The FP32-mixed form (an ensemble of one) on the same disk and step count."""
    from penguin_b200.ensemble import Ensemble

    e = Ensemble([p], device=local, stream=stream.cuda_stream)
    e.set_state(0, 0.0, state)
    e.run(W)
    e.sync()
    e.check()
    ms = timed(stream, lambda: e.run(K))
    e.check()
    prof = e.profile(max(5, min(50, K // 10)))
    out = {"value": p.cells * K / (ms / 1000.0), "ms_per_step": ms / K, "steps": K,
           "dtype": "f32 (FP64 dt, orbital shift, totals)", "stage_ms": prof,
           "roofline": roofline_of(prof, p.cells, ALGO_BYTES_F32, pk), "gpu_launches": e.kernels_per_step * K}
    e.close()
    return out


def measure_ensemble(job, local, stream, steps):
    """48 seeded disks of uneven size: one FP32-mixed ensemble (one persistent
    launch per pass, graph-captured step) against the same disks run one after
    another by the plain FP64 form, `steps` steps each with their own dt.  With
    several ranks each rank runs its share of whole disks (Replicas.share) as
    one ensemble, both arms are timed as the max over ranks, and rank 0 gathers
    every disk's final mass."""
    from penguin_b200 import initial as I
    from penguin_b200 import params as P
    from penguin_b200.disk import Disk
    from penguin_b200.ensemble import Ensemble

    ps_all = P.disk_ensemble()
    mine = job.share([p.cells for p in ps_all])
    ps = [ps_all[k] for k in mine]
    sts = [I.disk_state(ps_all[k], seed=100 + k) for k in mine]
    cells_all = sum(p.cells for p in ps_all)
    e = Ensemble(ps, device=local, stream=stream.cuda_stream)
    for k, st in enumerate(sts):
        e.set_state(k, 0.0, st)
    e.run(3)
    e.sync()
    tuning = e.autotune()
    e.run(1)
    e.sync()
    job.barrier(e.sync)
    ms_e = job.max_over_ranks(timed(stream, lambda: e.run(steps)))
    e.check()
    masses = {k: e.totals(n)[0] for n, k in enumerate(mine)}
    launches = e.kernels_per_step * steps
    e.close()
    # each disk timed on its own (device time of its graph launches), summed;
    # each autotuned like the ensemble
    ms_s = 0.0
    for p, st in zip(ps, sts):
        d = Disk(p, device=local, stream=stream.cuda_stream)
        d.set_state(0.0, st)
        d.run(3)
        d.sync()
        d.autotune()
        d.run(1)
        d.sync()
        ms_s += timed(stream, lambda: d.run(steps))
        d.check()
        d.close()
    ms_s = job.max_over_ranks(ms_s)
    gathered = job.gather(masses)
    v_e = cells_all * steps / (ms_e / 1000.0)
    v_s = cells_all * steps / (ms_s / 1000.0)
    out = {"disks": len(ps_all), "cells": cells_all, "steps": steps, "value": v_e, "ms_per_step": ms_e / steps,
           "gpu_launches": launches, "sequential_fp64": {"value": v_s, "ms_per_step": ms_s / steps},
           "over_sequential_fp64": v_e / v_s, "tuning": tuning,
           "note": "both arms autotuned (ensemble: pass variants and CTA caps; each FP64 disk: pencils per tile, CTA caps)",
           "config": "Nr in 32*[4,16], Nphi=3Nr, q log-U[1e-5,3e-3], alpha log-U[1e-4,1e-2], h/r U[0.03,0.08], seed 2024"}
    if job.world > 1:
        out["partition"] = {"ranks": job.world, "disks_per_rank": [len(g) for g in gathered] if gathered else None,
                            "scaling": "strong (the same 48 disks split by whole disks)"}
    return out


DUST_STEPS = 2000
# FP64 dust passes: the AoS dust cell (4 x FP64) read and written once by each
# dust sweep and the residual advection; the kicks also read and write it.
ALGO_BYTES_DUST = {"time": 0, "kick1": 96 + 64, "sweep_x": 80 + 64, "sweep_y": 80 + 64, "advect": 80 + 64,
                   "kick2": 96 + 64}


def measure_dust(local, stream, steps, pk):
    """Gas + one dust fluid, 768x2048, alpha 1e-4, q 3e-4, dust-to-gas 0.01,
    Stokes 0.01 and 0.1: the plain FP64 form for 3 warm-up + `steps` timed steps
    from t = 0, then the FP32-mixed form for the same number of steps from the
    same state (warm-up first, then reset; no end time, so no clip and no
    copy-through steps), and the dust profiles of the two compared at that step."""
    import numpy as np

    from penguin_b200 import initial as I
    from penguin_b200 import params as P
    from penguin_b200.disk import Disk
    from penguin_b200.ensemble import Ensemble

    out = {}
    for st in (0.01, 0.1):
        p = P.dust_disk(stokes=st)
        init = I.disk_state(p, seed=SEED_DUST)
        d = Disk(p, device=local, stream=stream.cuda_stream)
        d.set_state(0.0, init)
        m0 = float(d.get_dust()["r"].sum())
        d.run(3)
        d.sync()
        ms = timed(stream, lambda: d.run(steps))
        d.check()
        t64, _, n64 = d.clock()
        dust = d.get_dust()
        gas = d.get_state()
        prof = d.profile(20)  # advances the disk; everything compared is read before
        # the FP32-mixed form of the same disk, the same number of steps
        e = Ensemble([p], device=local, stream=stream.cuda_stream)
        e.set_state(0, 0.0, init)
        e.run(3)
        e.sync()
        e.set_state(0, 0.0, init)
        ms32 = timed(stream, lambda: e.run(n64))
        e.check()
        t32, _, n32 = e.clock(0)
        d32 = e.get_dust(0)
        prof64, prof32 = dust["r"].mean(axis=0), d32["r"].mean(axis=0)
        g64, g32 = gas["r"].mean(axis=0), e.get_state(0)["r"].mean(axis=0)
        fp32 = {"value": p.cells * n32 / (ms32 / 1000.0), "ms_per_step": ms32 / n32, "steps": n32,
                "dust_profile_l1_vs_fp64": float(np.abs(prof32 - prof64).sum() / np.abs(prof64).sum()),
                "dust_sigma_l1_vs_fp64": float(np.abs(d32["r"] - dust["r"]).sum() / np.abs(dust["r"]).sum()),
                "gas_profile_l1_vs_fp64": float(np.abs(g32 - g64).sum() / np.abs(g64).sum()),
                "t": t32, "t_fp64": t64, "gpu_launches": e.kernels_per_step * n32}
        e.close()
        out[f"stokes_{st}"] = {
            "value": p.cells * steps / (ms / 1000.0), "ms_per_step": ms / steps, "steps": steps,
            "steps_from_t0": n64,
            "stage_ms": prof, "roofline": roofline_of(prof, p.cells, ALGO_BYTES_DUST, pk),
            "gpu_launches": d.kernels_per_step * steps,
            "dust_sigma_sum_over_initial": float(dust["r"].sum()) / m0,
            "fp32_mixed": fp32,
        }
        out[f"stokes_{st}"]["fp32_mixed"]["over_fp64"] = fp32["value"] / out[f"stokes_{st}"]["value"]
        d.close()
    return {"workload": "768x2048 gas+dust planet-disk, FP64 form and FP32-mixed form, the same steps from t=0",
            "dtype": "f64 / f32 (FP64 dt, shift)", **out}


SEED_DUST = 1234
ADJOINT_STEPS = 256  # the finite-difference checks
ADJOINT_TIMING_STEPS = 1024  # the timed run: 16 checkpoint segments


def measure_adjoint(steps, local, stream, timing_steps=None):
    """Gradient of the azimuthally averaged Sigma(r) misfit after `steps` steps of the
    256x768 adjoint disk (q 5e-4, alpha 1e-3, h/r 0.05) with respect to the initial
    Sigma field and (q, alpha, h/r), against a target made by the same code at
    q 1e-3, alpha 3e-4 from the same seed; checkpoints every 64 steps.  Central
    finite differences (FP64) of the loss along a smooth Sigma0 direction and
    along each parameter check it.  Forward and adjoint are timed with CUDA
    events on a run of `timing_steps` steps (default `steps`): the backward
    overlaps the recompute of each segment with the transposition of the next,
    so only the first segment's recompute is exposed, and a longer run (config
    5 is about 10,900 steps, 170 segments) shows the steady cost."""
    import numpy as np
    import torch

    from penguin_b200 import initial as I
    from penguin_b200 import params as P
    from penguin_b200.adjoint import DiskAdjoint

    p = P.adjoint_disk()
    s0 = torch.tensor(I.disk_state(p, seed=SEED_DUST)["r"], device=f"cuda:{local}")
    tgt_model = DiskAdjoint(P.adjoint_disk(q=1.0e-3, alpha=3.0e-4), nsteps=steps, device=local,
                            stream=stream.cuda_stream)
    target = tgt_model.forward(s0).mean(0)
    tgt_model.close()
    m = DiskAdjoint(p, nsteps=steps, checkpoint_every=64, device=local, stream=stream.cuda_stream)

    def loss(sig):
        return float(((sig.mean(0) - target) ** 2).sum())

    out = None

    def fwd():
        nonlocal out
        out = m.forward(s0)

    ms_rec = timed(stream, fwd)  # the recording run: CFL dt read back every step
    g = (2.0 * (out.mean(0) - target) / p.yres)[None, :].expand(p.yres, p.xres).contiguous()
    res = {}

    def bwd():
        res["g"] = m.backward(g)

    bwd()
    gs0, gth = res["g"]
    # timing: medians of 3 after a warm-up, the forward replaying the recorded dt
    # schedule (what the backward recomputes per segment) and the backward
    tsteps = timing_steps or steps
    mt = m if tsteps == steps else DiskAdjoint(p, nsteps=tsteps, checkpoint_every=64, device=local,
                                               stream=stream.cuda_stream)
    if mt is not m:
        ms_rec = timed(stream, lambda: mt.forward(s0))
        mt.backward(torch.zeros_like(g))
    gt = torch.zeros_like(g) + g
    ms_f = sorted(timed(stream, lambda: mt.forward(s0, replay=True)) for _ in range(3))[1]
    ms_b = sorted(timed(stream, lambda: mt.backward(gt)) for _ in range(3))[1]
    if mt is not m:
        mt.close()
    x = I.cell_centres(p)
    y = (np.arange(p.yres) + 0.5) * 2 * np.pi / p.yres
    d = torch.tensor(np.cos(2 * y[:, None] + 1.0) * np.sin(3 * x[None, :]) + 0.3, device=s0.device) * s0
    ad = float((gs0 * d).sum())
    fd = {}
    # steps down to 1e-10: on a noisy disk the exact derivative differs from the
    # 1e-6 difference quotient at cells on azimuthal pressure extrema, where the
    # PPM flattening coefficient varies on a 1e-8 scale
    for eps in (1.0e-6, 1.0e-7, 1.0e-8, 1.0e-9, 1.0e-10):
        fd[str(eps)] = (loss(m.forward(s0 + eps * d, replay=True)) - loss(m.forward(s0 - eps * d, replay=True))) / (2 * eps)
    # the same check from a generic smooth state (no noise, a 1 % spiral; the
    # recorded dt schedule replayed): the quotients converge to the adjoint
    s0s = torch.tensor(I.disk_state(p, seed=SEED_DUST, noise=0.0)["r"]
                       * (1.0 + 0.01 * np.sin(y[:, None] + 3.0 * np.log(x[None, :]))), device=s0.device)
    outs = m.forward(s0s, replay=True)
    gsm = (2.0 * (outs.mean(0) - target) / p.yres)[None, :].expand(p.yres, p.xres).contiguous()
    gs_s, gth_s = m.backward(gsm)
    ds = d / s0 * s0s
    ad_s = float((gs_s * ds).sum())
    fd_s = {}
    for eps in (1.0e-6, 1.0e-7, 1.0e-8):
        fd_s[str(eps)] = (loss(m.forward(s0s + eps * ds, replay=True)) -
                          loss(m.forward(s0s - eps * ds, replay=True))) / (2 * eps)
    theta = [p.planet_mass, p.ss_alpha, p.sc_h]
    fdt = []
    for k in range(3):
        step = 1.0e-4 * theta[k]
        v = []
        for sg in (1, -1):
            th = list(theta)
            th[k] += sg * step
            m.set_theta(*th)
            v.append(loss(m.forward(s0, replay=True)))
        fdt.append((v[0] - v[1]) / (2 * step))
    m.set_theta(*theta)
    # the loss as a function of each parameter at 9 points 1e-6 apart (relative):
    # the forward map is two-valued there (a branch decision at a rounding-level
    # tie flips with the parameter's last bits, shifting the loss by a fixed
    # amount), so a central difference whose two points fall on different levels
    # is no derivative; the two-level least-squares slope is, and the plain
    # central difference at 1e-6 is reported beside it
    def theta_scan(state, model, target_loss):
        res = []
        for k in range(3):
            ss = [j * 1.0e-6 for j in range(-4, 5)]
            Ls = []
            for s_ in ss:
                th = list(theta)
                th[k] = theta[k] * (1.0 + s_)
                model.set_theta(*th)
                Ls.append(target_loss(model.forward(state, replay=True)))
            model.set_theta(*theta)
            res.append((np.array(ss) * theta[k], np.array(Ls)))
        return res

    def scan_summary(res, grad):
        out = []
        for k, (xs, Ls) in enumerate(res):
            fit = two_level_slope(xs, Ls)
            central = (Ls[5] - Ls[3]) / (xs[5] - xs[3])
            out.append({"two_level_slope": fit["slope"], "levels": fit["levels"], "jump": fit["jump"],
                        "central_1e-6": central,
                        "rel_err_two_level": abs(fit["slope"] - grad[k]) / abs(grad[k]),
                        "rel_err_central_1e-6": abs(central - grad[k]) / abs(grad[k])})
        return out

    scan = scan_summary(theta_scan(s0, m, loss), gth)
    # the same on the smooth state, against its adjoint of the same loss (gth_s)
    scan_s = scan_summary(theta_scan(s0s, m, loss), gth_s)
    out_line = {
        "workload": "256x768 gradient disk, FP64 forward + adjoint, checkpoint every 64 steps",
        "steps": steps, "timing_steps": tsteps, "forward_ms_per_step": ms_f / tsteps,
        "adjoint_ms_per_step": ms_b / tsteps, "adjoint_over_forward": ms_b / ms_f,
        "forward_record_ms_per_step": ms_rec / tsteps,
        "timing": "medians of 3 after a warm-up backward over timing_steps steps (checkpoint segments of 64); "
                  "forward = replay of the recorded dt schedule",
        "device_bytes": m.device_bytes,
        "fd_sigma0": {"state": "the workload's noisy disk", "adjoint": ad, "central": fd,
                      "rel_err": {k: abs(ad - v) / abs(v) for k, v in fd.items()}},
        "fd_sigma0_smooth": {"state": "no noise, 1 % spiral", "adjoint": ad_s, "central": fd_s,
                             "rel_err": {k: abs(ad_s - v) / abs(v) for k, v in fd_s.items()}},
        "fd_theta": {"names": ["q", "alpha", "h"], "adjoint": [float(v) for v in gth], "central_rel_step_1e-4": fdt,
                     "rel_err": [abs(a - b) / abs(b) for a, b in zip(gth, fdt)]},
        "fd_theta_scan": {"names": ["q", "alpha", "h"], "points": "9 at relative spacing 1e-6",
                          "state": "the workload's noisy disk", "per_parameter": scan},
        "fd_theta_scan_smooth": {"names": ["q", "alpha", "h"], "points": "9 at relative spacing 1e-6",
                                 "state": "no noise, 1 % spiral", "adjoint": [float(v) for v in gth_s],
                                 "per_parameter": scan_s},
    }
    m.close()
    return out_line


def two_level_slope(x, y):
    """Least-squares slope of y(x) allowing the samples to sit on two levels a
    fixed jump apart.  A robust line (Theil-Sen: the median of the pairwise
    slopes, which pairs on one level give exactly) leaves residuals in two
    clusters; they are split at their largest gap when it exceeds 20x the spread
    on either side, and y = a + J z + b x is solved with z the level of each
    sample."""
    import numpy as np

    n = len(x)
    pair = [(y[j] - y[i]) / (x[j] - x[i]) for i in range(n) for j in range(i + 1, n) if x[j] != x[i]]
    b0 = float(np.median(pair))
    r = y - b0 * x
    order = np.argsort(r)
    gaps = np.diff(r[order])
    z = np.zeros_like(x)
    if len(gaps):
        g = int(np.argmax(gaps))
        lo, hi = r[order[:g + 1]], r[order[g + 1:]]
        spread = max(np.ptp(lo) if len(lo) > 1 else 0.0, np.ptp(hi) if len(hi) > 1 else 0.0)
        if gaps[g] > 20.0 * spread and len(lo) >= 2 and len(hi) >= 2:
            z[order[g + 1:]] = 1.0
    if z.any():
        a, J, b = np.linalg.lstsq(np.vstack([np.ones_like(x), z, x]).T, y, rcond=None)[0]
    else:
        (a, b), J = np.linalg.lstsq(np.vstack([np.ones_like(x), x]).T, y, rcond=None)[0], 0.0
    return {"slope": float(b), "jump": float(J), "levels": [int((z == 0).sum()), int((z == 1).sum())]}


def measure_sph3d(local, stream, steps, pk, size=None):
    """The reference's 3D preset (include/para_files/Adiabatic_CPD.h: spherical r,
    phi, theta, 384x768x216 = 63.7 M cells, adiabatic, planet q 3e-5, wave
    damping) from the seeded disk after one orbit: zone-updates/s of the
    device-resident loop over ``steps`` steps, each pass's device time, and the
    slowest sweep against its HBM and FP64-issue rooflines."""
    import numpy as np
    import torch

    from penguin_b200 import initial as I
    from penguin_b200 import params as P
    from penguin_b200.disk3 import Disk3

    p = P.spherical_disk(*size) if size else P.spherical_disk()
    st = I.spherical_state(p, seed=1234, vnoise=1.0e-3)
    d = Disk3(p, device=local, stream=stream.cuda_stream)
    d.set_state(2.0 * np.pi, st)
    d.run(3)
    d.check()
    passes = d.pass_times(max(2, min(10, steps)))
    K = max(2, min(20, steps))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    d.run(K)
    e1.record(stream)
    e1.synchronize()
    d.check()
    ms = e0.elapsed_time(e1) / K
    d.close()
    cells = p.cells
    sweep = max(("sweep_x", "sweep_y", "sweep_z"), key=lambda k: passes[k])
    achieved = 80.0 * cells / (passes[sweep] / 1000.0) / 1e9
    out = {"workload": f"3D spherical preset {p.xres}x{p.yres}x{p.zres} (Adiabatic_CPD.h), FP64, "
                       "seeded disk after one orbit", "cells": cells, "steps": K,
           "value": cells / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms, "pass_ms": passes,
           "roofline": {"bound": "hbm", "kernel": sweep, "achieved": achieved, "peak": pk["hbm_gbs"],
                        "unit": "GB/s", "frac": achieved / pk["hbm_gbs"], "algorithmic_bytes_per_cell": 80,
                        "peak_source": pk["source"], "traffic": None}}
    tfile = os.path.join(ROOT, "profiles", "traffic.txt")
    if os.path.exists(tfile):  # per-cell DRAM bytes of a smaller capture, scaled to this grid
        for fl in open(tfile):
            f = fl.split()
            if len(f) >= 2 and not fl.startswith("#") and f[0] == f"sph3d_{sweep}_per_cell":
                out["roofline"]["traffic"] = float(f[1]) * cells
                out["roofline"]["traffic_note"] = "per-cell bytes of the 192x384x96 capture x cells"
    ffile = os.path.join(ROOT, "profiles", "fp64_per_cell.txt")
    if os.path.exists(ffile):
        for fl in open(ffile):
            f = fl.split()
            if len(f) >= 2 and not fl.startswith("#") and f[0] == "sph3d_" + sweep:
                nsm = torch.cuda.get_device_properties(local).multi_processor_count
                peak64 = 64.0 * nsm * 1965.0e6
                ach = float(f[1]) * cells / (passes[sweep] / 1000.0)
                out["roofline_fp64"] = {"kernel": sweep, "achieved": ach, "peak": peak64,
                                        "unit": "FP64 thread-instructions/s", "frac": ach / peak64,
                                        "instructions_per_cell": float(f[1])}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the FP32-mixed, ensemble and dust measurements")
    ap.add_argument("--no-tune", action="store_true", help="default launch configuration instead of the autotuner's")
    ap.add_argument("--adjoint-steps", type=int, default=ADJOINT_STEPS,
                    help="steps of the adjoint's finite-difference checks (the line reports it)")
    ap.add_argument("--adjoint-timing-steps", type=int, default=ADJOINT_TIMING_STEPS,
                    help="steps of the adjoint's timed run (the line reports it)")
    ap.add_argument("--tuning", default=None,
                    help="a fixed launch configuration instead of the autotuner's: comma list of "
                         "key=value over Disk.TUNING (v_sweep_x, ..., cps_kick2)")
    ap.add_argument("--forms", default="fp32,ensemble,dust,adjoint,sph3d",
                    help="comma list of the extra measurements after the FP64 headline "
                         "(fp32, ensemble, dust, adjoint, sph3d)")
    ap.add_argument("--sph3d-size", default=None,
                    help="NR,NPHI,NTHETA of the 3D leg instead of the preset's 384,768,216 (profiling)")
    args = ap.parse_args()

    if args.impl == "reference":
        run_reference(args, int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")))
        return

    import numpy as np
    import torch

    from penguin_b200.replicas import Replicas

    job = Replicas("nccl")
    world, local = job.world, job.local

    from penguin_b200 import initial as I
    from penguin_b200.disk import Disk

    p = workload()
    state = I.disk_state(p, seed=job.seed(1234))
    stream = torch.cuda.Stream()
    disk = Disk(p, device=local, stream=stream.cuda_stream)
    disk.set_state(0.0, state)
    W, K = max(3, args.warmup), args.steps
    if args.tuning:  # a fixed configuration applies from the first step on
        from penguin_b200.disk import describe_tuning

        choice = {k: int(v) for k, v in (kv.split("=") for kv in args.tuning.split(","))}
        disk.set_tuning(choice)
        tuning = dict(choice, passes=describe_tuning(choice), source="--tuning")
    disk.run(W)
    disk.sync()
    disk.check()
    if not args.tuning:
        tuning = disk.autotune(reps=5) if not args.no_tune else None

    def barrier():
        job.barrier(torch.cuda.synchronize)

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        barrier()
        e0.record(stream)
        disk.run(K)
        e1.record(stream)
        clk.wait(e1)
        barrier()
    ms = e0.elapsed_time(e1)
    disk.check()
    clocks = clk.summary()
    ms = job.max_over_ranks(ms)
    cells = p.cells
    value = job.job_rate(cells * K, ms)

    # per-stage device times (events between the launches, same stream)
    prof = disk.profile(max(5, min(50, K // 10)))
    stage = max((k for k in prof if ALGO_BYTES.get(k)), key=lambda k: prof[k])
    pk = peaks()
    achieved = ALGO_BYTES[stage] * cells / (prof[stage] / 1000.0) / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.txt")
    if os.path.exists(tfile):
        for line in open(tfile):
            f = line.split()
            if len(f) >= 2 and f[0] == stage and not line.startswith("#"):
                traffic = float(f[1])

    # the same kernel against its FP64-issue roofline: FP64 arithmetic
    # instructions per cell (ncu, profiles/fp64_per_cell.txt) x cells / its time,
    # against 64 FP64 lanes per SM x SMs x the max SM clock
    roofline_fp64 = None
    ffile = os.path.join(ROOT, "profiles", "fp64_per_cell.txt")
    if os.path.exists(ffile):
        per_cell = {}
        for fl in open(ffile):
            f = fl.split()
            if len(f) >= 2 and not fl.startswith("#"):
                per_cell[f[0]] = float(f[1])
        if stage in per_cell:
            nsm = torch.cuda.get_device_properties(local).multi_processor_count
            mhz = clocks.get("sm_max_mhz") or 1965.0
            peak64 = 64.0 * nsm * mhz * 1e6
            ach = per_cell[stage] * cells / (prof[stage] / 1000.0)
            roofline_fp64 = {"bound": "fp64", "kernel": stage, "achieved": ach, "peak": peak64,
                             "unit": "FP64 thread-instructions/s", "frac": ach / peak64,
                             "instructions_per_cell": per_cell[stage],
                             "peak_source": f"nominal: 64 FP64 lanes per SM x {nsm} SMs x {mhz:.0f} MHz"}

    # end to end through the public API with host buffers: pinned H2D of the
    # initial state, main.cu's host loop (global_dt read back every step, solve),
    # D2H of the final state
    pinned = {k: torch.empty((p.yres, p.xres), dtype=torch.float64, pin_memory=True).numpy() for k in "rpuv"}
    for k in "rpuv":
        pinned[k][...] = state[k]
    out = {k: torch.empty((p.yres, p.xres), dtype=torch.float64, pin_memory=True).numpy() for k in "rpuv"}
    # a run of at least 200 steps whatever --steps is (about 0.25 s): the state
    # exchange is paid once per run, as a user of the loop pays it
    Ke = max(E2E_MIN_STEPS, min(K, 1000))
    import ctypes

    from penguin_b200._lib import check, lib

    def dp(a):
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))

    barrier()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0 = time.perf_counter()
    g0.record(stream)
    check(lib().pg_disk_set_state(disk._h, 0.0, dp(pinned["r"]), dp(pinned["p"]), dp(pinned["u"]), dp(pinned["v"])))
    disk.t, disk.dt = 0.0, None
    h1 = time.perf_counter()
    disk.step_host(Ke)
    h2 = time.perf_counter()
    t_out = ctypes.c_double()
    check(lib().pg_disk_get_state(disk._h, dp(out["r"]), dp(out["p"]), dp(out["u"]), dp(out["v"]),
                                  ctypes.byref(t_out)))
    g1.record(stream)
    g1.synchronize()
    h3 = time.perf_counter()
    e2e_ms = g0.elapsed_time(g1)
    e2e_ms = job.max_over_ranks(e2e_ms)
    e2e = {"value": job.job_rate(cells * Ke, e2e_ms), "unit": UNIT,
           "h2d_bytes_per_step": 4 * 8 * cells // Ke,
           "d2h_bytes_per_step": 8 + 4 * 8 * cells // Ke,
           "steps": Ke,
           "host_ms": {"state_in": 1e3 * (h1 - h0), "loop": 1e3 * (h2 - h1), "state_out": 1e3 * (h3 - h2)},
           "note": "pinned host state in, main.cu host loop (dt read back each step), final state out; "
                   "at least 200 steps whatever --steps is"}
    if not np.isfinite(out["r"]).all():
        raise RuntimeError("non-finite density after the end-to-end run")

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": config_of(p, world),
        "tuning": tuning,
        "gpu_launches": disk.kernels_per_step * K,
        "stage_ms": prof,
        "roofline": {"bound": "hbm", "kernel": stage, "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / pk["hbm_gbs"], "traffic": traffic, "peak_source": pk["source"],
                     "algorithmic_bytes_per_cell": ALGO_BYTES[stage]},
        "roofline_fp64": roofline_fp64,
        "clocks": clocks,
        "e2e": e2e,
    }
    forms = set() if args.no_forms else set(x for x in args.forms.split(",") if x)
    if "fp32" in forms:
        f32 = measure_fp32(p, state, K, W, local, stream, pk)
        f32["over_fp64"] = f32["value"] / (value / world)
        line["fp32_mixed"] = f32
    if "ensemble" in forms:
        line["ensemble"] = measure_ensemble(job, local, stream, ENSEMBLE_STEPS)
    if "dust" in forms:
        line["dust"] = measure_dust(local, stream, min(DUST_STEPS, max(K, 3)), pk)
    if "adjoint" in forms:
        # fixed sizes, independent of --steps: the finite-difference checks over
        # ADJOINT_STEPS steps and the timing over ADJOINT_TIMING_STEPS (16
        # checkpoint segments); together well under a second of GPU time
        line["adjoint"] = measure_adjoint(args.adjoint_steps, local, stream, args.adjoint_timing_steps)
    if "sph3d" in forms:
        size = tuple(int(x) for x in args.sph3d_size.split(",")) if args.sph3d_size else None
        line["sph3d"] = measure_sph3d(local, stream, K, pk, size)
    if job.printer and world == 1 and not args.no_cpu_baseline:
        cb, orc, n_orc = cpu_baseline(p, state, 0.0, keep=True)
        line["cpu_baseline"] = cb
        line["parity"] = parity_vs_oracle(p, state, orc, n_orc, local, stream)
        orc.close()
    line["summary"] = summary_of(line)
    if job.printer:
        print(json.dumps(line), flush=True)
    disk.close()
    job.close()


def parity_vs_oracle(p, state, orc, n, local, stream):
    """The oracle's state after the CPU-baseline leg (n steps of main.cu's loop
    from the workload's initial state) against the CUDA path stepped the same n
    steps from the same state: relative L1 of Sigma, p and the momentum vector."""
    import numpy as np

    from penguin_b200.disk import Disk

    d = Disk(p, device=local, stream=stream.cuda_stream)
    d.set_state(0.0, state)
    d.run(n)
    d.sync()
    d.check()
    t, _, steps = d.clock()
    g, o = d.get_state(), orc.interior()
    d.close()

    def rl1(a, b):
        return float(np.abs(a - b).sum() / np.abs(b).sum())

    mom = float((np.abs(g["r"] * g["u"] - o["r"] * o["u"]) + np.abs(g["r"] * g["v"] - o["r"] * o["v"])).sum()
                / (np.abs(o["r"] * o["u"]) + np.abs(o["r"] * o["v"])).sum())
    return {"steps": int(steps), "rel_l1_r": rl1(g["r"], o["r"]), "rel_l1_p": rl1(g["p"], o["p"]),
            "rel_l1_mom": mom, "t_rel_diff": abs(t - orc.t) / orc.t,
            "against": "the oracle (CPU restatement of the reference step), same initial state and step count"}


def summary_of(line):
    """The headline rate and the ratios of every form against the FP64 form, in one
    place at the end of the line."""
    out = {"fp64_gzone_s": line["value"] / 1e9, "fp64_ms_per_step": line["ms_per_step"],
           "sweep_hbm_frac": line["roofline"]["frac"]}
    if line.get("roofline_fp64"):
        out["sweep_fp64_issue_frac"] = line["roofline_fp64"]["frac"]
    if "e2e" in line:
        out["e2e_gzone_s"] = line["e2e"]["value"] / 1e9
    if "fp32_mixed" in line:
        out["fp32_over_fp64"] = line["fp32_mixed"]["over_fp64"]
    if "ensemble" in line:
        out["ensemble_over_sequential_fp64"] = line["ensemble"]["over_sequential_fp64"]
    if "dust" in line:
        out["dust_fp32_over_fp64"] = {k: v["fp32_mixed"]["over_fp64"] for k, v in line["dust"].items()
                                      if isinstance(v, dict) and "fp32_mixed" in v}
    if "adjoint" in line:
        a = line["adjoint"]
        out["adjoint_over_forward"] = a["adjoint_over_forward"]
        out["adjoint_fd_rel_err"] = {"sigma0_smooth_1e-6": a["fd_sigma0_smooth"]["rel_err"]["1e-06"],
                                     "sigma0_noisy_1e-6": a["fd_sigma0"]["rel_err"]["1e-06"],
                                     "theta_1e-4": a["fd_theta"]["rel_err"],
                                     "theta_two_level_1e-6": [v["rel_err_two_level"]
                                                              for v in a["fd_theta_scan"]["per_parameter"]],
                                     "theta_smooth_two_level_1e-6": [
                                         v["rel_err_two_level"] for v in a["fd_theta_scan_smooth"]["per_parameter"]]}
    if "sph3d" in line:
        out["sph3d_gzone_s"] = line["sph3d"]["value"] / 1e9
    if "parity" in line:
        q = line["parity"]
        out["parity_rel_l1_max"] = max(q["rel_l1_r"], q["rel_l1_p"], q["rel_l1_mom"])
        out["parity_steps"] = q["steps"]
    return out


if __name__ == "__main__":
    main()
