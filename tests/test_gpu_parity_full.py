"""Parity of the CUDA path with the oracle at the benchmark workloads' own sizes:
the 1024x3072 planet-disk, the 768x2048 gas + dust disk (Stokes 0.01) and the
256x768 gradient disk, each stepped by main.cu's loop (CFL dt, 1.1x growth
cap) from the same seeded state on the GPU and in the oracle.  Needs a B200.

Bars (relative L1 of density, pressure and the momentum vector; dust density
and momentum), per workload after one step and after its step count: the
measured difference with margin.  The oracle evaluates the reference's
expressions without FMA contraction and with the host's libm, and on the
3072-cell azimuth that puts it 2e-11 from the reference after 5 steps
(test_gpu_reference_size.py prints the distance), while the CUDA path is
3.5e-13 from the reference there; so the bound against the oracle is the
oracle's own distance from the reference, not 1e-12.  On the 256x768 disk the
oracle is 6e-14 from the reference and the bar is 1e-12.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from penguin_b200 import initial as I
from penguin_b200 import params as P
from penguin_b200.disk import Disk

pytestmark = pytest.mark.gpu


def rel_l1(a, b):
    return float(np.abs(a - b).sum() / np.abs(b).sum())


def momentum_l1(a, b):
    ax, ay = a["r"] * a["u"], a["r"] * a["v"]
    bx, by = b["r"] * b["u"], b["r"] * b["v"]
    return float((np.abs(ax - bx) + np.abs(ay - by)).sum() / (np.abs(bx) + np.abs(by)).sum())


def _run_both(p, steps, seed=1234, t0=0.0):
    st = I.disk_state(p, seed=seed)
    o = Oracle(p, st, t0)
    d = Disk(p)
    d.set_state(t0, st)
    out = []
    done = 0
    for n in steps:
        o.run(n - done)
        d.run(n - done)
        d.sync()
        d.check()
        done = n
        g, r = d.get_state(), o.interior()
        errs = {"r": rel_l1(g["r"], r["r"]), "p": rel_l1(g["p"], r["p"]), "momentum": momentum_l1(g, r)}
        if p.dust_flag:
            gd, rd = d.get_dust(), o.dust()
            errs["dust_r"] = rel_l1(gd["r"], rd["r"])
            errs["dust_momentum"] = momentum_l1(gd, rd)
        t, _, nd = d.clock()
        assert nd == n
        assert t == pytest.approx(o.t, rel=1e-13)
        print(f"{p.xres}x{p.yres} after {n} steps: " + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
        out.append(errs)
    d.close()
    o.close()
    return out


# (workload, steps, bound after one step, bound after the last step); measured:
# 1024x3072 1.7e-11 / 2.2e-11, 768x2048 3.4e-12 / 4.4e-12, 256x768 7.8e-14 / 1.3e-13
WORKLOADS = {
    "disk1024x3072": (lambda: P.planet_disk(1024, 3072), 5, 4e-11, 5e-11),
    "dust768x2048_st001": (lambda: P.dust_disk(stokes=0.01), 5, 1e-11, 1e-11),
    "adjoint256x768": (lambda: P.adjoint_disk(), 20, 1e-12, 1e-12),
}


@pytest.mark.parametrize("name", sorted(WORKLOADS))
def test_cuda_matches_oracle_at_workload_size(name):
    make, n, bound1, bound = WORKLOADS[name]
    e1, en = _run_both(make(), [1, n])
    assert all(v < bound1 for v in e1.values()), e1
    assert all(v < bound for v in en.values()), en
