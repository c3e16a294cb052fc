"""Gas + one dust fluid (dust_flag, src/solver/dust/dust.cu) on the sm_100a
path, through the C ABI, against the oracle and the reference's own outputs.
Needs a B200."""
import os

import numpy as np
import pytest

import cases as C
from oracle.oracle import Oracle
from penguin_b200 import initial as I
from penguin_b200 import params as P
from penguin_b200._lib import PG_ERR_CONFIG, PGError
from penguin_b200.disk import Disk

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GAS = ("r", "p", "u", "v")


def rel_l1(a, b):
    return np.abs(a - b).sum() / np.abs(b).sum()


def momentum_l1(a, b):
    ax, ay, bx, by = a["r"] * a["u"], a["r"] * a["v"], b["r"] * b["u"], b["r"] * b["v"]
    return (np.abs(ax - bx) + np.abs(ay - by)).sum() / (np.abs(bx) + np.abs(by)).sum()


def _errors(gas, dust, gref, dref):
    return {
        "r": rel_l1(gas["r"], gref["r"]),
        "p": rel_l1(gas["p"], gref["p"]),
        "momentum": momentum_l1(gas, gref),
        "dust_r": rel_l1(dust["r"], dref["r"]),
        "dust_momentum": momentum_l1(dust, dref),
    }


@pytest.mark.parametrize("case", C.dust_cases(), ids=lambda c: c["name"])
def test_cuda_dust_matches_oracle(case):
    p, st = case["params"], C.initial_state(case)
    o = Oracle(p, st, case["t0"])
    n = o.run(case["max_step"], case["end_time"])
    d = Disk(p)
    d.set_state(case["t0"], st)
    assert d.step_host(case["max_step"], case["end_time"]) == n
    d.check()
    # the oracle's CFL reduction sums in another order (as for the gas-only cases)
    bar = max(case["tol"], case["cuda_tol"])  # the oracle's own distance from the reference bounds this
    assert d.t == pytest.approx(o.t, rel=max(1e-13, bar))
    # relative L1 bars per case ("tol", "cuda_tol" in tests/golden/cases.py)
    errs = _errors(d.get_state(), d.get_dust(), o.interior(), o.dust())
    assert all(e < bar for e in errs.values()), errs


@pytest.mark.parametrize("case", C.dust_cases(), ids=lambda c: c["name"])
def test_cuda_dust_matches_reference_fixture(case):
    z = np.load(os.path.join(GOLDEN, case["name"] + ".npz"))
    p = case["params"]
    d = Disk(p)
    d.set_state(float(z["t0"]), {k: z["init_" + k] for k in GAS})
    d.step_host(int(z["max_step"]), float(z["end_time"]))
    d.check()
    assert d.t == pytest.approx(float(z["t"]), rel=1e-13)
    errs = _errors(d.get_state(), d.get_dust(), {k: z["out_" + k] for k in GAS},
                   {k: z["out_dust_" + k] for k in ("r", "u", "v")})
    assert all(e < case["cuda_tol"] for e in errs.values()), errs


def test_dust_starts_from_init_cd():
    """init_CD is evaluated on the host, like the reference's fill_grid: bit for bit."""
    p = P.reference_disk(64, 192).replace(dust_flag=1, Stokes=0.01, D_G_ratio=0.01)
    st = I.disk_state(p, seed=1)
    d = Disk(p)
    d.set_state(0.0, st)
    g, o = d.get_dust(), Oracle(p, st, 0.0).dust()
    for k in ("r", "u", "v"):
        assert np.array_equal(g[k], o[k]), k


def test_dust_device_loop_equals_host_loop():
    """The CUDA-graph loop reproduces the host loop bit for bit, dust included."""
    case = [c for c in C.dust_cases() if c["name"] == "dust64_st01_n10"][0]
    p, st = case["params"], C.initial_state(case)
    a = Disk(p)
    a.set_state(case["t0"], st)
    a.step_host(10)
    b = Disk(p)
    b.set_state(case["t0"], st)
    b.run(10)
    b.sync()
    assert b.clock()[0] == a.t
    ga, gb = a.get_state(), b.get_state()
    da, db = a.get_dust(), b.get_dust()
    for k in GAS:
        assert np.array_equal(ga[k], gb[k]), k
    for k in ("r", "u", "v"):
        assert np.array_equal(da[k], db[k]), k


def test_set_dust_round_trip_and_restart():
    """set_dust writes the interior the next step reads; the dust speeds enter the
    CFL rate (a fast dust ring shortens the first step)."""
    p = P.reference_disk(64, 192).replace(dust_flag=1, Stokes=0.1, D_G_ratio=0.01)
    st = I.disk_state(p, seed=5)
    d = Disk(p)
    d.set_state(0.0, st)
    dust = d.get_dust()
    dust["r"] = dust["r"] * (1.0 + 0.1 * np.sin(np.arange(p.yres))[:, None])
    d.set_dust(dust)
    back = d.get_dust()
    for k in ("r", "u", "v"):
        assert np.array_equal(back[k], dust[k]), k
    dt0 = d.global_dt(1.0e30)
    fast = dict(dust, u=dust["u"] + 0 * dust["u"])
    fast["u"][:, 20] = 50.0
    d.set_dust(fast)
    assert d.global_dt(1.0e30) < dt0
    o = Oracle(p, st, 0.0)
    o.set_dust(dust)
    d.set_dust(dust)
    d.step_host(3)
    o.run(3)
    errs = _errors(d.get_state(), d.get_dust(), o.interior(), o.dust())
    assert all(e < 1e-10 for e in errs.values()), errs


def test_dust_rejected_where_unsupported():
    p1 = P.sod_tube(64).replace(dust_flag=1, Stokes=0.1, D_G_ratio=0.01)
    with pytest.raises(PGError) as e:
        Disk(p1)
    assert e.value.status == PG_ERR_CONFIG
    p = P.reference_disk(64, 192)
    d = Disk(p)
    d.set_state(0.0, I.disk_state(p, seed=1))
    with pytest.raises(PGError):
        d.get_dust()
