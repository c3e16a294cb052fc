"""The CPU oracle, pinned against the unmodified reference (fixtures in
tests/golden, made by tests/golden/make_golden.py on a B200) and against the
exact Sod solution.  CPU only."""
import json
import os

import numpy as np
import pytest

import cases as C
from exact_riemann import sample, star_state
from oracle.oracle import Oracle
from penguin_b200 import initial as I
from penguin_b200 import params as P

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# The oracle evaluates the reference's expressions in the same order but without
# FMA contraction and with glibc's pow/sin/sincos; killwave's FP32 __sinf ramp is
# evaluated with sinf.  Each golden case carries its relative-L1 bound ("tol",
# tests/golden/cases.py) for density, pressure and momentum.


def rel_l1(a, b):
    den = np.abs(b).sum()
    return np.abs(a - b).sum() / den if den > 0 else np.abs(a - b).sum()


def momentum_l1(a, b):
    """relative L1 of the momentum vector (rho u, rho v)"""
    ax, ay = a["r"] * a["u"], a["r"] * a.get("v", 0 * a["r"])
    bx, by = b["r"] * b["u"], b["r"] * b.get("v", 0 * b["r"])
    return (np.abs(ax - bx) + np.abs(ay - by)).sum() / (np.abs(bx) + np.abs(by)).sum()


def _load(name):
    path = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(path):
        pytest.skip(f"fixture {name} missing")
    return np.load(path)


@pytest.mark.parametrize("case", C.cases(), ids=lambda c: c["name"])
def test_oracle_matches_reference(case):
    z = _load(case["name"])
    p = case["params"]
    assert json.loads(str(z["params"]))["xres"] == p.xres
    keys = ["r", "p", "u"] + (["v"] if p.ndim > 1 else [])
    st = {k: z["init_" + k] for k in keys}
    for k in keys:
        assert np.isfinite(z["out_" + k]).all(), f"reference output {k} not finite"
    o = Oracle(p, st, float(z["t0"]))
    o.run(int(z["max_step"]), float(z["end_time"]))
    assert o.t == pytest.approx(float(z["t"]), rel=max(1e-13, case["tol"]), abs=1e-15)
    out = o.interior()
    ref = {k: z["out_" + k] for k in keys}
    for k in ("r", "p"):
        assert rel_l1(out[k], ref[k]) < case["tol"], (k, rel_l1(out[k], ref[k]))
    if p.ndim == 1:
        out["v"] = 0 * out["r"]
    assert momentum_l1(out, ref) < case["tol"], momentum_l1(out, ref)


@pytest.mark.parametrize("case", C.dust_cases(), ids=lambda c: c["name"])
def test_oracle_dust_matches_reference(case):
    """Gas + dust (src/solver/dust/dust.cu) against the reference's kernels run
    with the shared memory that its dust reconstruction reads zeroed (the
    fixtures' source; see tests/golden/make_golden.py, _run_dust)."""
    z = _load(case["name"])
    p = case["params"]
    st = {k: z["init_" + k] for k in ("r", "p", "u", "v")}
    o = Oracle(p, st, float(z["t0"]))
    o.run(int(z["max_step"]), float(z["end_time"]))
    assert o.t == pytest.approx(float(z["t"]), rel=max(1e-13, case["tol"]))
    out, d = o.interior(), o.dust()
    ref = {k: z["out_" + k] for k in ("r", "p", "u", "v")}
    assert rel_l1(out["r"], ref["r"]) < case["tol"]
    assert momentum_l1(out, ref) < case["tol"]
    dref = {k: z["out_dust_" + k] for k in ("r", "u", "v")}
    assert rel_l1(d["r"], dref["r"]) < case["tol"], rel_l1(d["r"], dref["r"])
    assert momentum_l1(d, dref) < case["tol"], momentum_l1(d, dref)
    assert np.all(z["out_dust_w"] == 0.0)


def test_oracle_dust_starts_from_init_cd():
    """init_CD (src/init/init.cu:351-454): Sigma_d = D_G_ratio Sigma_0, v_phi = v_K,
    and the drift speed solves the terminal-velocity relation of the pressure-
    supported gas (|v_r,d| grows with St below St = 1)."""
    p = P.planet_disk(64, 192).replace(dust_flag=1, Stokes=0.01, D_G_ratio=0.01)
    o = Oracle(p, I.disk_state(p, seed=1), 0.0)
    d = o.dust()
    x = I.cell_centres(p)
    assert np.allclose(d["r"][0], 0.01 / x, rtol=1e-14)
    assert np.allclose(d["v"][0], np.sqrt(1.0 / x), rtol=1e-14)
    assert (d["u"] < 0).all()
    q = P.planet_disk(64, 192).replace(dust_flag=1, Stokes=0.1, D_G_ratio=0.01)
    assert (np.abs(Oracle(q, I.disk_state(q, seed=1), 0.0).dust()["u"]) > np.abs(d["u"])).all()


def test_initial_state_regenerates_fixture():
    """The seeded initial states are reproducible (SplitMix64 noise)."""
    for case in C.cases():
        z = _load(case["name"])
        st = C.initial_state(case)
        for k in ("r", "p", "u"):
            np.testing.assert_allclose(st[k], z["init_" + k], rtol=1e-14, atol=0)


def test_sod_exact_solution():
    """Oracle Sod tube at t=0.2 against the exact Riemann solution (Toro ch. 4)."""
    p = P.sod_tube(1024)
    o = Oracle(p, I.sod_state(p), 0.0)
    o.run(10**6, 0.2)
    assert o.t == pytest.approx(0.2, abs=1e-15)
    st = o.interior()
    x = I.cell_centres(p)
    ex = sample((1.0, 0.0, 1.0), (0.125, 0.0, 0.1), (x - 0.5) / 0.2)
    l1 = [np.abs(st[k][0] - ex[n]).mean() for n, k in enumerate(("r", "u", "p"))]
    assert l1[0] < 2.5e-3 and l1[1] < 5e-3 and l1[2] < 2e-3, l1
    ps, us = star_state((1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    assert ps == pytest.approx(0.30313, abs=1e-5) and us == pytest.approx(0.92745, abs=1e-5)


def test_sod_conservation():
    """Outflow tube before the waves reach the ends: mass, momentum, energy exact to rounding."""
    p = P.sod_tube(256)
    s = I.sod_state(p)
    o = Oracle(p, s, 0.0)
    o.run(40, 0.2)
    st = o.interior()
    g = p.gam
    m0, m1 = s["r"].sum(), st["r"].sum()
    e0 = (s["p"] / (g - 1) + 0.5 * s["r"] * s["u"] ** 2).sum()
    e1 = (st["p"] / (g - 1) + 0.5 * st["r"] * st["u"] ** 2).sum()
    assert abs(m1 / m0 - 1) < 1e-14
    assert abs(e1 / e0 - 1) < 1e-14
    # zero-gradient ends: total momentum grows by (p_left - p_right) t
    assert abs((st["r"] * st["u"]).sum() / p.xres - (1.0 - 0.1) * o.t) < 1e-13


def test_disk_quiet_without_planet():
    """Unperturbed disk without planet stays near equilibrium (no spurious flows)."""
    p = P.reference_disk(32, 96, q=0.0).replace(kill_flag=0)
    st = I.disk_state(p, noise=0.0)
    o = Oracle(p, st, 0.0)
    o.run(20)
    out = o.interior()
    mid = slice(p.xres // 4, 3 * p.xres // 4)  # away from the boundary-adjustment layers
    assert np.abs(out["u"][:, mid]).max() < 1e-4
    assert rel_l1(out["r"][:, mid], st["r"][:, mid]) < 1e-4
