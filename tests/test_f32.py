"""FP32-mixed form and ensembles (pg_ens_*): agreement with the FP64 oracle at
the FP32 rounding level, bitwise independence of a member's result from the
ensemble it runs in, per-member clocks, totals and error reporting.  Needs a
B200."""
import numpy as np
import pytest

import cases as C
from oracle.oracle import Oracle
from penguin_b200 import initial as I
from penguin_b200 import params as P
from penguin_b200._lib import PG_ERR_NAN, PGError
from penguin_b200.disk import Disk, make_grid
from penguin_b200.ensemble import Ensemble

pytestmark = pytest.mark.gpu

# Bars of the FP32 form against FP64 after 20 steps of a planet-disk.  The state
# is stored as FP32 residuals against the FP64 initial disk and every flux is
# formed from deviations, so errors scale with the local variation of a field,
# not with its magnitude: density to ~1e-7 relative (FP32 epsilon 6e-8), the
# velocity residuals to ~1e-5 of their own size.
SIGMA_TOL = 2e-6
RESID_TOL = 1e-4


def rel_l1(a, b):
    return np.abs(a - b).sum() / np.abs(b).sum()


def _resid_err(got, ref, base, key):
    """L1 error of a field relative to the L1 size of its deviation from base."""
    return np.abs(got[key] - ref[key]).sum() / np.abs(ref[key] - base[key]).sum()


def _errs(g, ref, st):
    return {"r": rel_l1(g["r"], ref["r"]), "u": _resid_err(g, ref, st, "u"), "v": _resid_err(g, ref, st, "v")}


def test_f32_single_disk_tracks_fp64_oracle():
    p = P.planet_disk(64, 192)
    st = I.disk_state(p, seed=C.SEED)
    t0 = C.T0_DISK
    o = Oracle(p, st, t0)
    o.run(20)
    ref = o.interior()
    e = Ensemble([p])
    e.set_state(0, t0, st)
    e.run(20)
    e.sync()
    e.check()
    g = e.get_state(0)
    assert g["t"] == pytest.approx(o.t, rel=1e-6)
    errs = _errs(g, ref, st)
    assert errs["r"] < SIGMA_TOL and errs["u"] < RESID_TOL and errs["v"] < RESID_TOL, errs


def test_f32_tracks_fp64_cuda_path_on_a_larger_disk():
    p = P.planet_disk(256, 768)
    st = I.disk_state(p, seed=3)
    t0 = C.T0_DISK
    d = Disk(p)
    d.set_state(t0, st)
    d.run(100)
    d.sync()
    d.check()
    ref = d.get_state()
    e = Ensemble([p])
    e.set_state(0, t0, st)
    e.run(100)
    e.sync()
    e.check()
    errs = _errs(e.get_state(0), ref, st)
    assert errs["r"] < 5 * SIGMA_TOL and errs["u"] < 5 * RESID_TOL and errs["v"] < 5 * RESID_TOL, errs


MEMBERS = [
    dict(nr=64, nphi=192, q=1.0e-4, alpha=1.0e-3, h=0.05),
    dict(nr=96, nphi=288, q=3.0e-3, alpha=1.0e-2, h=0.08),
    dict(nr=128, nphi=384, q=1.0e-5, alpha=1.0e-4, h=0.03),
]


def _member(m):
    return P.planet_disk(m["nr"], m["nphi"], q=m["q"], alpha=m["alpha"], h=m["h"])


def test_ensemble_members_equal_solo_runs_bitwise():
    ps = [_member(m) for m in MEMBERS]
    sts = [I.disk_state(p, seed=11 + k) for k, p in enumerate(ps)]
    e = Ensemble(ps)
    for k, st in enumerate(sts):
        e.set_state(k, C.T0_DISK, st)
    e.run(30)
    e.sync()
    e.check()
    for k, (p, st) in enumerate(zip(ps, sts)):
        solo = Ensemble([p])
        solo.set_state(0, C.T0_DISK, st)
        solo.run(30)
        solo.sync()
        a, b = e.get_state(k), solo.get_state(0)
        for key in ("r", "u", "v"):
            assert np.array_equal(a[key], b[key]), (k, key)
        assert e.clock(k) == solo.clock(0)
        solo.close()
    # each member took its own CFL step
    dts = [e.clock(k)[1] for k in range(len(ps))]
    assert len(set(dts)) == len(dts)


def test_ensemble_autotune_keeps_results_bitwise():
    """The autotuner changes only launch configurations: after tuning (on the
    current state, which it leaves alone) the run equals an untuned one bit for
    bit, and every configuration it can pick is valid."""
    ps = [_member(m) for m in MEMBERS]
    sts = [I.disk_state(p, seed=21 + k) for k, p in enumerate(ps)]
    runs = []
    for tune in (False, True, "max"):
        e = Ensemble(ps)
        for k, st in enumerate(sts):
            e.set_state(k, C.T0_DISK, st)
        e.run(2)
        if tune is True:
            choice = e.autotune(reps=2)
            assert set(choice) == set(Ensemble.TUNING)
        elif tune == "max":  # the other occupancy variant of every pass, one CTA per SM
            e.set_tuning({k: 1 for k in Ensemble.TUNING})
        e.run(20)
        e.sync()
        e.check()
        runs.append([e.get_state(k) for k in range(len(ps))])
        e.close()
    for other in runs[1:]:
        for a, b in zip(runs[0], other):
            for key in ("r", "u", "v"):
                assert np.array_equal(a[key], b[key]), key


def test_f32_first_dt_matches_fp64():
    p = P.planet_disk(128, 384)
    st = I.disk_state(p, seed=5)
    d = Disk(p)
    d.set_state(C.T0_DISK, st)
    d.run(1)
    d.sync()
    e = Ensemble([p])
    e.set_state(0, C.T0_DISK, st)
    e.run(1)
    e.sync()
    assert e.clock(0)[1] == pytest.approx(d.clock()[1], rel=1e-6)


def test_totals_are_compensated_fp64_sums():
    p = P.planet_disk(128, 384)
    st = I.disk_state(p, seed=9)
    e = Ensemble([p])
    e.set_state(0, C.T0_DISK, st)
    m, l = e.totals(0)
    xa, xv, ya, yv = make_grid(p)
    dV = xv[3:3 + p.xres][None, :] * yv[3:3 + p.yres][:, None]
    x = I.cell_centres(p)
    m_ref = np.sum(st["r"] * dV)
    l_ref = np.sum(st["r"] * x[None, :] * st["v"] * dV)
    # the state is held as FP32 residuals (|dSigma| ~ 1e-4 Sigma) around FP64 Sigma_0
    assert m == pytest.approx(m_ref, rel=1e-10)
    assert l == pytest.approx(l_ref, rel=1e-10)


def test_end_time_stops_each_member_on_its_own_clock():
    ps = [_member(MEMBERS[0]), _member(MEMBERS[1])]

    def started():
        e = Ensemble(ps)
        for k, p in enumerate(ps):
            e.set_state(k, C.T0_DISK, I.disk_state(p, seed=k))
        e.run(5)
        e.sync()
        return e

    a = started()
    t_end = max(a.clock(0)[0], a.clock(1)[0]) + 0.1
    a.run(400, t_end)  # members finish after a few steps and are copied through after that
    a.sync()
    steps = [a.clock(k)[2] for k in range(2)]
    for k in range(2):
        assert a.clock(k)[0] == pytest.approx(t_end, abs=1e-12)
    b = started()
    b.run(max(steps) - 5, t_end)
    b.sync()
    for k in range(2):
        assert b.clock(k)[2] == steps[k]
        ga, gb = a.get_state(k), b.get_state(k)
        for key in ("r", "u", "v"):
            assert np.array_equal(ga[key], gb[key]), (k, key)


def test_f32_nan_sets_error_word():
    p = P.planet_disk(64, 192)
    st = I.disk_state(p, seed=1)
    st["r"][10, 10] = -1.0
    e = Ensemble([p])
    e.set_state(0, C.T0_DISK, st)
    e.run(1)
    e.sync()
    with pytest.raises(PGError) as ei:
        e.check()
    assert ei.value.status == PG_ERR_NAN


def test_f32_torque_tracks_fp64():
    p = P.planet_disk(128, 384)
    st = I.disk_state(p, seed=4)
    d = Disk(p)
    d.set_state(C.T0_DISK, st)
    d.run(20)
    d.sync()
    e = Ensemble([p])
    e.set_state(0, C.T0_DISK, st)
    e.run(20)
    e.sync()
    # the torque is dominated by the near-planet density, FP32-accurate to ~1e-6 here
    assert e.torque(0) == pytest.approx(d.torque(), rel=1e-4)
