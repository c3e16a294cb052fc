"""Dust in the FP32-mixed form (pg_ens_* with dust_flag): agreement with the
FP64 dust path at the FP32 rounding level, set/get and restart semantics, and
independence of a dusty member's result from the ensemble it runs in.  Needs a
B200."""
import numpy as np
import pytest

import cases as C
from penguin_b200 import initial as I
from penguin_b200 import params as P
from penguin_b200.disk import Disk
from penguin_b200.ensemble import Ensemble

pytestmark = pytest.mark.gpu

# FP32 residuals against init_CD, fluxes from deviations: the dust density
# agrees with FP64 to ~1e-7 relative, the dust velocities to ~1e-4 of the size of
# their deviation from init_CD (as for the gas, tests/test_f32.py).
SIGMA_TOL = 2e-6
RESID_TOL = 1e-4


def rel_l1(a, b):
    return np.abs(a - b).sum() / np.abs(b).sum()


def dusty(nr=64, nphi=192, stokes=0.1, **kw):
    return P.dust_disk(nr, nphi, stokes=stokes, **kw)


def _init_dust(p):
    d = Disk(p)
    d.set_state(0.0, I.disk_state(p, seed=1))
    out = d.get_dust()
    d.close()
    return out


@pytest.mark.parametrize("stokes", [0.01, 0.1])
def test_f32_dust_tracks_fp64(stokes):
    p = dusty(stokes=stokes)
    st = I.disk_state(p, seed=C.SEED)
    t0, t1 = C.T0_DISK, C.T0_DISK + 0.2
    d = Disk(p)
    d.set_state(t0, st)
    d.run(10 ** 6, t1)
    d.sync()
    d.check()
    e = Ensemble([p])
    e.set_state(0, t0, st)
    e.run(10 ** 6, t1)
    e.sync()
    e.check()
    ref, got = d.get_dust(), e.get_dust(0)
    base = _init_dust(p)
    assert e.clock(0)[0] == pytest.approx(t1, abs=1e-12)
    err = {"r": rel_l1(got["r"], ref["r"]),
           "u": np.abs(got["u"] - ref["u"]).sum() / np.abs(ref["u"] - base["u"]).sum(),
           "v": np.abs(got["v"] - ref["v"]).sum() / np.abs(ref["v"] - base["v"]).sum()}
    assert err["r"] < SIGMA_TOL and err["u"] < RESID_TOL and err["v"] < RESID_TOL, err
    assert rel_l1(e.get_state(0)["r"], d.get_state()["r"]) < SIGMA_TOL


def test_f32_dust_set_get_and_restart():
    p = dusty()
    st = I.disk_state(p, seed=2)
    e = Ensemble([p])
    e.set_state(0, 0.0, st)
    base = e.get_dust(0)
    ref = _init_dust(p)
    for k in ("r", "u", "v"):  # init_CD, to the FP32 rounding of the residual (zero)
        assert np.array_equal(base[k], ref[k]), k
    mod = dict(base, r=base["r"] * (1.0 + 0.01 * np.cos(np.arange(p.yres))[:, None]))
    e.set_dust(0, mod)
    back = e.get_dust(0)
    assert np.abs(back["r"] - mod["r"]).max() <= 1e-7 * mod["r"].max()
    e.run(3)
    e.sync()
    e.set_state(0, 0.0, st)  # a restart puts the dust back to init_CD
    again = e.get_dust(0)
    for k in ("r", "u", "v"):
        assert np.array_equal(again[k], ref[k]), k


def test_f32_dusty_member_independent_of_ensemble():
    pd = dusty(96, 288)
    pg = P.planet_disk(64, 192)
    sd, sg = I.disk_state(pd, seed=5), I.disk_state(pg, seed=6)
    alone = Ensemble([pd])
    alone.set_state(0, 0.0, sd)
    alone.run(8)
    alone.sync()
    both = Ensemble([pg, pd])
    both.set_state(0, 0.0, sg)
    both.set_state(1, 0.0, sd)
    both.run(8)
    both.sync()
    a, b = alone.get_dust(0), both.get_dust(1)
    for k in ("r", "u", "v"):
        assert np.array_equal(a[k], b[k]), k
    ga, gb = alone.get_state(0), both.get_state(1)
    assert np.array_equal(ga["r"], gb["r"])
