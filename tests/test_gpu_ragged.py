"""Grids whose sizes are not multiples of any tile: the last tile of every pass
is partly outside the grid (TMA fills it, the kernels write only interior
cells).  The CUDA path against the oracle on such grids, every tile variant
against the default one bit for bit, the FP32-mixed form against FP64 and an
ensemble of ragged members against their solo runs, and the 3D passes, whose
boxes are ragged along all three axes here.  Needs a B200."""
import numpy as np
import pytest

from oracle.oracle import Oracle, Oracle3
from penguin_b200 import initial as I
from penguin_b200 import params as P
from penguin_b200.disk import Disk, sweep_variant
from penguin_b200.disk3 import Disk3
from penguin_b200.ensemble import Ensemble

pytestmark = pytest.mark.gpu

T0 = 5.0 * 2.0 * np.pi  # planet mass halfway up its 10-orbit ramp

# 40 radii: one full 32-cell pencil and one of 8; 100 azimuths: 12 rows of 8 and
# one of 4, 3 pencils of 32 and one of 4.  70 x 206 is ragged against 16, 32
# and 64 alike.
RAGGED_2D = [(40, 100), (70, 206)]


def rel_l1(a, b):
    den = np.abs(b).sum()
    return np.abs(a - b).sum() / den if den > 0 else np.abs(a - b).sum()


def momentum_l1(a, b):
    ax, ay, bx, by = a["r"] * a["u"], a["r"] * a["v"], b["r"] * b["u"], b["r"] * b["v"]
    return (np.abs(ax - bx) + np.abs(ay - by)).sum() / (np.abs(bx) + np.abs(by)).sum()


def _disk(nr, nphi, **kw):
    return P.reference_disk(nr, nphi).replace(**kw)


@pytest.mark.parametrize("full,bar", [(False, 1e-13), (True, 3e-10)], ids=["visc_orbadv", "planet_damping"])
@pytest.mark.parametrize("size", RAGGED_2D, ids=lambda s: f"{s[0]}x{s[1]}")
def test_ragged_disk_matches_oracle(size, full, bar):
    """10 steps with viscosity and orbital advection, then with the planet and
    wave damping added.  With the first two the CUDA path and the oracle (the
    reference's arithmetic without FMA contraction) agree to rounding (the
    32x96 disks' 1e-14 class), so a cell of an overhanging tile that was read
    or written wrongly would stand out.  The damping ramp is the FP32 intrinsic
    __sinf, which the oracle evaluates as sinf (ramps ~4e-7 apart), and the
    planet amplifies contraction differences near it: with both on the bound is
    the order of the 64x192 disk's (1e-10; 1.1e-10 measured on 40x100)."""
    p = _disk(*size) if full else _disk(*size, planet_mass=0.0, kill_flag=0)
    st = I.disk_state(p, seed=17)
    o = Oracle(p, st, T0)
    n = o.run(10)
    d = Disk(p)
    d.set_state(T0, st)
    assert d.step_host(10) == n
    d.check()
    g, ref = d.get_state(), o.interior()
    d.close()
    errs = {k: rel_l1(g[k], ref[k]) for k in ("r", "p")}
    errs["momentum"] = momentum_l1(g, ref)
    assert all(e < bar for e in errs.values()), errs
    assert d.t == pytest.approx(o.t, rel=max(1e-13, bar))


def test_ragged_disk_every_tile_variant_bitwise():
    """Every tile variant the autotuner may choose (pencils per tile, pencil
    length 16/32/64, cells per thread, TMA stages) gives the default variant's
    result bit for bit when the tiles overhang the grid."""
    p = _disk(*RAGGED_2D[1])
    st = I.disk_state(p, seed=18)
    ref = Disk(p)
    ref.set_state(T0, st)
    ref.run(6)
    ref.sync()
    a = ref.get_state()
    ref.close()
    for v in range(10):
        vx = v if sweep_variant(v)["pencil_length"] + 6 <= 51 else 0  # radial boxes of at most 256 doubles
        forced = Disk(p)
        forced.set_state(T0, st)
        forced.set_tuning(dict(zip(Disk.TUNING, (vx, v, v, 1, 1, 1, 1, 1))))
        forced.run(6)
        forced.sync()
        c = forced.get_state()
        forced.close()
        for k in ("r", "p", "u", "v"):
            assert np.array_equal(a[k], c[k]), (v, k)


def test_ragged_sod_tube_matches_oracle():
    """1D: 100 cells (three full 32-cell pencils and one of 4) to t = 0.2."""
    p = P.sod_tube(100)
    st = I.sod_state(p)
    o = Oracle(p, st, 0.0)
    n = o.run(10 ** 9, 0.2)
    d = Disk(p)
    d.set_state(0.0, st)
    assert d.step_host(10 ** 9, 0.2) == n
    d.check()
    g, ref = d.get_state(), o.interior()
    d.close()
    assert d.t == pytest.approx(0.2, rel=1e-14)
    for k in ("r", "p", "u"):
        assert rel_l1(g[k], ref[k]) < 1e-12, k


def test_ragged_disk_fp32_tracks_fp64():
    """The FP32-mixed form (64 cells per axis at least) on the 70x206 disk
    against the FP64 oracle after 20 steps, at the bars of the 64x192 disk
    (density 2e-6 relative; the velocity residuals 1e-4 of their own L1 size)."""
    p = _disk(*RAGGED_2D[1])
    st = I.disk_state(p, seed=19)
    o = Oracle(p, st, T0)
    o.run(20)
    ref = o.interior()
    e = Ensemble([p])
    e.set_state(0, T0, st)
    e.run(20)
    e.sync()
    e.check()
    g = e.get_state(0)
    e.close()
    assert g["t"] == pytest.approx(o.t, rel=1e-6)
    assert rel_l1(g["r"], ref["r"]) < 2e-6
    for k in ("u", "v"):
        err = np.abs(g[k] - ref[k]).sum() / np.abs(ref[k] - st[k]).sum()
        assert err < 1e-4, (k, err)


def test_ragged_ensemble_members_equal_solo_runs_bitwise():
    """Members whose sizes share no tile multiple run in one launch per pass;
    each equals its own solo run bit for bit, with its own clock."""
    ps = [_disk(70, 206, planet_mass=1.0e-4), _disk(66, 130, ss_alpha=1.0e-2), _disk(98, 250, sc_h=0.07)]
    sts = [I.disk_state(p, seed=31 + k) for k, p in enumerate(ps)]
    e = Ensemble(ps)
    for k, st in enumerate(sts):
        e.set_state(k, T0, st)
    e.run(12)
    e.sync()
    e.check()
    for k, (p, st) in enumerate(zip(ps, sts)):
        solo = Ensemble([p])
        solo.set_state(0, T0, st)
        solo.run(12)
        solo.sync()
        a, b = e.get_state(k), solo.get_state(0)
        for key in ("r", "u", "v"):
            assert np.array_equal(a[key], b[key]), (k, key)
        assert e.clock(k) == solo.clock(0)
        solo.close()
    e.close()


def _dist3(a, b):
    out = {k: float(np.abs(a[k] - b[k]).sum() / np.abs(b[k]).sum()) for k in ("r", "p")}
    ma = [a["r"] * a[k] for k in "uvw"]
    mb = [b["r"] * b[k] for k in "uvw"]
    out["momentum"] = float(sum(np.abs(x - y).sum() for x, y in zip(ma, mb)) / sum(np.abs(y).sum() for y in mb))
    return out


def test_ragged_box_3d_matches_oracle():
    """26x22x14 cartesian box, 8 steps: the boxes of all three sweeps overhang
    the grid.  Uniform cells leave no room for operation-order differences
    beyond FMA contraction (the 32^3-class box cases agree to ~5e-16)."""
    p = P.cartesian_box(26, 22, 14)
    st = I.box_state(p, seed=9)
    d = Disk3(p)
    d.set_state(0.0, st)
    d.step_host(8)
    d.check()
    g = d.get_state()
    d.close()
    o = Oracle3(p, st, 0.0)
    o.run(8)
    e = _dist3(g, o.interior())
    o.close()
    assert all(v < 1e-13 for v in e.values()), e


def test_ragged_spherical_3d_matches_oracle_and_host_loop():
    """36x70x18 of the spherical preset, 3 steps, against the oracle at the
    64x128x32 case's bound (the oracle is the reference's arithmetic without
    FMA contraction); the device loop equals the host loop bit for bit."""
    p = P.spherical_disk(36, 70, 18)
    st = I.spherical_state(p, seed=23, vnoise=1.0e-3)
    a = Disk3(p)
    a.set_state(2.0 * np.pi, st)
    a.step_host(3)
    a.check()
    ga = a.get_state()
    a.close()
    b = Disk3(p)
    b.set_state(2.0 * np.pi, st)
    b.run(3)
    b.check()
    gb = b.get_state()
    b.close()
    for k in "rpuvw":
        assert np.array_equal(ga[k], gb[k]), k
    o = Oracle3(p, st, 2.0 * np.pi)
    o.run(3)
    e = _dist3(ga, o.interior())
    o.close()
    assert all(v < 3e-8 for v in e.values()), e
