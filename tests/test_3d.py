"""The 3D (ndim 3) form on the CPU: the oracle against the unmodified
reference's own 3D runs (fixtures in tests/golden, made by make_golden.py on a
B200), against the 2D oracle on states that do not depend on one of the three
coordinates, and the grid the library builds.  CPU only."""
import os

import numpy as np
import pytest

import cases as C
from oracle.oracle import Oracle, Oracle3
from penguin_b200 import initial as I
from penguin_b200 import params as P

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def dist3(a, b):
    """relative L1 of density and pressure and of the momentum vector"""
    out = {k: float(np.abs(a[k] - b[k]).sum() / np.abs(b[k]).sum()) for k in ("r", "p")}
    ma = [a["r"] * a[k] for k in "uvw"]
    mb = [b["r"] * b[k] for k in "uvw"]
    out["momentum"] = float(sum(np.abs(x - y).sum() for x, y in zip(ma, mb)) / sum(np.abs(y).sum() for y in mb))
    return out


@pytest.mark.parametrize("case", C.cases3d(), ids=lambda c: c["name"])
def test_oracle_matches_reference_3d(case):
    path = os.path.join(GOLDEN, case["name"] + ".npz")
    if not os.path.exists(path):
        pytest.skip("fixture missing")
    z = np.load(path)
    o = Oracle3(case["params"], C.initial_state(case), case["t0"])
    n = o.run(case["max_step"], case["end_time"])
    assert n == case["max_step"]
    assert o.t == pytest.approx(float(z["t"]), rel=1e-13)
    e = dist3(o.interior(), {k: z["out_" + k] for k in "rpuvw"})
    o.close()
    print(case["name"], e)
    assert all(v < case["tol"] for v in e.values()), e


def test_3d_fixtures_have_a_measured_floor_and_a_deterministic_reference():
    import json

    with open(os.path.join(GOLDEN, "floors.json")) as f:
        fl = json.load(f)
    for c in C.cases3d():
        assert c["name"] in fl, c["name"]
        assert fl[c["name"]]["deterministic"], c["name"]
        assert max(fl[c["name"]]["floor"].values()) < 1e-14


def _box(nx, ny, nz, **kw):
    return P.cartesian_box(nx, ny, nz).replace(**kw)


def _state2d(p2, seed=11):
    """a 2D cartesian state (yres, xres) with every velocity component"""
    u = I.splitmix64_uniform(seed, 5 * p2.xres * p2.yres).reshape(5, p2.yres, p2.xres)
    return {"r": 1.0 + 0.2 * u[0], "p": 1.0 + 0.2 * u[1] + np.where(u[2] > 0.7, 1.0, 0.0),
            "u": 0.1 * u[2], "v": 0.1 * u[3], "w": 0.1 * u[4]}


def test_3d_oracle_reduces_to_2d_in_the_xy_plane():
    """A 3D box state that does not depend on z, with w = 0, evolves like the 2D
    oracle's (x, y) state: the polar sweep of a uniform pencil only moves the
    energy by the update's rounding, and a very deep box keeps the polar CFL
    term out of dt."""
    p3 = _box(16, 12, 6, zmin=0.0, zmax=1000.0, bound_bom=3, bound_top=3)
    p2 = P.Params(ndim=2, xres=16, yres=12, geomx=0, geomy=0, gridx=0, gridy=0, xmin=0.0, xmax=1.0, ymin=0.0,
                  ymax=1.0, EOS_flag=2, internal_e_flag=0, gam=1.4, CFL=0.4, bound_lft=2, bound_rgh=1, init_flag=4,
                  frame_omega=0.0, visc_flag=0, OrbAdv_flag=0, kill_flag=0, n_planet=1, planet_mass=0.0)
    s2 = _state2d(p2)
    s3 = {k: np.repeat(s2[k][None], p3.zres, axis=0) for k in "rpuv"}
    s3["w"] = np.zeros_like(s3["r"])
    o2 = Oracle(p2, {k: s2[k] for k in "rpuv"}, 0.0)
    o3 = Oracle3(p3, s3, 0.0)
    o2.run(8)
    o3.run(8)
    assert o3.t == pytest.approx(o2.t, rel=1e-14)
    a, b = o3.interior(), o2.interior()
    for k in "rpuv":
        assert np.abs(a[k] - b[k][None]).max() < 1e-13, k
    assert np.abs(a["w"]).max() == 0.0


def test_3d_oracle_reduces_to_2d_in_the_xz_plane():
    """A 3D box state that does not depend on y, with v = 0, evolves like the 2D
    oracle's state with z as its azimuth: the polar sweep is the 2D azimuthal
    sweep with the transverse velocities in the other slot, and periodic polar
    boundaries are the 2D azimuth's."""
    p3 = _box(16, 6, 12, ymin=0.0, ymax=1000.0, bound_bom=3, bound_top=3)
    p2 = P.Params(ndim=2, xres=16, yres=12, geomx=0, geomy=0, gridx=0, gridy=0, xmin=0.0, xmax=1.0, ymin=0.0,
                  ymax=1.0, EOS_flag=2, internal_e_flag=0, gam=1.4, CFL=0.4, bound_lft=2, bound_rgh=1, init_flag=4,
                  frame_omega=0.0, visc_flag=0, OrbAdv_flag=0, kill_flag=0, n_planet=1, planet_mass=0.0)
    s2 = _state2d(p2, seed=12)
    # 3D (r, p, u, w) on (z, x) <- 2D (r, p, u, v) on (y, x)
    s3 = {"r": s2["r"], "p": s2["p"], "u": s2["u"], "w": s2["v"]}
    s3 = {k: np.repeat(v[:, None, :], p3.yres, axis=1) for k, v in s3.items()}
    s3["v"] = np.zeros_like(s3["r"])
    o2 = Oracle(p2, {k: s2[k] for k in "rpuv"}, 0.0)
    o3 = Oracle3(p3, s3, 0.0)
    o2.run(8)
    o3.run(8)
    assert o3.t == pytest.approx(o2.t, rel=1e-14)
    a, b = o3.interior(), o2.interior()
    for k3, k2 in (("r", "r"), ("p", "p"), ("u", "u"), ("w", "v")):
        assert np.abs(a[k3] - b[k2][:, None, :]).max() < 1e-13, k3
    assert np.abs(a["v"]).max() == 0.0


def test_3d_closed_box_conserves_mass():
    """Reflecting walls on both radial ends and both polar ends, periodic y: the
    oracle keeps the total mass to round-off."""
    p = _box(16, 8, 8, bound_lft=2, bound_rgh=2, bound_bom=2, bound_top=2)
    s = I.box_state(p, seed=3)
    o = Oracle3(p, s, 0.0)
    m0 = o.interior()["r"].sum()
    o.run(20)
    assert abs(o.interior()["r"].sum() - m0) < 1e-13 * m0


@pytest.mark.parametrize("make", [lambda: P.spherical_disk(32, 64, 16), lambda: P.spherical_disk(),
                                  lambda: P.cartesian_box(24, 20, 10)], ids=["sph32", "preset", "box"])
def test_library_grid_is_the_oracles_bit_for_bit(make):
    from penguin_b200.disk3 import make_axis

    p = make()
    o = Oracle3(p)
    for axis in range(3):
        a, v = make_axis(p, axis)
        oa, ov = o.axis(axis)
        assert np.array_equal(a, oa) and np.array_equal(v, ov), axis
        pa, pv = P.axes_np(p)[axis]
        assert np.array_equal(a, pa), axis
        assert np.allclose(v, pv, rtol=1e-14, atol=0), axis
    o.close()


def test_3d_parameters_outside_the_form_are_rejected():
    import ctypes

    from penguin_b200._lib import PG_ERR_CONFIG, lib

    bad = [
        P.spherical_disk(32, 64, 16).replace(visc_flag=1),
        P.spherical_disk(32, 64, 16).replace(OrbAdv_flag=1),
        P.spherical_disk(32, 64, 16).replace(geomz=0),
        P.cartesian_box(16, 16, 8).replace(bound_lft=0),  # analytic ghosts need the spherical disk state
        P.cartesian_box(15, 16, 8),                        # odd xres: 16-byte rows for TMA
    ]
    for p in bad:
        with pytest.raises(ValueError):
            p.validate()
        PP = P.PGParams(*[getattr(P.PGParams.from_params(P.cartesian_box()), f) for f, _ in P.PGParams._fields_])
        for f, _ in P.PGParams._fields_:
            setattr(PP, f, getattr(p, {"eos_flag": "EOS_flag", "cfl": "CFL", "orbadv_flag": "OrbAdv_flag",
                                       "stokes": "Stokes", "d_g_ratio": "D_G_ratio"}.get(f, f)))
        h = ctypes.c_void_p()
        assert lib().pg_disk3_create(ctypes.byref(PP), 0, None, ctypes.byref(h)) == PG_ERR_CONFIG
    with pytest.raises(ValueError):
        P.spherical_disk(16, 32, 16).validate()  # the preset's stretched radial grid needs 20+ cells
