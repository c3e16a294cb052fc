"""Parity of the sm_100a CUDA path (through the C ABI) with the oracle and with
the reference's own outputs.  Needs a B200."""
import os

import numpy as np
import pytest

import cases as C
from exact_riemann import sample
from oracle.oracle import Oracle
from penguin_b200 import initial as I
from penguin_b200 import params as P
from penguin_b200._lib import PG_ERR_NAN, PGError
from penguin_b200.disk import Disk, sweep_variant

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# FP64 relative-L1 bars, per golden case ("tol" in tests/golden/cases.py) for
# density, pressure and momentum.  The CUDA kernels evaluate the reference's
# expressions in its order except the 4th-order PPM edge slopes, which use
# per-index linear weights computed once in extended precision (the reference
# re-derives them per call, with cancellation in its grid moments); FMA
# contraction is allowed in both.


def rel_l1(a, b):
    den = np.abs(b).sum()
    return np.abs(a - b).sum() / den if den > 0 else np.abs(a - b).sum()


def momentum_l1(a, b):
    ax, ay = a["r"] * a["u"], a["r"] * a.get("v", 0 * a["r"])
    bx, by = b["r"] * b["u"], b["r"] * b.get("v", 0 * b["r"])
    return (np.abs(ax - bx) + np.abs(ay - by)).sum() / (np.abs(bx) + np.abs(by)).sum()


def _check(got, ref, p, tol):
    if p.ndim == 1:
        got = dict(got, v=0 * got["r"])
        ref = dict(ref, v=0 * ref["r"])
    errs = {k: rel_l1(got[k], ref[k]) for k in ("r", "p")}
    errs["momentum"] = momentum_l1(got, ref)
    assert all(e < tol for e in errs.values()), errs


def _keys(p):
    return ["r", "p", "u"] + (["v"] if p.ndim > 1 else [])


@pytest.mark.parametrize("case", C.cases(), ids=lambda c: c["name"])
def test_cuda_matches_oracle(case):
    p = case["params"]
    st = C.initial_state(case)
    o = Oracle(p, st, case["t0"])
    n = o.run(case["max_step"], case["end_time"])
    d = Disk(p)
    d.set_state(case["t0"], st)
    nh = d.step_host(case["max_step"], case["end_time"])
    d.check()
    g = d.get_state()
    assert nh == n
    tol = max(case["tol"], case["cuda_tol"])
    assert d.t == pytest.approx(o.t, rel=max(1e-13, tol))
    _check(g, o.interior(), p, tol)


@pytest.mark.parametrize("case", C.cases(), ids=lambda c: c["name"])
def test_cuda_matches_reference_fixture(case):
    path = os.path.join(GOLDEN, case["name"] + ".npz")
    if not os.path.exists(path):
        pytest.skip("fixture missing")
    z = np.load(path)
    p = case["params"]
    st = {k: z["init_" + k] for k in _keys(p)}
    d = Disk(p)
    d.set_state(float(z["t0"]), st)
    d.step_host(int(z["max_step"]), float(z["end_time"]))
    g = d.get_state()
    assert d.t == pytest.approx(float(z["t"]), rel=max(1e-13, case["cuda_tol"]))
    _check(g, {k: z["out_" + k] for k in _keys(p)}, p, case["cuda_tol"])


@pytest.mark.parametrize("name", ["disk64_n50", "sod_t02"])
def test_device_loop_equals_host_loop(name):
    """The CUDA-graph loop with dt on the device reproduces main.cu's host loop bit for bit."""
    case = [c for c in C.cases() if c["name"] == name][0]
    p, st = case["params"], C.initial_state(case)
    a = Disk(p)
    a.set_state(case["t0"], st)
    a.step_host(case["max_step"], case["end_time"])
    b = Disk(p)
    b.set_state(case["t0"], st)
    b.run(case["max_step"], case["end_time"])
    b.sync()
    t, dt, n = b.clock()
    assert t == a.t
    ga, gb = a.get_state(), b.get_state()
    for k in _keys(p):
        assert np.array_equal(ga[k], gb[k]), k


def test_sod_exact_solution_gpu():
    p = P.sod_tube(1024)
    d = Disk(p)
    d.set_state(0.0, I.sod_state(p))
    d.run(10**6, 0.2)
    d.sync()
    t, _, n = d.clock()
    assert t == pytest.approx(0.2, abs=1e-15)
    g = d.get_state()
    x = I.cell_centres(p)
    ex = sample((1.0, 0.0, 1.0), (0.125, 0.0, 0.1), (x - 0.5) / 0.2)
    l1 = [np.abs(g[k][0] - ex[m]).mean() for m, k in enumerate(("r", "u", "p"))]
    assert l1[0] < 2.5e-3 and l1[1] < 5e-3 and l1[2] < 2e-3, l1


def test_mass_conserved_closed_box():
    """Cartesian box, reflecting x walls, periodic y, no sources: mass to round-off."""
    p = P.Params(ndim=2, xres=64, yres=96, geomx=0, geomy=0, gridx=0, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.5,
                 EOS_flag=0, sc_h=0.3, planet_radius=1.0, p_beta=0.0, CFL=0.4, bound_lft=2, bound_rgh=2,
                 init_flag=1, OrbAdv_flag=0, visc_flag=0, kill_flag=0, n_planet=0, planet_mass=0.0,
                 frame_omega=0.0, zmin=0.0, zmax=1.0)
    x = I.cell_centres(p)
    y = (np.arange(p.yres) + 0.5) * 1.5 / p.yres
    r = 1.0 + 0.3 * np.exp(-((x[None, :] - 0.4) ** 2 + (y[:, None] - 0.7) ** 2) / 0.01)
    st = {"r": r, "p": 0.09 * r, "u": 0.1 * np.sin(2 * np.pi * y)[:, None] + 0 * r, "v": 0.05 + 0 * r}
    d = Disk(p)
    d.set_state(0.0, st)
    d.run(200)
    d.sync()
    g = d.get_state()
    assert abs(g["r"].sum() / r.sum() - 1.0) < 1e-13
    # parity on a linear-amplitude blob at rest (acoustic waves only): the sheared
    # flow above drives shocks into the walls, where limiter branches amplify
    # rounding-level differences
    st = {"r": 1.0 + 1e-3 * (r - 1.0) / 0.3, "u": 0 * r, "v": 0 * r}
    st["p"] = 0.09 * st["r"]
    d = Disk(p)
    d.set_state(0.0, st)
    d.run(20)
    d.sync()
    g = d.get_state()
    o = Oracle(p, st, 0.0)
    o.run(20)
    ref = o.interior()
    assert rel_l1(g["r"], ref["r"]) < 1e-14 and rel_l1(g["p"], ref["p"]) < 1e-14
    # the acoustic momentum is ~1e-4 of rho*cs, so an ulp of the pressure
    # gradient is ~1e-12 of it: the momentum bound is relative to that small signal
    assert momentum_l1(g, ref) < 5e-11


def test_planet_follows_reference_orbit():
    case = [c for c in C.cases() if c["name"] == "disk64_n10"][0]
    p, st = case["params"], C.initial_state(case)
    d = Disk(p)
    d.set_state(case["t0"], st)
    d.step_host(10)
    o = Oracle(p, st, case["t0"])
    o.run(10)
    a, b = d.planet(), o.planet()
    for k in ("m", "x", "y", "vy", "rs"):
        assert a[k] == pytest.approx(b[k], rel=1e-14, abs=1e-15), k


def test_error_word_reports_nan():
    """A NaN density injected on the host is reported by the device error word."""
    p = P.reference_disk(32, 96)
    st = I.disk_state(p, seed=3)
    st["r"][10, 10] = np.nan
    d = Disk(p)
    d.set_state(0.0, st)
    d.solve(0.0, 1.0e-3)
    with pytest.raises(PGError) as e:
        d.check()
    assert e.value.status == PG_ERR_NAN


def test_bounded_wait_gives_up_and_leaves_the_context_usable():
    """A pass's wait on a tile copy that never lands (its barrier expects bytes
    that no copy delivers) gives up after its limit instead of hanging: the
    device error word reports PG_ERR_TIMEOUT, the CTA leaves through the
    timed-out path, and the same context then steps a disk as before."""
    import ctypes

    from penguin_b200._lib import PG_ERR_TIMEOUT, check, lib

    p = P.reference_disk(32, 96)
    st = I.disk_state(p, seed=4)

    def five_steps():
        d = Disk(p)
        d.set_state(C.T0_DISK, st)
        d.run(5)
        d.sync()
        d.check()
        g = d.get_state()
        d.close()
        return g

    before = five_steps()
    err, left, ms = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_float(0.0)
    check(lib().pg_test_bounded_wait(ctypes.byref(err), ctypes.byref(left), ctypes.byref(ms)))
    assert err.value & (1 << PG_ERR_TIMEOUT), err.value
    assert left.value == 1
    assert 45.0 <= ms.value < 2000.0, ms.value  # 50 ms, then up to 50 ms more
    after = five_steps()
    for k in _keys(p):
        assert np.array_equal(before[k], after[k]), k


def test_drop_in_grid_entry_points_match_handle_api():
    """main.cu's loop on the pg_grid_* entry points (caller-owned buffers, C/T
    pointer swaps) gives the same state as the handle API."""
    from penguin_b200.grid import ReferenceLoop

    case = [c for c in C.cases() if c["name"] == "disk64_n10"][0]
    p, st = case["params"], C.initial_state(case)
    loop = ReferenceLoop(p, case["t0"], st)
    loop.step(10)
    g = loop.interior()
    d = Disk(p)
    d.set_state(case["t0"], st)
    d.step_host(10)
    h = d.get_state()
    loop.close()
    assert loop.t == d.t
    for k in _keys(p):
        assert np.array_equal(g[k], h[k]), k


def test_torque_matches_oracle():
    """Torque of the planet on the disk (src/output/output.cu:336-412) after 10 steps."""
    case = [c for c in C.cases() if c["name"] == "disk64_n10"][0]
    p = case["params"]
    st = C.initial_state(case)
    o = Oracle(p, st, case["t0"])
    o.run(10)
    d = Disk(p)
    d.set_state(case["t0"], st)
    d.step_host(10)
    d.check()
    # the state after 10 steps agrees to ~1e-12 (disk64_n10) and the sum is compensated
    assert d.torque() == pytest.approx(o.torque(), rel=1e-9)


def test_autotuned_launches_give_identical_results():
    """The autotuner changes tiles and grid sizes, not the arithmetic of a cell:
    the tuned step equals the default one bit for bit, and so does every tile
    variant it may choose (pencils per tile, pencil length, cells per thread,
    TMA stages), each with one CTA per SM."""
    case = [c for c in C.cases() if c["name"] == "disk64_n10"][0]
    p, st = case["params"], C.initial_state(case)
    ref = Disk(p)
    ref.set_state(case["t0"], st)
    ref.run(10)
    ref.sync()
    a = ref.get_state()
    tuned = Disk(p)
    tuned.set_state(case["t0"], st)
    choice = tuned.autotune(reps=3)
    assert set(choice) == set(Disk.TUNING) | {"passes"}
    assert set(choice["passes"]) == {"kick1", "sweep_x", "sweep_y", "advect", "kick2"}
    tuned.run(10)
    tuned.sync()
    b = tuned.get_state()
    for k in _keys(p):
        assert np.array_equal(a[k], b[k]), k
    for v in range(10):
        vx = v if sweep_variant(v)["pencil_length"] + 6 <= 51 else 0  # radial boxes of at most 256 doubles
        forced = Disk(p)
        forced.set_state(case["t0"], st)
        forced.set_tuning(dict(zip(Disk.TUNING, (vx, v, v, 1, 1, 1, 1, 1))))
        forced.run(10)
        forced.sync()
        c = forced.get_state()
        forced.close()
        for k in _keys(p):
            assert np.array_equal(a[k], c[k]), (v, k)


def test_state_exchange_round_trip_allocates_nothing():
    """set_state / get_state stage through a device buffer kept between calls:
    repeated exchanges leave free device memory unchanged and return the
    injected interior fields bit for bit."""
    import torch

    p = P.reference_disk(64, 192)
    st = I.disk_state(p, seed=3)
    d = Disk(p)
    d.set_state(0.0, st)
    d.get_state()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(5):
        d.set_state(0.0, st)
        out = d.get_state()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    for k in ("r", "p", "u", "v"):
        assert np.array_equal(out[k], st[k]), k
    d.close()


def test_division_by_1p5_is_the_ieee_quotient():
    """The kernels' division-free x / 1.5 (the PPM average's 1 - x/1.5) equals
    the correctly rounded quotient bit for bit: the swept fractions in [0, 1],
    their complements, random doubles of every magnitude and the edges."""
    import ctypes

    from penguin_b200._lib import check, lib

    rng = np.random.default_rng(5)
    q = rng.random(4_000_000)
    raw = rng.integers(0, 2 ** 63 - 1, size=2_000_000, dtype=np.int64).view(np.float64)
    raw = raw[np.isfinite(raw)]
    edge = np.array([0.0, -0.0, 1.0, 0.5, 1.5, 3.0, 2.0 ** -1074, 2.0 ** -1022, 1.0 - 2.0 ** -53, np.nextafter(1.0, 0),
                     1e-300, 1e300, 1.7976931348623157e308])
    x = np.ascontiguousarray(np.concatenate([q, 1.0 - q, raw, -raw[:1000], edge]))
    out = np.zeros(2 * x.size)
    dp = ctypes.POINTER(ctypes.c_double)
    check(lib().pg_test_div_1p5(x.ctypes.data_as(dp), x.size, out.ctypes.data_as(dp)))
    a, b = out[0::2], out[1::2]
    bad = ~((a == b) | (np.isnan(a) & np.isnan(b)))
    assert not bad.any(), (x[bad][:5], a[bad][:5], b[bad][:5])
    assert np.array_equal(np.signbit(a), np.signbit(b))
