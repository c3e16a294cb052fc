"""Snapshots in the reference's checkpoint format, restarts, time averages
(ave_flag) and main.cu's dump semantics on the device loop.  Needs a B200."""
import numpy as np
import pytest

import cases as C
from penguin_b200 import initial as I
from penguin_b200 import params as P
from penguin_b200 import snapshot as S
from penguin_b200.disk import Disk, make_grid

pytestmark = pytest.mark.gpu
KEYS = ("r", "p", "u", "v")


def disk_case():
    c = [c for c in C.cases() if c["name"] == "disk64_n10"][0]
    return c["params"], C.initial_state(c), c["t0"]


def test_snapshot_matches_state_and_grid(tmp_path):
    p, st, t0 = disk_case()
    d = Disk(p)
    d.set_state(t0, st)
    d.run(5)
    d.sync()
    path = tmp_path / S.file_name(p, 1)
    d.write_snapshot(str(path))
    g = S.read_snapshot(str(path), p.xres, p.yres, p.ndim)
    s = d.get_state()
    assert g["t"] == d.clock()[0]
    xa, _, ya, _ = make_grid(p)
    assert np.array_equal(g["xa"], xa[3:3 + p.xres + 1]) and np.array_equal(g["ya"], ya[3:3 + p.yres + 1])
    for k in KEYS:
        assert np.array_equal(g[k], s[k]), k


def test_restart_from_snapshot_equals_restart_from_arrays(tmp_path):
    p, st, t0 = disk_case()
    a = Disk(p)
    a.set_state(t0, st)
    a.run(5)
    a.sync()
    path = tmp_path / "ck"
    a.write_snapshot(str(path))
    mid = a.get_state()
    b = Disk(p)
    t = b.read_snapshot(str(path))
    c = Disk(p)
    c.set_state(mid["t"], {k: mid[k] for k in KEYS})
    assert t == mid["t"]
    for x in (b, c):
        x.run(5)
        x.sync()
    gb, gc = b.get_state(), c.get_state()
    for k in KEYS:
        assert np.array_equal(gb[k], gc[k]), k


def test_dust_snapshot_holds_the_dust(tmp_path):
    p = P.reference_disk(64, 192, q=3.0e-4, alpha=1.0e-4).replace(dust_flag=1, Stokes=0.1, D_G_ratio=0.01)
    d = Disk(p)
    d.set_state(0.0, I.disk_state(p, seed=2))
    d.run(3)
    d.sync()
    path = tmp_path / "dust"
    d.write_snapshot(str(path))
    g = S.read_snapshot(str(path), p.xres, p.yres, p.ndim, dust=True)
    du = d.get_dust()
    assert np.array_equal(g["dust_r"], du["r"]) and np.array_equal(g["dust_u"], du["u"])
    assert np.array_equal(g["dust_v"], du["v"]) and np.all(g["dust_w"] == 0.0)


def test_time_average_is_the_trapezoid_of_main_loop(tmp_path):
    """averaging(dev, dt/2, T) before and after every solve (main.cu:343-351):
    A = sum over steps of (C_n + C_n+1) dt / (2 T), accumulated inside the step."""
    p, st, t0 = disk_case()
    T = 0.37
    d = Disk(p)
    d.set_state(t0, st)
    d.set_average(T)
    acc = {k: np.zeros((p.yres, p.xres)) for k in KEYS}
    prev = d.get_state()
    for _ in range(6):
        d.step_host(1)
        fac = (0.5 * d.dt) / T
        cur = d.get_state()
        for k in KEYS:
            acc[k] += prev[k] * fac
            acc[k] += cur[k] * fac
        prev = cur
    got = d.get_average()
    # the device accumulates with fused multiply-adds: one rounding per step
    # and field against the host's two, measured against the field's scale
    for k in KEYS:
        assert np.abs(got[k] - acc[k]).max() <= 1e-14 * np.abs(acc[k]).max(), k
    path = tmp_path / "ave"
    d.write_snapshot(str(path), average=True)
    g = S.read_snapshot(str(path), p.xres, p.yres, p.ndim)
    for k in KEYS:
        assert np.array_equal(g[k], got[k]), k
    d.reset_average()
    assert np.all(d.get_average()["r"] == 0.0)


def test_device_loop_dumps_like_main_loop():
    """run(.., t1) then run(.., t2) equals main.cu's loop with a dump at t1: the
    step clipped to the save time, then dt = old_dt (main.cu:333-338, 425)."""
    p = P.reference_disk(64, 192)
    st = I.disk_state(p, seed=4)
    t1, t2 = 0.3, 0.5
    a = Disk(p)
    a.set_state(0.0, st)
    a.run(10 ** 6, t1)
    a.run(10 ** 6, t2)
    a.sync()
    b = Disk(p)
    b.set_state(0.0, st)
    t, sav, dt = 0.0, 0.0, t1 - 0.0
    while True:
        dt = b.global_dt(dt)
        save, last = False, False
        if t + dt > t2:
            dt, last = t2 - t, True
        elif sav + dt > t1:
            old, dt, save = dt, t1 - sav, True
        b.solve(t, dt)
        t += dt
        sav += dt
        if last:
            break
        if save:
            sav, dt = 0.0, old
    assert a.clock()[0] == t
    ga, gb = a.get_state(), b.get_state()
    for k in KEYS:
        assert np.array_equal(ga[k], gb[k]), k
