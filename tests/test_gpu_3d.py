"""The 3D (ndim 3) CUDA path against the unmodified reference's own 3D runs
(fixtures in tests/golden), against the 3D oracle, its device loop against its
host loop, and mass conservation in a closed box.  Needs a B200."""
import glob
import os
import re
import subprocess

import numpy as np
import pytest

import cases as C
from oracle.oracle import Oracle3
from penguin_b200 import initial as I
from penguin_b200 import params as P
from penguin_b200 import snapshot as S
from penguin_b200.disk3 import Disk3

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def dist3(a, b):
    out = {k: float(np.abs(a[k] - b[k]).sum() / np.abs(b[k]).sum()) for k in ("r", "p")}
    ma = [a["r"] * a[k] for k in "uvw"]
    mb = [b["r"] * b[k] for k in "uvw"]
    out["momentum"] = float(sum(np.abs(x - y).sum() for x, y in zip(ma, mb)) / sum(np.abs(y).sum() for y in mb))
    return out


def _fmt(e):
    return ", ".join(f"{k} {v:.2e}" for k, v in e.items())


@pytest.mark.parametrize("case", C.cases3d(), ids=lambda c: c["name"])
def test_cuda_matches_reference_3d(case):
    path = os.path.join(GOLDEN, case["name"] + ".npz")
    if not os.path.exists(path):
        pytest.skip("fixture missing")
    z = np.load(path)
    st = C.initial_state(case)
    d = Disk3(case["params"])
    d.set_state(case["t0"], st)
    n = d.step_host(case["max_step"], case["end_time"])
    d.check()
    assert n == case["max_step"]
    g = d.get_state()
    d.close()
    ref = {k: z["out_" + k] for k in "rpuvw"}
    e = dist3(g, ref)
    o = Oracle3(case["params"], st, case["t0"])
    o.run(case["max_step"], case["end_time"])
    eo = dist3(g, o.interior())
    o.close()
    print(f"{case['name']}: CUDA vs reference {_fmt(e)} | CUDA vs oracle {_fmt(eo)}")
    assert g["t"] == pytest.approx(float(z["t"]), rel=1e-13)
    assert all(v < case["cuda_tol"] for v in e.values()), e


@pytest.mark.parametrize("case", C.cases3d(), ids=lambda c: c["name"])
def test_device_loop_equals_host_loop_3d(case):
    st = C.initial_state(case)
    a = Disk3(case["params"])
    a.set_state(case["t0"], st)
    a.step_host(5)
    b = Disk3(case["params"])
    b.set_state(case["t0"], st)
    b.run(5)
    b.check()
    t, dt, n = b.clock()
    assert n == 5
    ga, gb = a.get_state(), b.get_state()
    assert t == ga["t"]
    for k in "rpuvw":
        assert np.array_equal(ga[k], gb[k]), k
    a.close()
    b.close()


def test_closed_box_conserves_mass_3d():
    p = P.cartesian_box(32, 16, 16).replace(bound_lft=2, bound_rgh=2, bound_bom=2, bound_top=2)
    d = Disk3(p)
    st = I.box_state(p, seed=5)
    d.set_state(0.0, st)
    m0 = st["r"].sum()
    d.run(50)
    d.check()
    m1 = d.get_state()["r"].sum()
    d.close()
    assert abs(m1 - m0) < 1e-13 * m0


def test_cuda_matches_oracle_on_a_larger_spherical_disk():
    """64x128x32 of the spherical preset (4 tiles along the azimuth, two along
    the polar angle), 3 steps.  The oracle is the reference's arithmetic without
    FMA contraction, which on these grids moves the result by ~1e-9 (the
    fma_floor of tests/golden/cases.py, larger here where the cells are finer):
    the bound is that distance with margin (measured 4.9e-9 r, 8.2e-9 momentum)."""
    p = P.spherical_disk(64, 128, 32)
    st = I.spherical_state(p, seed=21, vnoise=1.0e-3)
    d = Disk3(p)
    d.set_state(2.0 * np.pi, st)
    d.step_host(3)
    d.check()
    g = d.get_state()
    d.close()
    o = Oracle3(p, st, 2.0 * np.pi)
    o.run(3)
    e = dist3(g, o.interior())
    o.close()
    print("64x128x32 after 3 steps, CUDA vs oracle:", _fmt(e))
    assert all(v < 3e-8 for v in e.values()), e


def _reference3(case, st, run_dir, build=""):
    """The reference binary of the case (build "" or "_nofma") from a restart file
    written here; returns its output fields and its seconds per step."""
    p = case["params"]
    exe = os.path.join(ROOT, "oracle", "_ref", case["name"] + build, "penguin")
    if not os.path.exists(exe):
        pytest.skip("reference binary not built")
    run_dir.mkdir()
    (xa, _), (ya, _), (za, _) = P.axes_np(p)
    S.write_snapshot(str(run_dir / "init.bin"), case["t0"], xa[3:3 + p.xres + 1], ya[3:3 + p.yres + 1], st, 3,
                     za=za[3:3 + p.zres + 1])
    r = subprocess.run([exe, "init.bin", "0"], cwd=run_dir, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    out = [f for f in glob.glob(str(run_dir / "binary_*_00001")) if "_ave_" not in os.path.basename(f)]
    assert len(out) == 1, r.stdout[-2000:]
    res = S.read_snapshot(out[0], p.xres, p.yres, 3, zres=p.zres)
    os.remove(out[0])
    os.remove(str(run_dir / "init.bin"))
    sps = re.findall(r"([0-9.eE+-]+) seconds per step", r.stdout)
    return res, float(sps[-1]) if sps else None


@pytest.mark.parametrize("case", C.size_cases3d(), ids=lambda c: c["name"])
def test_cuda_matches_reference_at_preset_size(case, tmp_path):
    """The 3D preset at its own size (384x768x216): the CUDA path against the
    unmodified reference and against the reference's own build without FMA
    contraction, from the same restart state; CUDA must sit well inside the
    reference's operation-order floor (5 % of it)."""
    p = case["params"]
    st = C.initial_state(case)
    ref, sps = _reference3(case, st, tmp_path / "ref")
    nofma, _ = _reference3(case, st, tmp_path / "nofma", "_nofma")
    floor = dist3(nofma, ref)
    d = Disk3(p)
    d.set_state(case["t0"], st)
    n = d.step_host(case["max_step"], case["end_time"])
    d.check()
    assert n == case["max_step"]
    g = d.get_state()
    d.close()
    e = dist3(g, ref)
    print(f"{case['name']}: CUDA vs reference {_fmt(e)} | reference -fmad=false vs reference {_fmt(floor)} | "
          f"reference {sps} s/step")
    assert g["t"] == pytest.approx(float(ref["t"]), rel=1e-13)
    assert all(e[k] < 0.05 * floor[k] for k in e), (e, floor)


def test_snapshot_round_trip_and_reference_reader_3d(tmp_path):
    """The library's 3D checkpoint has the reference's layout (penguin_b200.snapshot
    reads it with the faces of the grid) and restarts the same run bit for bit."""
    case = C.cases3d()[0]
    p = case["params"]
    d = Disk3(p)
    d.set_state(case["t0"], C.initial_state(case))
    d.run(3)
    d.check()
    path = tmp_path / "binary_3d_00001"
    d.write_snapshot(str(path))
    assert os.path.getsize(path) == 8 * (1 + p.xres + 1 + p.yres + 1 + p.zres + 1 + 5 * p.cells)
    f = S.read_snapshot(str(path), p.xres, p.yres, 3, zres=p.zres)
    g = d.get_state()
    (xa, _), (ya, _), (za, _) = P.axes_np(p)
    assert f["t"] == g["t"]
    assert np.array_equal(f["xa"], xa[3:3 + p.xres + 1]) and np.array_equal(f["za"], za[3:3 + p.zres + 1])
    for k in "rpuvw":
        assert np.array_equal(f[k], g[k]), k
    e = Disk3(p)
    assert e.read_snapshot(str(path)) == g["t"]
    h = Disk3(p)  # the same restart from the arrays
    h.set_state(g["t"], {k: g[k] for k in "rpuvw"})
    e.run(2)
    h.run(2)
    a, b = h.get_state(), e.get_state()
    for k in "rpuvw":
        assert np.array_equal(a[k], b[k]), k
    for x in (d, e, h):
        x.close()
