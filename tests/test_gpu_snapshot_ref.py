"""Snapshots and time averages against files the reference itself wrote.

* The reference's main.cu, relinked against the library (the drop-in check of
  test_dropin.py) writes its checkpoint and, with ave_flag, its time average
  through the reference's own write_check_point and averaging/add_grid
  (src/output/output.cu:125-180, 250-330; main.cu:343-351, 397-422).  The
  library's writer, given the same steps from the same restart file, must write
  the same file names and sizes, the same faces bit for bit, and the same time
  and fields within the case's bound.  (main.cu fills the ghost cells with the
  reference's own init, evaluated with the device pow, the library with its
  tables, so the two runs agree to rounding, not bit for bit.)
* The unmodified reference run with ave_flag (golden case disk64_ave_n10) gives
  the time average over 10 steps; the library's average of the same run must
  match it within the case's CUDA bound.

Needs a B200 and the relinked executable (built where the reference sources
are, by __graft_entry__.build())."""
import glob
import os
import subprocess

import numpy as np
import pytest

import cases as C
from penguin_b200 import snapshot as S
from penguin_b200.disk import Disk
from penguin_b200.params import make_grid_np

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
KEYS = ("r", "p", "u", "v")


def _case():
    return C.ave_cases()[0]


def _dist(a, b):
    """relative L1 of density and pressure and of the momentum vector"""
    out = {k: float(np.abs(a[k] - b[k]).sum() / np.abs(b[k]).sum()) for k in ("r", "p")}
    ax, ay, bx, by = a["r"] * a["u"], a["r"] * a["v"], b["r"] * b["u"], b["r"] * b["v"]
    out["momentum"] = float((np.abs(ax - bx) + np.abs(ay - by)).sum() / (np.abs(bx) + np.abs(by)).sum())
    return out


def _restart_file(path, case, st):
    p = case["params"]
    xa, _ = make_grid_np(p.xmin, p.xmax, p.xres, 3, p.geomx, p.gridx)
    ya, _ = make_grid_np(p.ymin, p.ymax, p.yres, 3, p.geomy, p.gridy)
    S.write_snapshot(str(path), case["t0"], xa[3:3 + p.xres + 1], ya[3:3 + p.yres + 1], st, 2)


def _library_run(case, st):
    """main.cu's loop on the library's handle API with the time average on."""
    p = case["params"]
    d = Disk(p)
    d.set_state(case["t0"], st)
    d.set_average(case["ave_interval"])
    n = d.step_host(case["max_step"], case["end_time"])
    assert n == case["max_step"]
    return d


def test_snapshot_and_average_files_match_the_reference_writer(tmp_path):
    case = _case()
    exe = os.path.join(ROOT, "oracle", "_ref", case["name"], "dropin", "penguin")
    if not os.path.exists(exe):
        pytest.skip("relinked executable not available")
    p = case["params"]
    st = C.initial_state(case)
    ref_dir = tmp_path / "ref"
    ref_dir.mkdir()
    _restart_file(ref_dir / "init.bin", case, st)
    r = subprocess.run([exe, "init.bin", "0"], cwd=ref_dir, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    state_files = [f for f in glob.glob(str(ref_dir / "binary_*_00001")) if "_ave_" not in os.path.basename(f)]
    ave_files = glob.glob(str(ref_dir / "binary_*_ave_00001"))
    assert len(state_files) == 1 and len(ave_files) == 1, r.stdout

    d = _library_run(case, st)
    ours = tmp_path / "ours"
    ours.mkdir()
    name, ave_name = S.file_name(p, 1), S.file_name(p, 1, average=True)
    assert name == os.path.basename(state_files[0])
    assert ave_name == os.path.basename(ave_files[0])
    d.write_snapshot(str(ours / name))
    d.write_snapshot(str(ours / ave_name), average=True)
    d.close()
    tol = case["cuda_tol"]
    for mine, theirs in ((ours / name, state_files[0]), (ours / ave_name, ave_files[0])):
        assert os.path.getsize(mine) == os.path.getsize(theirs), (mine, theirs)
        a = S.read_snapshot(str(mine), p.xres, p.yres, p.ndim)
        b = S.read_snapshot(theirs, p.xres, p.yres, p.ndim)
        assert a["t"] == pytest.approx(b["t"], rel=1e-13)
        assert np.array_equal(a["xa"], b["xa"]) and np.array_equal(a["ya"], b["ya"])
        errs = _dist(a, b)
        assert all(v < tol for v in errs.values()), (os.path.basename(theirs), errs)


def test_time_average_matches_the_reference_run():
    case = _case()
    path = os.path.join(GOLDEN, case["name"] + ".npz")
    if not os.path.exists(path):
        pytest.skip("fixture missing")
    z = np.load(path)
    assert float(z["ave_interval"]) == case["ave_interval"]
    st = {k: z["init_" + k] for k in KEYS}
    d = _library_run(case, st)
    got = d.get_average()
    d.close()
    errs = _dist(got, {k: z["ave_" + k] for k in KEYS})
    print("time average vs the reference's:", errs)
    assert all(v < case["cuda_tol"] for v in errs.values()), errs
