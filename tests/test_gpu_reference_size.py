"""Parity with the unmodified reference at the workloads' own sizes.

The reference (built for sm_100a by oracle/ref_build.py for every case of
cases.size_cases) runs from a restart file written here, on the same GPU, and
its output snapshot is compared with the CUDA path stepped the same steps from
the same state: relative L1 of density, pressure and the momentum vector after
the case's step count.  The outputs (100 MB and more) are made at test time.

The bar is 1e-12 relative L1.  Printed beside it for the record: the
reference's own sensitivity floor, measured here by running it again from the
same restart file with every density moved by one ulp (as make_golden.py's
floor phase does for the golden cases), and the oracle's distance from the same
reference output.  The remaining CUDA difference grows across the azimuth like
(phi / dphi)^2: it is the rounding of the reference's per-call slope algebra
(src/solver/recon/recon.cu:216-378), whose grid moments cancel more at larger
phi.  Needs a B200 and the reference binaries."""
import glob
import os
import subprocess

import numpy as np
import pytest

import cases as C
from make_golden import perturb_ulp
from oracle.oracle import Oracle
from penguin_b200 import snapshot as S
from penguin_b200.disk import Disk
from penguin_b200.params import make_grid_np

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _dist(a, b):
    out = {k: float(np.abs(a[k] - b[k]).sum() / np.abs(b[k]).sum()) for k in ("r", "p")}
    ax, ay, bx, by = a["r"] * a["u"], a["r"] * a["v"], b["r"] * b["u"], b["r"] * b["v"]
    out["momentum"] = float((np.abs(ax - bx) + np.abs(ay - by)).sum() / (np.abs(bx) + np.abs(by)).sum())
    return out


def _reference(case, st, tmp_path, tag=""):
    exe = os.path.join(ROOT, "oracle", "_ref", case["name"], "penguin")
    if not os.path.exists(exe):
        pytest.skip("reference binary not built")
    p = case["params"]
    xa, _ = make_grid_np(p.xmin, p.xmax, p.xres, 3, p.geomx, p.gridx)
    ya, _ = make_grid_np(p.ymin, p.ymax, p.yres, 3, p.geomy, p.gridy)
    run_dir = tmp_path / ("ref" + tag)
    run_dir.mkdir()
    S.write_snapshot(str(run_dir / "init.bin"), case["t0"], xa[3:3 + p.xres + 1], ya[3:3 + p.yres + 1], st, 2)
    r = subprocess.run([exe, "init.bin", "0"], cwd=run_dir, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    out = [f for f in glob.glob(str(run_dir / "binary_*_00001")) if "_ave_" not in os.path.basename(f)]
    assert len(out) == 1, r.stdout[-2000:]
    res = S.read_snapshot(out[0], p.xres, p.yres, 2)
    os.remove(out[0])
    return res


@pytest.mark.parametrize("case", C.size_cases(), ids=lambda c: c["name"])
def test_cuda_matches_reference_at_workload_size(case, tmp_path):
    p = case["params"]
    st = C.initial_state(case)
    ref = _reference(case, st, tmp_path)
    floor = _dist(_reference(case, perturb_ulp(st), tmp_path, ".ulp"), ref)
    d = Disk(p)
    d.set_state(case["t0"], st)
    n = d.step_host(case["max_step"], case["end_time"])
    assert n == case["max_step"]
    g = d.get_state()
    d.close()
    e = _dist(g, ref)
    o = Oracle(p, st, case["t0"])
    o.run(case["max_step"], case["end_time"])
    eo = _dist(o.interior(), ref)
    o.close()
    print(f"{case['name']}: CUDA vs reference " + ", ".join(f"{k} {v:.2e}" for k, v in e.items()) +
          " | reference 1-ulp floor " + ", ".join(f"{k} {v:.2e}" for k, v in floor.items()) +
          " | oracle vs reference " + ", ".join(f"{k} {v:.2e}" for k, v in eo.items()))
    assert d.t == pytest.approx(float(ref["t"]), rel=1e-13)
    assert all(v < case["cuda_tol"] for v in e.values()), (e, floor)
