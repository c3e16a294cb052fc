"""The CUDA bounds of the golden cases against the reference's own sensitivity.

floors.json (made by make_golden.py's floor phase on a B200) holds, per golden
case, how far the unmodified reference moves from itself when every input
density moves by one ulp, and whether a rerun reproduced the committed fixture
bit for bit.  Every bound above the 1e-12 bar must sit within 3x that floor, or, for
the 3D cases, within 5 % of the reference's distance from its own build
without FMA contraction ("fma_floor", make_golden.py's fmafloor phase): on the
3D preset's stretched grids the reference's result is defined only to that
operation-order level."""
import json
import os

import cases as C

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _floors():
    with open(os.path.join(HERE, "floors.json")) as f:
        return json.load(f)


def test_every_golden_case_has_a_measured_floor_and_a_deterministic_reference():
    fl = _floors()
    for c in C.cases() + C.dust_cases():
        assert c["name"] in fl, c["name"]
        assert fl[c["name"]]["deterministic"], c["name"]


def test_bounds_above_the_bar_sit_at_the_reference_floor():
    fl = _floors()
    for c in C.cases() + C.dust_cases():
        if c["cuda_tol"] > 1e-12:
            floor = max(fl[c["name"]]["floor"].values())
            assert c["cuda_tol"] <= 3.0 * floor, (c["name"], c["cuda_tol"], floor)
    for c in C.cases3d():
        if c["cuda_tol"] > 1e-12:
            fma = min(fl[c["name"]]["fma_floor"].values())
            assert c["cuda_tol"] <= 0.05 * fma, (c["name"], c["cuda_tol"], fma)
