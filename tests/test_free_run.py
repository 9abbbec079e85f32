"""Free-running parity of the wing configurations against the FP64 oracle
over many steps (tests/golden/free_run.npz, made by make_free_run.py).

Unlike the per-step tests, neither side is ever re-synchronised: the device
(FP32) and the FP64 oracle port (pinned bit for bit to the reference build)
each step the wing from rest with the benchmark's settings, and the device's
state after hundreds of steps is compared with the oracle's.  The oracle ran
on the definition permuted into the device sweep order; each case first
checks that the device still sweeps in that order.

Bounds.  The north star asks that after 600 steps the settled shape and the
constraint-violation norms agree within 1e-3 m.  How far a free run can
agree is limited by the configuration itself: the fixture holds a second
FP64 run started from positions moved by N(0, 1e-7 m), about the rounding
of an FP32 coordinate of a metre.  On the mid-size wing that run stays
within 4e-6 m of the first over 600 steps, and the device must meet 1e-3 m.
On the full wing the suspension cascade amplifies it to centimetres (the
line particles and, through them, the canopy: about 2 cm at 600 steps)
although both runs are FP64, so no solver that does not reproduce the FP64
run bit for bit can meet 1e-3 m there; the device is bounded by four times
that measured sensitivity instead.  Compared, each relative to its centre
of mass (the wing falls freely): the shape of the fabric nodes and of the
line nodes at the stored steps; every step, the largest distance error and
the largest cable extension, and the centre of mass.  The membrane-element
wing runs 25 steps (the benchmark's membrane leg) and must also match the
largest membrane strain to 1e-3 of its value.
"""
import hashlib
import os

import numpy as np
import pytest

import simwing_b200 as sw
from simwing_b200 import abi
from tests.conftest import step_settings

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIXTURE = os.path.join(ROOT, "tests", "golden", "free_run.npz")

TOL = 1e-3           # metres, the north star's bound
SENSITIVITY_FACTOR = 4.0
STRAIN_TOL = 1e-3    # relative

CASES = {
    "mid": {"cells": 8, "chordwise": 20, "spanwise_per_cell": 2, "rib_layers": 3},
    "full": {},
    "fabric": {"fabric": 1},
}


def order_hash(*orders):
    h = hashlib.sha256()
    for o in orders:
        h.update(np.ascontiguousarray(o, dtype=np.uint64).tobytes())
    return h.hexdigest()


def centred(x, com):
    return np.asarray(x, dtype=np.float64) - np.asarray(com, dtype=np.float64)[None, :]


@pytest.fixture(scope="module")
def golden():
    return np.load(FIXTURE)


def free_run(name, golden):
    """Steps the device like the fixture's case; returns the largest
    deviations from the FP64 run (shape of the fabric and of the line nodes
    per stored step, norms, centre of mass, membrane strain)."""
    d = sw.generate_wing(**CASES[name])
    s = sw.Structure(d)
    orders = [s.sweep_order(abi.SWEEP_DISTANCE), s.sweep_order(abi.SWEEP_DIHEDRAL)]
    if d.view.membrane_count:
        orders.append(s.sweep_order(abi.SWEEP_MEMBRANE))
    assert order_hash(*orders) == str(golden[f"{name}_order_hash"]), "device sweep order changed: regenerate"
    steps = int(golden[f"{name}_steps"])
    ref = golden[f"{name}_diag"]
    fabric = golden[f"{name}_fabric"]
    st = step_settings()
    worst = {"fabric": [], "lines": [], "norms": 0.0, "com": 0.0, "strain": 0.0}
    for k in range(1, steps + 1):
        g = s.step(st)
        r = ref[k - 1]
        worst["norms"] = max(worst["norms"], abs(g.maximum_distance_error - r[0]),
                             abs(g.maximum_cable_extension - r[1]))
        com = np.array([g.center_of_mass.x, g.center_of_mass.y, g.center_of_mass.z])
        worst["com"] = max(worst["com"], float(np.abs(com - r[3:6]).max()))
        if r[2] > 0.0:
            worst["strain"] = max(worst["strain"], abs(g.maximum_absolute_membrane_strain - r[2]) / r[2])
        key = f"{name}_x{k}"
        if key in golden:
            dev = np.abs(centred(s.positions(), com) - centred(golden[key], r[3:6])).max(axis=1)
            worst["fabric"].append(float(dev[fabric].max()))
            worst["lines"].append(float(dev[~fabric].max()) if (~fabric).any() else 0.0)
    s.close()
    return worst


def bound(golden, name, key):
    return np.maximum(TOL, SENSITIVITY_FACTOR * np.asarray(golden[f"{name}_sens_{key}"], dtype=np.float64))


@pytest.mark.parametrize("name", ["mid", "full", "fabric"])
def test_free_running_wing_against_fp64(cuda_device, golden, name):
    worst = free_run(name, golden)
    assert np.all(np.array(worst["fabric"]) <= bound(golden, name, "shape_fabric")), worst
    assert np.all(np.array(worst["lines"]) <= bound(golden, name, "shape_lines")), worst
    assert worst["norms"] <= bound(golden, name, "norms"), worst
    assert worst["com"] <= bound(golden, name, "com"), worst
    assert worst["strain"] <= STRAIN_TOL, worst


def test_mid_wing_meets_the_north_star_bound(golden):
    """The mid-size wing is not sensitive (its FP64 runs agree to far below
    1e-3 m), so the bounds above are the north star's own there."""
    for key in ("shape_fabric", "shape_lines", "norms", "com"):
        assert np.all(bound(golden, "mid", key) == TOL)
