"""Free-running parity of the wing configurations against the FP64 oracle
over many steps (tests/golden/free_run.npz, made by make_free_run.py).

Unlike the per-step tests, neither side is ever re-synchronised: the device
(FP32) and the FP64 oracle port (pinned bit for bit to the reference build)
each step the wing from rest with the benchmark's settings, and the device's
state after hundreds of steps is compared with the oracle's.  The oracle ran
on the definition permuted into the device sweep order; each case first
checks that the device still sweeps in that order.

Bounds (north star: after 600 steps the settled shape and the
constraint-violation norms agree within 1e-3 m):
  * SHAPE_TOL  largest node distance between the two shapes, each relative
               to its centre of mass (the wing falls freely, so its absolute
               position is a sum of 600 steps of gravity and damping);
  * NORM_TOL   the largest distance error and the largest cable extension,
               every step;
  * COM_TOL    the centre of mass, every step.
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

SHAPE_TOL = 1e-3
NORM_TOL = 1e-3
COM_TOL = 1e-3

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
    deviations from the FP64 run."""
    d = sw.generate_wing(**CASES[name])
    s = sw.Structure(d)
    orders = [s.sweep_order(abi.SWEEP_DISTANCE), s.sweep_order(abi.SWEEP_DIHEDRAL)]
    if d.view.membrane_count:
        orders.append(s.sweep_order(abi.SWEEP_MEMBRANE))
    assert order_hash(*orders) == str(golden[f"{name}_order_hash"]), "device sweep order changed: regenerate"
    steps = int(golden[f"{name}_steps"])
    ref = golden[f"{name}_diag"]
    st = step_settings()
    worst = {"shape": 0.0, "norms": 0.0, "com": 0.0, "strain": 0.0}
    for k in range(1, steps + 1):
        g = s.step(st)
        r = ref[k - 1]
        worst["norms"] = max(worst["norms"], abs(g.maximum_distance_error - r[0]),
                             abs(g.maximum_cable_extension - r[1]))
        com = np.array([g.center_of_mass.x, g.center_of_mass.y, g.center_of_mass.z])
        worst["com"] = max(worst["com"], float(np.abs(com - r[3:6]).max()))
        worst["strain"] = max(worst["strain"], abs(g.maximum_absolute_membrane_strain - r[2]))
        key = f"{name}_x{k}"
        if key in golden:
            worst["shape"] = max(worst["shape"],
                                 float(np.abs(centred(s.positions(), com) - centred(golden[key], r[3:6])).max()))
    s.close()
    return worst


@pytest.mark.parametrize("name", ["mid", "full"])
def test_free_running_wing_against_fp64(cuda_device, golden, name):
    worst = free_run(name, golden)
    assert worst["shape"] <= SHAPE_TOL, worst
    assert worst["norms"] <= NORM_TOL, worst
    assert worst["com"] <= COM_TOL, worst
