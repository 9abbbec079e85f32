"""The device gradient of the adjoint calibration workload against its FP64
reference (tests/golden/calibration.npz, made by make_calibration.py).

The calibration wing (20 cells x 30 chordwise, 13,338 triangles, 266 line
rest lengths) starts from the fixture's settled state; the loss is the mean
squared distance of its fabric nodes, after a 240-step rollout with a
checkpoint every 16 steps, to the fixture's target.  The device's forward /
backward pair (swb_rollout_*) gives the gradient with respect to the
calibration parameters: each line's rest length, the scale of each
compliance class (distance, cable, dihedral), the riser rest lengths and
the pilot mass.  They are compared, each solver on its own trajectory, with
  * the FP64 reference gradient (oracle/libadjoint.so), per parameter class
    by relative norm, and
  * central finite differences (h = 1e-4) of the FP64 loss on a sample of
    the parameters.
"""
import hashlib
import os

import numpy as np
import pytest

import simwing_b200 as sw
from simwing_b200 import abi
from tests.conftest import step_settings
from tests.test_adjoint import calibration_parameters, relative

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIXTURE = os.path.join(ROOT, "tests", "golden", "calibration.npz")

CLASS_TOL = 1e-3
FD_TOL = 1e-3
LOSS_TOL = 1e-3


def order_hash(distance_order, dihedral_order):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(distance_order, dtype=np.uint64).tobytes())
    h.update(np.ascontiguousarray(dihedral_order, dtype=np.uint64).tobytes())
    return h.hexdigest()


@pytest.fixture(scope="module")
def calibration():
    """The device loss, gradient (calibration parameters) and the fixture."""
    f = np.load(FIXTURE)
    d = sw.generate_calibration_wing()
    s = sw.Structure(d)
    assert order_hash(s.sweep_order(abi.SWEEP_DISTANCE), s.sweep_order(abi.SWEEP_DIHEDRAL)) == \
        str(f["order_hash"]), "device sweep order changed: regenerate the fixture"
    s.write_node_states(f["state"])
    p = f["payload"]
    s.write_payload_state(p[0:3], p[3:7], p[7:10], p[10:13])
    weights = np.zeros(d.node_count)
    weights[d.triangles()["nodes"].astype(np.int64).ravel()] = 1.0
    r = sw.Rollout(s, int(f["steps"]), 16)
    loss = r.forward(step_settings(), f["target"], weights)
    grad = r.backward()
    final = r.final_positions()
    params = calibration_parameters(d, grad)
    r.close()
    s.close()
    return {"loss": loss, "params": params, "final": final, "fixture": f}


def test_calibration_loss_and_shape(cuda_device, calibration):
    f = calibration["fixture"]
    assert abs(calibration["loss"] - float(f["loss"])) <= LOSS_TOL * float(f["loss"])
    assert float(np.abs(calibration["final"] - f["final"]).max()) <= 1e-3


def test_calibration_gradient_against_fp64(cuda_device, calibration):
    f, mine = calibration["fixture"], calibration["params"]
    theirs = {"lines": f["grad_lines"], "compliance classes": f["grad_classes"],
              "riser rest": f["grad_riser_rest"], "pilot mass": np.atleast_1d(f["grad_pilot_mass"])}
    errors = {k: relative(mine[k], theirs[k]) for k in theirs}
    assert all(v <= CLASS_TOL for v in errors.values()), errors


def test_calibration_gradient_against_finite_differences(cuda_device, calibration):
    f, mine = calibration["fixture"], calibration["params"]
    got = []
    for kind, index in zip(f["fd_kind"], f["fd_index"]):
        key = {"line": "lines", "class": "compliance classes", "riser": "riser rest", "mass": "pilot mass"}[str(kind)]
        got.append(float(mine[key][int(index)]))
    got, fd = np.array(got), f["fd_value"]
    # per class of parameter, relative to the class's largest difference
    errors = {}
    for kind in set(str(k) for k in f["fd_kind"]):
        m = np.array([str(k) == kind for k in f["fd_kind"]])
        errors[kind] = float(np.abs(got[m] - fd[m]).max() / max(np.abs(fd[m]).max(), 1e-30))
    assert all(v <= FD_TOL for v in errors.values()), errors
