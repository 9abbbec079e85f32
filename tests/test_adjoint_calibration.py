"""The device gradient of the adjoint calibration workload against its FP64
reference (tests/golden/calibration.npz, made by make_calibration.py).

The calibration wing (20 cells x 30 chordwise, 13,338 triangles, 266 line
rest lengths) starts from the fixture's settled state; the loss is the mean
squared distance of its fabric nodes, after a 240-step rollout with a
checkpoint every 16 steps, to the fixture's target.  The device's forward /
backward pair (swb_rollout_*) gives the gradient with respect to the
calibration parameters: each line's rest length, the scale of each
compliance class (distance, cable, dihedral), the riser rest lengths and
the pilot mass.

Three comparisons:
  * along the device trajectory (GPU): the FP64 reference gradient
    (oracle/libadjoint.so) restarted at every step from the device's state,
    so that both reverse sweeps see the same inputs and only the adjoint
    arithmetic differs: every parameter class within 1e-3 relative norm;
  * each solver on its own trajectory (GPU): the loss.  Over 240 steps FP32
    arithmetic of the reference algorithm itself moves the loss by a few
    per cent (the FP32 restatement's loss in the fixture: the line cables
    and the rigid pilot turn systematic rounding into a growing drift of
    the shape), so the device's loss is bounded by the larger of 1e-3 and
    three times that FP32 drift, relative to the FP64 loss;
  * the FP64 reference gradient against central differences of the FP64
    loss (CPU, from the fixture), each within 1e-3 of its parameter class's
    largest difference: the differences with h = 1e-6 for every sampled
    parameter, and those with h = 1e-4 for every sampled parameter at which
    the two steps agree within that.  Where they do not (two of the eight
    lines, the dihedral compliance class, both risers), a line cable
    crosses its slack/taut switch within +-1e-4 somewhere along the 240
    steps (the loss is piecewise smooth), and the wide difference is the
    mean slope across that switch, not a derivative; the list of those
    parameters is asserted too.
"""
import hashlib
import os

import numpy as np
import pytest

import simwing_b200 as sw
from simwing_b200 import abi
from oracle import oracle as O
from tests.conftest import step_settings
from tests.test_adjoint import calibration_parameters, payload_vector, relative, to_definition_order

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIXTURE = os.path.join(ROOT, "tests", "golden", "calibration.npz")

ALONG_TOL = 1e-3
FD_TOL = 1e-3
LOSS_TOL = 1e-3
F32_FACTOR = 3.0


def order_hash(distance_order, dihedral_order):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(distance_order, dtype=np.uint64).tobytes())
    h.update(np.ascontiguousarray(dihedral_order, dtype=np.uint64).tobytes())
    return h.hexdigest()


@pytest.fixture(scope="module")
def fixture():
    return np.load(FIXTURE)


@pytest.fixture(scope="module")
def calibration(fixture):
    """The device loss and gradient, the device trajectory and the FP64
    gradient along it."""
    f = fixture
    d = sw.generate_calibration_wing()
    s = sw.Structure(d)
    assert order_hash(s.sweep_order(abi.SWEEP_DISTANCE), s.sweep_order(abi.SWEEP_DIHEDRAL)) == \
        str(f["order_hash"]), "device sweep order changed: regenerate the fixture"
    s.write_node_states(f["state"])
    p = f["payload"]
    s.write_payload_state(p[0:3], p[3:7], p[7:10], p[10:13])
    state, pay = s.node_states(), payload_vector(s)
    weights = np.zeros(d.node_count)
    weights[d.triangles()["nodes"].astype(np.int64).ravel()] = 1.0
    steps, st = int(f["steps"]), step_settings()
    r = sw.Rollout(s, steps, 16)
    loss = r.forward(st, f["target"], weights)
    grad = r.backward()
    r.close()
    # the device trajectory, step by step (the same kernel and schedule)
    traj, tpay = [state], [pay]
    for _ in range(steps - 1):
        s.step(st, diagnostics=False)
        traj.append(s.node_states())
        tpay.append(payload_vector(s))
    along = O.rollout_gradient(s.oracle_definition(), st, steps, f["target"], weights, state=state, payload=pay,
                               trajectory=np.array(traj), trajectory_payloads=np.array(tpay))
    along["d_rest"] = to_definition_order(along["d_rest"], s.sweep_order(abi.SWEEP_DISTANCE))
    along["d_comp"] = to_definition_order(along["d_comp"], s.sweep_order(abi.SWEEP_DISTANCE))
    along["d_dihedral_comp"] = to_definition_order(along["d_dihedral_comp"], s.sweep_order(abi.SWEEP_DIHEDRAL))
    s.close()
    return {"loss": loss, "params": calibration_parameters(d, grad), "along": calibration_parameters(d, along)}


@pytest.mark.gpu
def test_calibration_gradient_along_the_device_trajectory(cuda_device, calibration):
    mine, theirs = calibration["params"], calibration["along"]
    errors = {k: relative(mine[k], theirs[k]) for k in theirs}
    assert all(v <= ALONG_TOL for v in errors.values()), errors


@pytest.mark.gpu
def test_calibration_loss_on_its_own_trajectory(cuda_device, calibration, fixture):
    f = fixture
    fp64, fp32 = float(f["loss"]), float(f["loss_f32"])
    bound = max(LOSS_TOL, F32_FACTOR * abs(fp32 - fp64) / fp64)
    assert abs(calibration["loss"] - fp64) / fp64 <= bound, (calibration["loss"], fp64, fp32)


def class_scales(f):
    """Each sampled parameter's class scale: the largest fine difference
    of its class."""
    kinds = [str(k) for k in f["fd_kind"]]
    return np.array([max(abs(float(f["fd_fine_value"][j])) for j in range(len(kinds)) if kinds[j] == kinds[i])
                     for i in range(len(kinds))])


def smooth_at_h(f):
    """Sampled parameters at which the loss is smooth within +-1e-4: the
    differences with h = 1e-4 and h = 1e-6 agree within 1e-3 of the class
    scale."""
    fd, fine, scale = f["fd_value"], f["fd_fine_value"], class_scales(f)
    return [i for i in range(len(fd)) if abs(fd[i] - fine[i]) <= FD_TOL * scale[i]]


def test_fp64_gradient_against_finite_differences(fixture):
    f = fixture
    theirs = {"line": f["grad_lines"], "class": f["grad_classes"], "riser": f["grad_riser_rest"],
              "mass": np.atleast_1d(f["grad_pilot_mass"])}
    kinds = [str(k) for k in f["fd_kind"]]
    smooth, scale = smooth_at_h(f), class_scales(f)
    for i in range(len(kinds)):
        got = float(theirs[kinds[i]][int(f["fd_index"][i])])
        assert abs(got - float(f["fd_fine_value"][i])) <= FD_TOL * scale[i], (kinds[i], int(f["fd_index"][i]), "h=1e-6")
        if i in smooth:
            assert abs(got - float(f["fd_value"][i])) <= FD_TOL * scale[i], (kinds[i], int(f["fd_index"][i]), "h=1e-4")
    # the parameters whose +-1e-4 stencil straddles a slack/taut switch
    kinked = sorted(f"{kinds[i]}{int(f['fd_index'][i])}" for i in range(len(kinds)) if i not in smooth)
    assert kinked == ["class2", "line0", "line151", "riser0", "riser1"], kinked
