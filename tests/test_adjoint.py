"""Device adjoint (swb_rollout_*): the gradient of a rollout loss computed
by the reverse cluster sweep in FP32, checked against the FP64 reference
gradient (oracle/xpbd_adjoint.cpp, itself pinned to central finite
differences in test_adjoint_oracle.py) on the same discrete step: the oracle
runs the definition permuted into the device sweep order, from the device's
state.

Two comparisons:
  * along the device trajectory -- the oracle restarts every step from the
    device's state, so both reverse sweeps see the same inputs and only the
    adjoint arithmetic is compared: the calibration parameters (below)
    within 1e-3, and element by element every constraint's rest length (seam
    stitches excepted: their rest length is fixed at zero and their two nodes
    coincide, so the direction is undefined) and compliance, every dihedral's
    compliance, the riser rest lengths and the pilot mass, each class within
    1e-3 relative norm -- cables within 3e-3: inside a step the FP32 and FP64
    iterations can leave a cable that sits at its slack/taut switch on
    different sides, which moves that cable's own entries;
  * each solver on its own trajectory -- the calibration parameters (line
    rest lengths, the three compliance classes, riser rest lengths, pilot
    mass) within 5e-3: the FP32 and FP64 trajectories drift apart over the
    rollout (the loss agrees to 1e-3), which moves the gradient by more than
    the adjoint arithmetic does."""
import numpy as np
import pytest

import simwing_b200 as sw
from simwing_b200 import abi
from oracle import oracle as O
from tests.conftest import step_settings

pytestmark = pytest.mark.gpu

ALONG_TOL = 1e-3
ALONG_CABLE_TOL = 3e-3
OWN_TOL = 5e-3
LOSS_TOL = 1e-3


def payload_vector(structure):
    s = structure.suspension_state()
    if s is None:
        return None
    return np.concatenate([s.center_of_mass, s.body_to_world, s.linear_velocity, s.angular_velocity])


def to_definition_order(values, order):
    out = np.zeros_like(values)
    out[order] = values
    return out


def relative(got, want):
    scale = np.linalg.norm(want)
    return float(np.linalg.norm(got - want) / scale) if scale > 0 else float(np.linalg.norm(got))


def calibration_case(definition, settle, steps, interval, seed=1):
    """Device gradient and FP64 references (own trajectory and along the
    device trajectory) of a rollout from a settled state."""
    st = step_settings()
    structure = sw.Structure(definition)
    for _ in range(settle):
        structure.step(st, diagnostics=False)
    n = structure.node_count
    rng = np.random.default_rng(seed)
    state = structure.node_states()
    pay = payload_vector(structure)
    target = state[:, 0, :] + rng.normal(0.0, 0.02, (n, 3))
    weights = np.zeros(n)
    weights[definition.triangles()["nodes"].astype(np.int64).ravel()] = 1.0
    rollout = sw.Rollout(structure, steps, interval)
    loss = rollout.forward(st, target, weights)
    grad = rollout.backward()
    grad["loss"] = loss
    final = rollout.final_positions()
    # the device trajectory, step by step (the same kernel and schedule)
    traj, tpay = [state], [pay]
    for _ in range(steps - 1):
        structure.step(st, diagnostics=False)
        traj.append(structure.node_states())
        tpay.append(payload_vector(structure))
    dist_order = structure.sweep_order(abi.SWEEP_DISTANCE)
    dih_order = structure.sweep_order(abi.SWEEP_DIHEDRAL)
    od = structure.oracle_definition()
    refs = {}
    for tag, extra in (("own", {}), ("along", {"trajectory": np.array(traj),
                                              "trajectory_payloads": None if pay is None else np.array(tpay)})):
        ref = O.rollout_gradient(od, st, steps, target, weights, state=state, payload=pay, **extra)
        ref["d_rest"] = to_definition_order(ref["d_rest"], dist_order)
        ref["d_comp"] = to_definition_order(ref["d_comp"], dist_order)
        ref["d_dihedral_comp"] = to_definition_order(ref["d_dihedral_comp"], dih_order)
        refs[tag] = ref
    return grad, refs, final


def per_constraint_errors(definition, grad, ref):
    kinds = definition.constraints()["kind"]
    comp0 = definition.constraints()["compliance"]
    h0 = definition.dihedrals()["compliance"]
    checks = {}
    for name, mask in (("distance rest", (kinds == abi.DISTANCE) | (kinds == abi.SUSPENSION_TIE)),
                       ("cable rest", kinds == abi.CABLE)):
        if mask.any():
            checks[name] = relative(grad["d_rest"][mask], ref["d_rest"][mask])
    for name, mask in (("distance compliance", (kinds == abi.DISTANCE) | (kinds == abi.SUSPENSION_TIE)),
                       ("cable compliance", kinds == abi.CABLE)):
        if mask.any():
            checks[name] = relative(grad["d_comp"][mask] * comp0[mask], ref["d_comp"][mask] * comp0[mask])
    checks["dihedral compliance"] = relative(grad["d_dihedral_comp"] * h0, ref["d_dihedral_comp"] * h0)
    if definition.has_suspension:
        checks["riser rest"] = relative(grad["d_segment_rest"], ref["d_segment_rest"])
        checks["pilot mass"] = relative(np.array([grad["d_mass"]]), np.array([ref["d_mass"]]))
    return checks


def calibration_parameters(definition, grad):
    """Gradient with respect to the calibration's parameters: each line's
    rest length (its cables scaled together), the scale of each compliance
    class (distance, cable, dihedral), the riser rest lengths and the pilot
    mass."""
    cons = definition.constraints()
    kinds, rest0, comp0 = cons["kind"], cons["rest_length"], cons["compliance"]
    lines = [np.sum(grad["d_rest"][g] * rest0[g]) / np.sum(rest0[g]) for g in sw.line_groups(definition)]
    classes = [np.sum((grad["d_comp"] * comp0)[(kinds == abi.DISTANCE) | (kinds == abi.SUSPENSION_TIE)]),
               np.sum((grad["d_comp"] * comp0)[kinds == abi.CABLE]),
               np.sum(grad["d_dihedral_comp"] * definition.dihedrals()["compliance"])]
    out = {"lines": np.array(lines), "compliance classes": np.array(classes)}
    if definition.has_suspension:
        out["riser rest"] = grad["d_segment_rest"]
        out["pilot mass"] = np.array([grad["d_mass"]])
    return out


def check_case(definition, settle, steps, interval):
    grad, refs, final = calibration_case(definition, settle, steps, interval)
    along = per_constraint_errors(definition, grad, refs["along"])
    bad = {k: v for k, v in along.items() if not v <= (ALONG_CABLE_TOL if k.startswith("cable") else ALONG_TOL)}
    assert not bad, ("along the device trajectory", along)
    mine, theirs = calibration_parameters(definition, grad), calibration_parameters(definition, refs["along"])
    along_params = {k: relative(mine[k], theirs[k]) for k in mine}
    bad = {k: v for k, v in along_params.items() if not v <= ALONG_TOL}
    assert not bad, ("calibration parameters along the device trajectory", along_params)
    theirs = calibration_parameters(definition, refs["own"])
    own = {k: relative(mine[k], theirs[k]) for k in mine}
    own["loss"] = abs(grad["loss"] - refs["own"]["loss"]) / abs(refs["own"]["loss"])
    bad = {k: v for k, v in own.items() if not v <= (LOSS_TOL if k == "loss" else OWN_TOL)}
    assert not bad, ("own trajectories", own)
    return final, refs


def test_patch_gradient_matches_fp64_reference(cuda_device):
    d = sw.generate_patch(nx=17, ny=17, seed=2)
    final, refs = check_case(d, settle=30, steps=20, interval=8)
    np.testing.assert_allclose(final, refs["own"]["final"], rtol=0, atol=1e-4)


def test_wing_with_pilot_gradient_matches_fp64_reference(cuda_device):
    d = sw.generate_wing(cells=4, chordwise=10, spanwise_per_cell=2, rib_layers=2, seed=3)
    check_case(d, settle=40, steps=48, interval=16)


def test_rollout_leaves_the_structure_untouched_and_replays(cuda_device):
    d = sw.generate_patch(nx=12, ny=12, seed=4)
    st = step_settings()
    s = sw.Structure(d)
    s.step(st, diagnostics=False)
    before = s.node_states()
    n = s.node_count
    r = sw.Rollout(s, 5, 2)
    target = before[:, 0, :]
    w = np.ones(n)
    l1 = r.forward(st, target, w)
    g1 = r.backward()
    l2 = r.forward(st, target, w)
    g2 = r.backward()
    assert l1 == l2
    np.testing.assert_array_equal(g1["d_rest"], g2["d_rest"])
    np.testing.assert_array_equal(s.node_states(), before)
    assert s.accepted_step_count() == 1
    for _ in range(5):
        s.step(st, diagnostics=False)
    np.testing.assert_allclose(s.positions(), r.final_positions(), rtol=0, atol=1e-6)


def test_rollout_rejects_what_it_cannot_differentiate(cuda_device):
    d = sw.generate_patch(nx=12, ny=12)
    s = sw.Structure(d)
    r = sw.Rollout(s, 4)
    with pytest.raises(sw.Unsupported):
        r.forward(step_settings(substeps=2), np.zeros((s.node_count, 3)), np.ones(s.node_count))
    with pytest.raises(sw.InvalidArgument):
        r.backward()
    with pytest.raises(sw.InvalidArgument):
        r.forward(step_settings(), np.zeros((s.node_count, 3)), np.zeros(s.node_count))
    with pytest.raises(sw.InvalidArgument):
        sw.Rollout(s, 0)


def test_rollouts_side_by_side_equal_one_at_a_time(cuda_device):
    """swb_rollout_forward_many / backward_many enqueue every rollout's
    launches on its own structure's stream before waiting for any: three
    wings of different sizes, one against a wall (a plane 1 cm inside its
    trailing edge), give bit for bit the losses and gradients they give one
    at a time."""
    st = step_settings()
    defs = [sw.generate_wing(cells=4, chordwise=10, spanwise_per_cell=2, rib_layers=2, seed=s) for s in (1, 2)]
    defs.append(sw.generate_wing(cells=6, chordwise=12, spanwise_per_cell=2, rib_layers=2, seed=3))

    def make():
        out = []
        for k, d in enumerate(defs):
            s = sw.Structure(d)
            for _ in range(20):
                s.step(st, diagnostics=False)
            if k == 2:
                x_max = s.node_states()[:, 0, 0].max()
                s.set_ground((-1.0, 0.0, 0.0), -(x_max - 0.01), 0.0)
            out.append(s)
        return out

    rng = np.random.default_rng(9)
    structures = make()
    targets = [s.node_states()[:, 0, :] + rng.normal(0.0, 0.02, (s.node_count, 3)) for s in structures]
    weights = [np.ones(s.node_count) for s in structures]
    one = []
    for s, t, w in zip(structures, targets, weights):
        r = sw.Rollout(s, 32, 16)
        loss = r.forward(st, t, w)
        one.append((loss, r.backward()))
        r.close()
    rollouts = [sw.Rollout(s, 32, 16) for s in structures]
    losses = sw.rollout_forward_many(rollouts, st, targets, weights)
    grads = sw.rollout_backward_many(rollouts)
    for (loss, g), l2, g2 in zip(one, losses, grads):
        assert loss == l2
        for key in ("d_rest", "d_comp", "d_dihedral_comp", "d_segment_rest"):
            np.testing.assert_array_equal(g[key], g2[key])
        assert g["d_mass"] == g2["d_mass"]
    for r in rollouts:
        r.close()
    for s in structures:
        s.close()


def test_overflowed_gradient_is_reported(cuda_device):
    """A gradient beyond FP32's range comes back as SWB_NON_FINITE, the
    arrays written all the same: a target 1e42 m away makes the reverse
    sweep's FP32 seed overflow (the loss itself, in FP64, stays finite).  Side by side, the other rollout's
    status stays SWB_OK and its gradient equals the one it gives alone."""
    st = step_settings()
    d = sw.generate_patch(nx=12, ny=12, seed=4)
    a, b = sw.Structure(d), sw.Structure(d)
    n = a.node_count
    target = a.positions().copy()
    w = np.ones(n)
    far = target.copy()
    far[5] = 1e42
    r = sw.Rollout(a, 4, 2)
    r.forward(st, far, w)
    with pytest.raises(sw.NonFiniteState):
        r.backward()
    good = sw.Rollout(b, 4, 2)
    good.forward(st, target, w)
    alone = good.backward()
    r.forward(st, far, w)
    good.forward(st, target, w)
    statuses = np.zeros(2, dtype=np.int32)
    grads = sw.rollout_backward_many([r, good], statuses)
    assert list(statuses) == [abi.NON_FINITE, abi.OK]
    assert not np.isfinite(grads[0]["d_rest"]).all()
    np.testing.assert_array_equal(grads[1]["d_rest"], alone["d_rest"])
    with pytest.raises(sw.NonFiniteState):
        sw.rollout_backward_many([r, good])
    r.close()
    good.close()
    a.close()
    b.close()
