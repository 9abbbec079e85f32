"""Line-line contact (swb_structure_set_line_contact).

The reference rejects contact between two line colliders
(src/softwing/contact.cpp:2336-2339), so this contact has no reference
counterpart and its parity is pinned to this project's own FP64
restatement in the oracle port (`swo_set_line_contact`,
oracle/xpbd_oracle.c): the substep's candidates are the pairs of cable
segments that share no node and whose boxes at the predicted positions,
widened by radius + margin / 2, overlap; after every iteration they are
projected in key order, the segments' closest points pushed apart to
2 x radius.  Known answers pin the restatement (two crossing segments end
exactly 2 x radius apart; segments that share a node or lie beyond reach
are left alone); on the GPU the device matches the port per step on
crossing ropes and on a wing whose lines are nodal cables, and the
refusals (batches, grid schedule, bad radius) hold.  Differentiable
rollouts take it: the FP64 adjoint's reverse of a projection (its Jacobian
by forward mode at the taped inputs) agrees with central differences of
its own forward, and the device's rollout gradient, whose reverse of a
projection is written out by hand, agrees with the FP64 adjoint along the
device trajectory."""
import numpy as np
import pytest

import simwing_b200 as sw
from simwing_b200 import abi
from oracle import oracle as O
from tests.conftest import step_settings
from tests.test_gpu_parity import REL_TOL, rel_error, sync_oracle_to_device

RADIUS = 0.004


def two_segments(dz, angle=np.pi / 2, mass=0.01):
    """Two free two-node cables of length 0.2 m crossing above the origin,
    the first dz above the second."""
    c, s = 0.1 * np.cos(angle), 0.1 * np.sin(angle)
    nodes = [(-0.1, 0.0, 0.5 * dz, mass, False), (0.1, 0.0, 0.5 * dz, mass, False),
             (-c, -s, -0.5 * dz, mass, False), (c, s, -0.5 * dz, mass, False)]
    cons = [(abi.CABLE, 0, 1, 0.2, 1e-8), (abi.CABLE, 2, 3, 0.2, 1e-8)]
    return sw.definition_from_arrays(nodes, constraints=cons)


def segment_distance(p1, q1, p2, q2):
    """Closest distance of two segments, by dense sampling of the first
    and projection onto the second (test-side check, independent of the
    port's closed form)."""
    t = np.linspace(0.0, 1.0, 2001)[:, None]
    a = p1 + t * (q1 - p1)
    d = q2 - p2
    u = np.clip(((a - p2) @ d) / (d @ d), 0.0, 1.0)[:, None]
    return float(np.linalg.norm(a - (p2 + u * d), axis=1).min())


def zero_gravity(iterations, cable_sweep_pairs=None):
    st = step_settings(iterations=iterations, gravity=(0.0, 0.0, 0.0), damping=0.0)
    if cable_sweep_pairs is not None:
        st.cable_sweep_pairs = cable_sweep_pairs
    return st


def test_port_crossing_segments_end_two_radii_apart():
    port = O.PortStructure(two_segments(0.001))
    port.set_line_contact(RADIUS, 0.0)
    port.step(zero_gravity(iterations=4))
    x = port.node_states()[:, 0, :]
    # equal masses, crossing at both midpoints: each segment moves half the
    # overlap along z, rigidly
    np.testing.assert_allclose(x[:2, 2], RADIUS, rtol=0, atol=1e-12)
    np.testing.assert_allclose(x[2:, 2], -RADIUS, rtol=0, atol=1e-12)
    np.testing.assert_allclose(x[:, :2], two_segments(0.001).positions()[:, :2], rtol=0, atol=1e-12)
    assert segment_distance(x[0], x[1], x[2], x[3]) == pytest.approx(2 * RADIUS, abs=1e-9)


def test_port_heavier_segment_moves_less():
    d = two_segments(0.0, angle=np.pi / 3)
    nodes = d.nodes()
    nodes["mass"][:2] = 0.03  # three times the second segment's mass
    port = O.PortStructure(d)
    port.set_line_contact(RADIUS, 0.0)
    z0 = d.positions()[:, 2].copy()
    # no separation direction at zero distance: nothing moves
    port.step(zero_gravity(iterations=2))
    np.testing.assert_array_equal(port.node_states()[:, 0, 2], z0)
    d2 = two_segments(0.002, angle=np.pi / 3)
    d2.nodes()["mass"][:2] = 0.03
    port = O.PortStructure(d2)
    port.set_line_contact(RADIUS, 0.0)
    port.step(zero_gravity(iterations=2))
    x = port.node_states()[:, 0, :]
    up, down = x[0, 2] - 0.001, -0.001 - x[2, 2]
    assert up == pytest.approx((2 * RADIUS - 0.002) / 4, rel=1e-9)
    assert down == pytest.approx(3 * (2 * RADIUS - 0.002) / 4, rel=1e-9)


@pytest.mark.parametrize("case", ["shared node", "beyond reach", "disabled"])
def test_port_leaves_pairs_alone(case):
    if case == "shared node":
        # a sharp V: two cables meeting at node 1, their far ends 1 mm apart
        # (no candidate: the closest points of such a pair are the shared node)
        nodes = [(-0.2, 0.0005, 0.0, 0.01, False), (0.0, 0.0, 0.0, 0.01, False), (-0.2, -0.0005, 0.0, 0.01, False)]
        rest = float(np.hypot(0.2, 0.0005))
        d = sw.definition_from_arrays(nodes, constraints=[(abi.CABLE, 0, 1, rest, 1e-8),
                                                          (abi.CABLE, 1, 2, rest, 1e-8)])
    else:
        d = two_segments(3 * RADIUS)
    port = O.PortStructure(d)
    port.set_line_contact(RADIUS, 0.0)
    if case == "disabled":
        d = two_segments(0.001)
        port = O.PortStructure(d)
        port.set_line_contact(RADIUS, 0.0)
        port.set_line_contact(RADIUS, 0.0, enabled=False)
    x0 = port.node_states()[:, 0, :].copy()
    port.step(zero_gravity(iterations=4, cable_sweep_pairs=0))
    x = port.node_states()[:, 0, :]
    assert np.abs(x - x0).max() <= 1e-9 * max(1.0, np.abs(x0).max()), np.abs(x - x0).max()


def crossing_ropes(k=6, n=12, mass=0.02, rest_scale=1.0, spacing=0.002):
    """k ropes of n nodes, each pinned at its top end, hanging slanted so
    that all of them cross the vertical axis at mid height, `spacing` apart
    in y: every rope overlaps every other at the start.  The cables' rest
    lengths are rest_scale x their initial lengths."""
    nodes, cons = [], []
    for i in range(k):
        a = 0.1 * (i - 0.5 * (k - 1))
        y = spacing * i
        top = np.array([a, y, 1.0])
        bottom = np.array([-a, y, 0.0])
        base = len(nodes)
        for j in range(n):
            p = top + (bottom - top) * j / (n - 1)
            nodes.append((p[0], p[1], p[2], mass, j == 0))
        seg = rest_scale * float(np.linalg.norm(bottom - top)) / (n - 1)
        cons += [(abi.CABLE, base + j, base + j + 1, seg, 1e-7) for j in range(n - 1)]
    return sw.definition_from_arrays(nodes, constraints=cons)


def cable_segments(d):
    c = d.constraints()
    keep = c["kind"] == abi.CABLE
    return np.stack([c["first_node"][keep], c["second_node"][keep]], axis=1).astype(np.int64)


def min_separation(x, segs):
    """The smallest closest distance over pairs of segments that share no
    node and whose midpoints lie within 0.15 m."""
    best = np.inf
    mids = 0.5 * (x[segs[:, 0]] + x[segs[:, 1]])
    for i in range(len(segs)):
        for j in range(i + 1, len(segs)):
            if set(segs[i]) & set(segs[j]) or np.linalg.norm(mids[i] - mids[j]) > 0.15:
                continue
            best = min(best, segment_distance(x[segs[i, 0]], x[segs[i, 1]], x[segs[j, 0]], x[segs[j, 1]]))
    return best


def test_port_ropes_are_kept_apart():
    d = crossing_ropes()
    port = O.PortStructure(d)
    port.set_line_contact(RADIUS, 0.002)
    st = step_settings(gravity=(1.0, 2.0, -9.81))
    for _ in range(10):
        port.step(st)
    x = port.node_states()[:, 0, :]
    assert min_separation(x, cable_segments(d)) >= 2 * RADIUS * 0.9


@pytest.mark.gpu
def test_device_matches_the_port_on_crossing_ropes(cuda_device):
    d = crossing_ropes()
    dev = sw.Structure(d)
    dev.set_line_contact(RADIUS, 0.002)
    orc = O.PortStructure(dev.oracle_definition())
    orc.set_line_contact(RADIUS, 0.002)
    st = step_settings(gravity=(1.0, 2.0, -9.81))
    errs = []
    for _ in range(40):
        sync_oracle_to_device(dev, orc)
        dev.step(st, diagnostics=False)
        orc.step(st)
        errs.append(rel_error(dev.node_states(), orc.node_states()))
    assert max(errs) <= REL_TOL, max(errs)
    assert min_separation(dev.node_states()[:, 0, :], cable_segments(d)) >= 2 * RADIUS * 0.9


@pytest.mark.gpu
def test_device_matches_the_port_on_a_wing_with_cable_lines(cuda_device):
    """The small wing without its pilot: the cascaded lines are nodal
    cables, the segments near each junction come within reach of one
    another."""
    d = sw.generate_wing(cells=4, chordwise=10, spanwise_per_cell=2, rib_layers=2, pilot=0)
    assert d.counts()["cable"] > 0
    dev = sw.Structure(d)
    dev.set_line_contact(0.002, 0.004)
    orc = O.PortStructure(dev.oracle_definition())
    orc.set_line_contact(0.002, 0.004)
    st = step_settings()
    errs = []
    for _ in range(30):
        sync_oracle_to_device(dev, orc)
        dev.step(st, diagnostics=False)
        orc.step(st)
        errs.append(rel_error(dev.node_states(), orc.node_states()))
    assert max(errs) <= REL_TOL, max(errs)


@pytest.mark.gpu
def test_line_contact_refusals(cuda_device):
    d = crossing_ropes(k=3, n=6)
    s = sw.Structure(d)
    with pytest.raises(sw.InvalidArgument):
        s.set_line_contact(0.0)
    with pytest.raises(sw.InvalidArgument):
        s.set_line_contact(RADIUS, -1.0)
    s.set_line_contact(RADIUS)
    st = step_settings()
    s.step(st, diagnostics=False)
    r = sw.Rollout(s, 4, 2)
    r.forward(st, s.node_states()[:, 0, :], np.ones(s.node_count))
    s.set_line_contact(RADIUS, enabled=False)
    with pytest.raises(sw.InvalidArgument):
        r.backward()  # switched between the forward and the backward
    r.close()
    s.step(st, diagnostics=False)
    s.close()
    grid = sw.Structure(d, sw.SolverOptions(flags=abi.OPT_GRID))
    with pytest.raises(sw.Unsupported):
        grid.set_line_contact(RADIUS)
    grid.close()
    with sw.Batch([d, d]) as batch:
        batch.structure(1).set_line_contact(RADIUS)
        with pytest.raises(sw.Unsupported):
            batch.step(st, 1)


ROPES_STEPS = 8


def ropes_rollout_case():
    """Four crossing ropes from rest (every rope within reach of the others
    at the crossing), a target near the start, tilted gravity.  The cables
    start stretched 2 % (rest lengths 0.98 x their lengths): a cable that
    starts exactly at its rest length sits on its slack/taut switch, where
    the FP32 and FP64 iterations of one step may take different sides and
    the rest-length gradients then differ by a few per cent."""
    d = crossing_ropes(k=4, n=8, rest_scale=0.98)
    st = step_settings(gravity=(1.0, 2.0, -9.81))
    rng = np.random.default_rng(1)
    x0 = d.positions()
    return d, st, x0 + rng.normal(0.0, 0.01, x0.shape), np.ones(d.node_count)


def test_fp64_adjoint_with_line_contact_against_finite_differences():
    d, st, target, w = ropes_rollout_case()
    lines = (RADIUS, 0.002)
    g = O.rollout_gradient(d, st, ROPES_STEPS, target, w, lines=lines)
    plain = O.rollout_gradient(d, st, ROPES_STEPS, target, w)
    assert abs(g["loss"] - plain["loss"]) > 0.1 * plain["loss"]  # the contact acts
    rng = np.random.default_rng(2)
    u = rng.normal(size=d.view.constraint_count)
    h = 1e-7
    a, b = d.copy(), d.copy()
    a.constraints()["rest_length"][:] += h * u
    b.constraints()["rest_length"][:] -= h * u
    fd = (O.rollout_gradient(a, st, ROPES_STEPS, target, w, lines=lines)["loss"] -
          O.rollout_gradient(b, st, ROPES_STEPS, target, w, lines=lines)["loss"]) / (2 * h)
    assert abs(g["d_rest"] @ u - fd) <= 1e-6 * abs(fd), (g["d_rest"] @ u, fd)
    c0 = d.constraints()["compliance"].copy()
    a, b = d.copy(), d.copy()
    a.constraints()["compliance"][:] = c0 * (1 + 1e-5)
    b.constraints()["compliance"][:] = c0 * (1 - 1e-5)
    fd = (O.rollout_gradient(a, st, ROPES_STEPS, target, w, lines=lines)["loss"] -
          O.rollout_gradient(b, st, ROPES_STEPS, target, w, lines=lines)["loss"]) / 2e-5
    assert abs((g["d_comp"] * c0).sum() - fd) <= 1e-4 * abs(fd)
    # the adjoint's forward is the port's
    port = O.PortStructure(d)
    port.set_line_contact(*lines)
    for _ in range(ROPES_STEPS):
        port.step(st)
    np.testing.assert_array_equal(g["final"], port.node_states()[:, 0, :])


@pytest.mark.gpu
def test_rollout_gradient_with_line_contact(cuda_device):
    """The device rollout with line contact: its final positions are those of
    plain steps, and its gradient agrees with the FP64 adjoint along the
    device trajectory within 1e-3 per parameter class."""
    from tests.test_adjoint import relative, to_definition_order

    d, st, target, w = ropes_rollout_case()
    s = sw.Structure(d)
    s.set_line_contact(RADIUS, 0.002)
    state = s.node_states()
    r = sw.Rollout(s, ROPES_STEPS, 4)
    r.forward(st, target, w)
    grad = r.backward()
    final = r.final_positions()
    r.close()
    traj = [state]
    for _ in range(ROPES_STEPS):
        s.step(st, diagnostics=False)
        traj.append(s.node_states())
    np.testing.assert_allclose(final, traj[-1][:, 0, :], rtol=0, atol=1e-6)
    ref = O.rollout_gradient(s.oracle_definition(), st, ROPES_STEPS, target, w, state=state,
                             trajectory=np.array(traj[:-1]), lines=(RADIUS, 0.002))
    order = s.sweep_order(abi.SWEEP_DISTANCE)
    c0 = d.constraints()["compliance"]
    mine = {"rest": grad["d_rest"], "comp": grad["d_comp"] * c0}
    theirs = {"rest": to_definition_order(ref["d_rest"], order), "comp": to_definition_order(ref["d_comp"], order) * c0}
    errors = {k: relative(mine[k], theirs[k]) for k in mine}
    assert all(v <= 1e-3 for v in errors.values()), errors
    s.close()


@pytest.mark.gpu
def test_wing_rollout_gradient_with_line_contact(cuda_device):
    """The small wing with its pilot and line-line contact of its cascaded
    lines (2 mm radius, 4 mm margin: candidates near every junction), a
    16-step rollout: the calibration parameters' gradient (each line's rest
    length, the compliance classes, the risers and the pilot mass) agrees
    with the FP64 adjoint along the device trajectory within 1e-3."""
    from tests.test_adjoint import calibration_parameters, payload_vector, relative, to_definition_order

    d = sw.generate_wing(cells=4, chordwise=10, spanwise_per_cell=2, rib_layers=2, seed=3)
    st = step_settings()
    s = sw.Structure(d)
    s.set_line_contact(0.002, 0.004)
    for _ in range(20):
        s.step(st, diagnostics=False)
    state, pay = s.node_states(), payload_vector(s)
    rng = np.random.default_rng(7)
    target = state[:, 0, :] + rng.normal(0.0, 0.01, state[:, 0, :].shape)
    w = np.ones(d.node_count)
    steps = 16
    r = sw.Rollout(s, steps, 8)
    r.forward(st, target, w)
    grad = r.backward()
    r.close()
    traj, tpay = [state], [pay]
    for _ in range(steps - 1):
        s.step(st, diagnostics=False)
        traj.append(s.node_states())
        tpay.append(payload_vector(s))
    ref = O.rollout_gradient(s.oracle_definition(), st, steps, target, w, state=state, payload=pay,
                             trajectory=np.array(traj), trajectory_payloads=np.array(tpay), lines=(0.002, 0.004))
    ref["d_rest"] = to_definition_order(ref["d_rest"], s.sweep_order(abi.SWEEP_DISTANCE))
    ref["d_comp"] = to_definition_order(ref["d_comp"], s.sweep_order(abi.SWEEP_DISTANCE))
    ref["d_dihedral_comp"] = to_definition_order(ref["d_dihedral_comp"], s.sweep_order(abi.SWEEP_DIHEDRAL))
    mine, theirs = calibration_parameters(d, grad), calibration_parameters(d, ref)
    errors = {k: relative(mine[k], theirs[k]) for k in theirs}
    assert all(v <= 1e-3 for v in errors.values()), errors
    s.close()


@pytest.mark.gpu
def test_rollout_tape_capacity(cuda_device):
    """A rollout tapes at most 4,096 line-line candidates per step: 100
    ropes crossing within 5 mm of one another give about 18,000 in the first
    step; the plain step and the rollout's forward take them, the backward
    fails with SWB_CONTACT_ERROR and says why."""
    d = crossing_ropes(k=100, n=4, spacing=0.00005)
    st = step_settings(iterations=4)
    s = sw.Structure(d)
    s.set_line_contact(RADIUS, 0.002)
    r = sw.Rollout(s, 2, 2)
    r.forward(st, s.positions(), np.ones(s.node_count))
    with pytest.raises(sw.ContactStepError, match="rollout's tape"):
        r.backward()
    r.close()
    s.step(st, diagnostics=False)
    assert np.isfinite(s.node_states()).all()
    s.close()
