"""The ground plane (swb_structure_set_ground, swb_batch_set_ground).

The reference's structural step has no ground (its only plane is the
payload's support plane, which the adapter leaves free), so the plane's
parity is pinned to this project's own restatement: the FP64 oracle port
(`swo_set_ground`, oracle/xpbd_oracle.c) and the FP64 adjoint
(oracle/xpbd_adjoint.cpp) take the same projection after every iteration.
Known answers pin the restatement: a node that falls onto the plane stops
on it, a node sliding on it with friction stops where Coulomb friction
says, and the FP64 adjoint agrees with central differences.  On the GPU the
device matches the port per step, the rollout gradient matches the FP64
adjoint along the device trajectory, and a batch with the plane equals
plain structures bit for bit."""
import numpy as np
import pytest

import simwing_b200 as sw
from simwing_b200 import abi
from oracle import oracle as O
from tests.conftest import step_settings
from tests.test_adjoint import payload_vector, relative, to_definition_order
from tests.test_gpu_parity import REL_TOL, rel_error, sync_oracle_to_device

FLOOR = 0.05      # the patch hangs from its pinned corners at z = 1 down to z = 0


def single_node(z=0.5):
    return sw.definition_from_arrays([(0.0, 0.0, z, 1.0, False)])


def test_port_node_falls_onto_the_plane():
    port = O.PortStructure(single_node())
    port.set_ground((0.0, 0.0, 1.0), 0.0, 0.0)
    st = step_settings(iterations=4, damping=0.0)
    for _ in range(60):
        port.step(st)
    x = port.node_states()
    assert x[0, 0, 2] == 0.0            # projected exactly onto the plane
    assert x[0, 2, 2] == 0.0            # and at rest on it


def test_port_friction_stops_a_sliding_node():
    """A node resting on the plane with horizontal speed v slides under
    Coulomb friction mu: each step takes mu g dt^2 of its displacement, so
    it stops after about v / (mu g) seconds, having slid v^2 / (2 mu g)."""
    mu, v = 0.5, 1.0
    port = O.PortStructure(single_node(z=0.0))
    s = port.node_states()
    s[0, 2, 0] = v
    port.write_node_states(s)
    port.set_ground((0.0, 0.0, 1.0), 0.0, mu)
    st = step_settings(iterations=1, damping=0.0)
    for _ in range(120):
        port.step(st)
    x = port.node_states()
    dt, g = 1.0 / 120.0, 9.81
    assert x[0, 2, 0] == 0.0                                    # stopped
    assert x[0, 0, 0] == pytest.approx(v * v / (2 * mu * g), rel=0.05, abs=v * dt)
    assert x[0, 0, 2] == 0.0


def resting_patch(nx=17, ny=17, **kw):
    """The hanging patch (pinned top corners) whose lower edge the plane
    lifts and then carries."""
    return sw.generate_patch(nx=nx, ny=ny, **kw)


def test_fp64_adjoint_with_the_plane_against_finite_differences():
    """The FP64 adjoint of a rollout in which the plane carries the patch's
    lower rows, against central differences of its own forward: the
    compliance scale and a direction of rest lengths."""
    d = resting_patch()
    st = step_settings()
    port = O.PortStructure(d)
    port.set_ground((0.0, 0.0, 1.0), FLOOR, 0.0)
    for _ in range(30):
        port.step(st)
    state = port.node_states()
    assert state[:, 0, 2].min() == pytest.approx(FLOOR, abs=1e-12)
    rng = np.random.default_rng(3)
    target = state[:, 0, :] + rng.normal(0.0, 0.01, state[:, 0, :].shape)
    w = np.ones(d.node_count)
    ground = ((0.0, 0.0, 1.0), FLOOR)
    steps = 10
    g = O.rollout_gradient(d, st, steps, target, w, state=state, ground=ground)

    def loss(defn):
        return O.rollout_gradient(defn, st, steps, target, w, state=state, ground=ground)["loss"]

    h0 = d.dihedrals()["compliance"].copy()
    h = 1e-5
    a, b = d.copy(), d.copy()
    a.dihedrals()["compliance"][:] = h0 * (1 + h)
    b.dihedrals()["compliance"][:] = h0 * (1 - h)
    fd = (loss(a) - loss(b)) / (2 * h)
    got = (g["d_dihedral_comp"] * h0).sum()
    assert abs(got - fd) <= 1e-3 * abs(fd), (got, fd)
    u = rng.normal(size=d.view.constraint_count)
    a, b = d.copy(), d.copy()
    a.constraints()["rest_length"][:] += 1e-7 * u
    b.constraints()["rest_length"][:] -= 1e-7 * u
    fd = (loss(a) - loss(b)) / 2e-7
    assert abs(g["d_rest"] @ u - fd) <= 1e-3 * abs(fd)


@pytest.mark.gpu
@pytest.mark.parametrize("friction", [0.0, 0.6])
def test_device_matches_the_port_with_the_plane(cuda_device, friction):
    d = resting_patch()
    dev = sw.Structure(d)
    dev.set_ground((0.0, 0.0, 1.0), FLOOR, friction)
    orc = O.PortStructure(dev.oracle_definition())
    orc.set_ground((0.0, 0.0, 1.0), FLOOR, friction)
    st = step_settings(gravity=(1.5, 0.0, -9.81))
    errs = []
    for _ in range(40):
        sync_oracle_to_device(dev, orc)
        dev.step(st, diagnostics=False)
        orc.step(st)
        errs.append(rel_error(dev.node_states(), orc.node_states()))
    assert max(errs) <= REL_TOL, max(errs)
    z = dev.node_states()[:, 0, 2]
    # the lower edge rests on the plane (without friction the sideways pull
    # swings part of it up again)
    assert z.min() >= FLOOR - 1e-6 and np.count_nonzero(z < FLOOR + 1e-4) >= 4


@pytest.mark.gpu
def test_wing_lands_on_the_plane(cuda_device):
    """The small wing with its pilot, dropped onto a plane 0.4 m below the
    pilot: per-step parity with the port while the pilot's harness and
    lines settle on it."""
    d = sw.generate_wing(cells=4, chordwise=10, spanwise_per_cell=2, rib_layers=2)
    dev = sw.Structure(d)
    pilot_z = dev.suspension_state().center_of_mass[2]
    floor = pilot_z - 0.4
    dev.set_ground((0.0, 0.0, 1.0), floor, 0.3)
    orc = O.PortStructure(dev.oracle_definition())
    orc.set_ground((0.0, 0.0, 1.0), floor, 0.3)
    st = step_settings()
    errs = []
    for _ in range(40):
        sync_oracle_to_device(dev, orc)
        dev.step(st, diagnostics=False)
        orc.step(st)
        errs.append(rel_error(dev.node_states(), orc.node_states()))
    assert max(errs) <= REL_TOL, max(errs)
    assert dev.node_states()[:, 0, 2].min() >= floor - 1e-6


@pytest.mark.gpu
def test_rollout_gradient_with_the_plane(cuda_device):
    """The device's rollout gradient with the frictionless plane against
    the FP64 adjoint along the device trajectory (both reverse sweeps see
    the same inputs): every class within 1e-3."""
    d = resting_patch()
    st = step_settings()
    s = sw.Structure(d)
    s.set_ground((0.0, 0.0, 1.0), FLOOR, 0.0)
    for _ in range(30):
        s.step(st, diagnostics=False)
    state = s.node_states()
    rng = np.random.default_rng(5)
    target = state[:, 0, :] + rng.normal(0.0, 0.01, state[:, 0, :].shape)
    w = np.ones(d.node_count)
    steps = 16
    r = sw.Rollout(s, steps, 4)
    r.forward(st, target, w)
    grad = r.backward()
    r.close()
    traj = [state]
    for _ in range(steps - 1):
        s.step(st, diagnostics=False)
        traj.append(s.node_states())
    ref = O.rollout_gradient(s.oracle_definition(), st, steps, target, w, state=state, trajectory=np.array(traj),
                             ground=((0.0, 0.0, 1.0), FLOOR))
    dist_order = s.sweep_order(abi.SWEEP_DISTANCE)
    dih_order = s.sweep_order(abi.SWEEP_DIHEDRAL)
    c0 = d.constraints()["compliance"]
    h0 = d.dihedrals()["compliance"]
    mine = {"rest": grad["d_rest"], "comp": grad["d_comp"] * c0, "dihedral": grad["d_dihedral_comp"] * h0}
    theirs = {"rest": to_definition_order(ref["d_rest"], dist_order),
              "comp": to_definition_order(ref["d_comp"], dist_order) * c0,
              "dihedral": to_definition_order(ref["d_dihedral_comp"], dih_order) * h0}
    errors = {k: relative(mine[k], theirs[k]) for k in mine}
    assert all(v <= 1e-3 for v in errors.values()), errors
    with pytest.raises(sw.Unsupported):
        s.set_ground((0.0, 0.0, 1.0), FLOOR, 0.5)
        r = sw.Rollout(s, steps, 4)
        r.forward(st, target, w)


@pytest.mark.gpu
def test_batch_with_the_plane_equals_plain_structures(cuda_device):
    defs = [resting_patch(), resting_patch(seed=4, nx=21, ny=13)]
    st = step_settings(gravity=(1.0, 0.0, -9.81))
    with sw.Batch(defs, sw.BatchOptions(target_patch_nodes=512, graph_steps=8)) as batch:
        # plain structures on the same rank counts step bit for bit alike
        plain = [sw.Structure(d, sw.SolverOptions(cluster_ctas=batch.structure(k).schedule_report().cluster_ctas))
                 for k, d in enumerate(defs)]
        for p in plain:
            p.set_ground((0.0, 0.0, 1.0), FLOOR, 0.4)
        batch.set_ground((0.0, 0.0, 1.0), FLOOR, 0.4)
        statuses = batch.step(st, 60)
        assert not statuses.any()
        for p in plain:
            for _ in range(60):
                p.step(st, diagnostics=False)
        for k, p in enumerate(plain):
            ranks = batch.structure(k)
            np.testing.assert_array_equal(ranks.node_states(), p.node_states())
