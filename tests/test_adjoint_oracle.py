"""The FP64 reference gradient (oracle/xpbd_adjoint.cpp) that the device
adjoint is checked against is itself pinned here:

  * its forward rollout equals the oracle port's (xpbd_oracle.c, pinned bit
    for bit to the reference) bit for bit;
  * from a settled state, its gradient of the rollout loss agrees with
    central finite differences of the same FP64 forward for every parameter
    class the calibration uses -- rest lengths (random directions over all
    constraints and over the cables alone), the three compliance classes,
    the riser rest lengths and the pilot mass -- to 1e-3 relative.

A rollout that starts from rest sits on the slack/taut switch of every line
(cables are built at exactly their rest length), where the step is not
differentiable; the calibration therefore starts from a settled state."""
import numpy as np
import pytest

import simwing_b200 as sw
from oracle import oracle as O
from tests.conftest import step_settings

REL_TOL = 1e-3


def settled(definition, steps=40):
    port = O.PortStructure(definition)
    st = step_settings()
    for _ in range(steps):
        port.step(st)
    p, _, _ = port.payload()
    pay = np.array([p.center_of_mass.x, p.center_of_mass.y, p.center_of_mass.z, p.body_to_world.w,
                    p.body_to_world.x, p.body_to_world.y, p.body_to_world.z, p.linear_velocity.x,
                    p.linear_velocity.y, p.linear_velocity.z, p.angular_velocity.x, p.angular_velocity.y,
                    p.angular_velocity.z])
    return port.node_states(), pay


def surface_weights(definition):
    w = np.zeros(definition.node_count)
    tri = definition.triangles()["nodes"].astype(np.int64)
    w[tri.ravel()] = 1.0
    return w


@pytest.fixture(scope="module")
def case():
    d = sw.generate_wing(cells=4, chordwise=10, spanwise_per_cell=2, rib_layers=2, seed=3)
    state, pay = settled(d)
    rng = np.random.default_rng(1)
    target = state[:, 0, :] + rng.normal(0.0, 0.02, (d.node_count, 3))
    w = surface_weights(d)
    steps = 12
    g = O.rollout_gradient(d, step_settings(), steps, target, w, state=state, payload=pay)

    def loss(defn):
        return O.rollout_gradient(defn, step_settings(), steps, target, w, state=state, payload=pay)["loss"]

    def fd(mod, h):
        a, b = d.copy(), d.copy()
        mod(a, h)
        mod(b, -h)
        return (loss(a) - loss(b)) / (2 * h)

    return d, g, fd, rng, (state, pay, target, w, steps)


def close(adjoint, fd):
    assert abs(adjoint - fd) <= REL_TOL * abs(fd), (adjoint, fd)


def test_forward_equals_the_port_bitwise(case):
    d, g, _, _, (state, pay, _, _, steps) = case
    port = O.PortStructure(d)
    port.write_node_states(state)
    import simwing_b200.abi as abi
    port.write_payload(abi.PayloadState(abi.Vec3(*pay[0:3]), abi.Quat(*pay[3:7]), abi.Vec3(*pay[7:10]),
                                        abi.Vec3(*pay[10:13])))
    for _ in range(steps):
        port.step(step_settings())
    np.testing.assert_array_equal(port.positions(), g["final"])


def test_rest_length_directions(case):
    d, g, fd, rng, _ = case
    kinds = d.constraints()["kind"]
    u = rng.normal(size=len(kinds))
    u[kinds == 4] = 0.0
    cable = np.where(kinds == 2, u, 0.0)
    for direction in (u, cable):
        def mod(defn, h, direction=direction):
            defn.constraints()["rest_length"][:] += h * direction
        close(g["d_rest"] @ direction, fd(mod, 1e-7))


def test_compliance_classes(case):
    d, g, fd, _, _ = case
    cons = d.constraints()
    kinds = cons["kind"]
    c0 = cons["compliance"].copy()
    for mask in ((kinds == 1) | (kinds == 3), kinds == 2):
        def mod(defn, h, mask=mask):
            defn.constraints()["compliance"][mask] = c0[mask] * (1.0 + h)
        close((g["d_comp"] * c0)[mask].sum(), fd(mod, 1e-5))
    h0 = d.dihedrals()["compliance"].copy()

    def hmod(defn, h):
        defn.dihedrals()["compliance"][:] = h0 * (1.0 + h)
    close((g["d_dihedral_comp"] * h0).sum(), fd(hmod, 1e-5))


def test_riser_rest_lengths_and_pilot_mass(case):
    d, g, fd, _, _ = case
    for k in range(2):
        def mod(defn, h, k=k):
            defn.view.suspension.contents.segments[k].rest_length += h
        close(g["d_segment_rest"][k], fd(mod, 1e-7))

    def mass(defn, h):
        defn.view.suspension.contents.pilot_mass += h
    assert abs(g["d_mass"] - fd(mass, 1e-4)) <= 2e-3 * abs(g["d_mass"])
