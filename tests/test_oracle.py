"""Pins the CPU oracle.

The C restatement (oracle/liboracle.so) must reproduce the reference's own
solver (oracle/_ref/libswref.so, compiled from the reference sources) bit
for bit, and both must pass the reference's known-answer tests
(tests/simwing_structure_test.cpp:104-177, softwing_material_test.cpp:
182-362 in the reference) and the committed golden trajectories.
"""
import os

import numpy as np
import pytest

import simwing_b200 as sw
from oracle import oracle as O
from tests.conftest import step_settings

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

DIST, CABLE, TIE, SEAM = 1, 2, 3, 4


def checkers():
    out = [O.PortStructure]
    if O.ref_available():
        out.append(O.RefStructure)
    return out


# ---- simwing_structure_test.cpp:104-126 ------------------------------------
@pytest.mark.parametrize("cls", checkers())
def test_gravity_and_nodal_force_known_answer(cls):
    d = sw.definition_from_arrays([(0.0, 0.0, 0.0, 2.0, False)])
    s = cls(d)
    s.add_external_force(0, (4.0, 0.0, 0.0))
    s.step(sw.StepSettings(time_step=0.25, substeps=1, constraint_iterations=0, gravity=(0, 0, -2.0),
                           velocity_damping=0.0))
    st = s.node_states()
    assert st[0, 2, 0] == pytest.approx(0.5, abs=1e-15)
    assert st[0, 2, 2] == pytest.approx(-0.5, abs=1e-15)
    assert st[0, 0, 0] == pytest.approx(0.125, abs=1e-15)
    assert st[0, 0, 2] == pytest.approx(-0.125, abs=1e-15)
    diag = s.diagnostics()
    assert diag.linear_momentum.x == pytest.approx(1.0, abs=1e-15)


def _pair(kind, length):
    return sw.definition_from_arrays([(0.0, 0.0, 0.0, 0.0, True), (length, 0.0, 0.0, 1.0, False)],
                                     constraints=[(kind, 0, 1, 1.0, 0.0)])


CONSTRAINT_SETTINGS = dict(time_step=1.0 / 60.0, substeps=1, constraint_iterations=1, gravity=(0, 0, 0),
                           velocity_damping=0.0)


# ---- simwing_structure_test.cpp:149-177 ------------------------------------
@pytest.mark.parametrize("cls", checkers())
@pytest.mark.parametrize("kind,length,expected", [(DIST, 2.0, 1.0), (CABLE, 0.5, 0.5), (CABLE, 2.0, 1.0),
                                                  (TIE, 2.0, 1.0)])
def test_distance_cable_tie_known_answers(cls, kind, length, expected):
    s = cls(_pair(kind, length))
    s.step(sw.StepSettings(**CONSTRAINT_SETTINGS))
    x = s.node_states()[1, 0, 0]
    if kind == CABLE and length < 1.0:
        assert x == 0.5  # a slack cable is not pushed
    else:
        assert x == pytest.approx(expected, abs=1e-12)


def _hinge(mirrored=False, fixed=True, moves=None, rest=0.0):
    side = -1.0 if mirrored else 1.0
    pts = [[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, side, 0.0], [1.0, -side, 0.0]]
    for i, p in (moves or {}).items():
        pts[i] = list(p)
    nodes = [(p[0], p[1], p[2], 0.0 if (fixed and i < 3) else 1.0, fixed and i < 3) for i, p in enumerate(pts)]
    return sw.definition_from_arrays(nodes, dihedrals=[(0, 1, 2, 3, rest, 0.0)])


HINGE_SETTINGS = dict(time_step=1.0 / 60.0, substeps=1, constraint_iterations=1, gravity=(0, 0, 0),
                      velocity_damping=0.0)


# ---- softwing_material_test.cpp:182-239 ------------------------------------
@pytest.mark.parametrize("cls", checkers())
def test_dihedral_flat_folded_inplane_mirror_degenerate(cls):
    flat = cls(_hinge())
    before = flat.positions()
    flat.step(sw.StepSettings(**HINGE_SETTINGS))
    assert np.abs(flat.positions() - before).max() < 1e-15

    folded = cls(_hinge(moves={3: (1.0, -1.0, 0.5)}))
    folded.step(sw.StepSettings(**HINGE_SETTINGS))
    p = folded.positions()
    assert abs(p[3, 2]) < 0.5
    assert np.array_equal(p[:3], np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], dtype=float))

    inplane = cls(_hinge(moves={2: (-0.25, 1.3, 0.0), 3: (1.4, -0.7, 0.0)}))
    before = inplane.positions()
    inplane.step(sw.StepSettings(**HINGE_SETTINGS))
    assert np.abs(inplane.positions() - before).max() < 1e-15

    right = cls(_hinge(moves={3: (1.0, -1.0, 0.4)}))
    left = cls(_hinge(mirrored=True, moves={3: (1.0, 1.0, 0.4)}))
    right.step(sw.StepSettings(**HINGE_SETTINGS))
    left.step(sw.StepSettings(**HINGE_SETTINGS))
    assert abs(right.positions()[3, 2] - left.positions()[3, 2]) < 1e-12

    degenerate = cls(_hinge(moves={3: (0.5, 0.0, 0.0)}))
    degenerate.step(sw.StepSettings(**HINGE_SETTINGS))
    assert np.isfinite(degenerate.node_states()).all()


# ---- softwing_material_test.cpp:281-318: analytic gradient vs FD -----------
def test_dihedral_gradient_matches_finite_difference():
    pts = np.array([[-0.2, 0.1, 0.3], [1.1, -0.15, 0.25], [0.15, 1.0, -0.2], [0.75, -0.8, 0.65]])
    angle, grad, valid = O.evaluate_dihedral(pts.ravel())
    assert valid
    eps = 1e-6
    worst = 0.0
    for n in range(4):
        for axis in range(3):
            plus, minus = pts.copy(), pts.copy()
            plus[n, axis] += eps
            minus[n, axis] -= eps
            a = O.evaluate_dihedral(plus.ravel())[0]
            b = O.evaluate_dihedral(minus.ravel())[0]
            numerical = np.remainder(a - b + np.pi, 2 * np.pi) - np.pi
            worst = max(worst, abs(numerical / (2 * eps) - grad[n, axis]))
    assert worst < 2e-6


def test_closed_form_dihedral_equals_reference_evaluation():
    """The device evaluates the hinge angle and gradient in closed form; it
    must be the same function as the reference's reverse-mode evaluation
    (soft_body.cpp:1648-1711), up to FP64 round-off."""
    rng = np.random.default_rng(0)
    worst_g = worst_a = 0.0
    for _ in range(2000):
        p = rng.normal(size=(4, 3))
        angle, grad, valid = O.evaluate_dihedral(p.ravel())
        if not valid:
            continue
        a, b, c, d = p
        e = b - a
        A1, A2 = np.cross(e, c - a), np.cross(d - a, e)
        e2, q1, q2 = e @ e, A1 @ A1, A2 @ A2
        el = np.sqrt(e2)
        theta = np.arctan2(e @ np.cross(A1, A2) / el, A1 @ A2)
        gc, gd = -(el / q1) * A1, -(el / q2) * A2
        gb = -((c - a) @ e / e2) * gc - ((d - a) @ e / e2) * gd
        ga = -(gb + gc + gd)
        worst_g = max(worst_g, np.abs(np.array([ga, gb, gc, gd]) - grad).max() / np.abs(grad).max())
        worst_a = max(worst_a, abs(np.remainder(theta - angle + np.pi, 2 * np.pi) - np.pi))
    assert worst_g < 1e-12 and worst_a < 1e-12


# ---- the restatement is the reference, bit for bit -------------------------
@needs_ref
def test_port_matches_reference_bitwise_on_patch():
    d = sw.generate_patch()
    ref, port = O.RefStructure(d), O.PortStructure(d)
    st = step_settings()
    for _ in range(5):
        ref.step(st)
        port.step(st)
    assert np.array_equal(ref.node_states(), port.node_states())


@needs_ref
def test_port_matches_reference_bitwise_on_wing_with_pilot():
    d = sw.generate_wing(cells=6, chordwise=12, spanwise_per_cell=2, rib_layers=3)
    assert d.has_suspension
    ref, port = O.RefStructure(d), O.PortStructure(d)
    st = step_settings()
    for _ in range(3):
        ref.step(st)
        port.step(st)
    assert np.array_equal(ref.node_states(), port.node_states())
    rp, _ = ref.payload(2)
    pp, _, _ = port.payload()
    assert rp.center_of_mass.z == pp.center_of_mass.z
    assert rp.body_to_world.x == pp.body_to_world.x


@needs_ref
def test_port_matches_reference_on_permuted_definition():
    d = sw.generate_patch(nx=12, ny=12)
    _, do, ho = sw.plan_schedule(d, sw.SolverOptions(blocks=4))
    p = d.permuted(do, ho)
    ref, port = O.RefStructure(p), O.PortStructure(p)
    st = step_settings()
    for _ in range(4):
        ref.step(st)
        port.step(st)
    assert np.array_equal(ref.node_states(), port.node_states())


# ---- load-path cable sweeps --------------------------------------------------
@needs_ref
@pytest.mark.parametrize("pairs,pilot,permuted", [(1, 1, False), (8, 1, False), (96, 1, True), (96, 0, True)])
def test_port_matches_reference_bitwise_with_cable_pairs(pairs, pilot, permuted):
    """Graph-depth load-path sweeps (soft_body.cpp:528-629, 1265-1388):
    a quarter of the pairs interleaved before the first iterations' general
    sweeps, the rest closing the substep; on a wing with cascaded lines, with
    and without the pilot, on the generator's constraint order and on the
    device sweep order (the load-path order follows the definition's).  The
    outcome must agree too: where the reference rejects a step (96 pairs
    stretch the lines past the suspension's residual bound here), the
    restatement rejects it with the same status and both roll back."""
    d = sw.generate_wing(cells=6, chordwise=12, spanwise_per_cell=2, rib_layers=3, pilot=pilot)
    if permuted:
        _, do, ho = sw.plan_schedule(d)
        d = d.permuted(do, ho)
    ref, port = O.RefStructure(d), O.PortStructure(d)
    st = step_settings()
    st.cable_sweep_pairs = pairs
    for _ in range(3):
        outcome = []
        for s in (ref, port):
            try:
                s.step(st)
                outcome.append(0)
            except O.OracleError as e:
                outcome.append(e.status)
        assert outcome[0] == outcome[1]
        assert np.array_equal(ref.node_states(), port.node_states())


# ---- membranes ---------------------------------------------------------------
# material of the reference's membrane tests (softwing_material_test.cpp:30-39,
# simwing_structure_test.cpp:271-274)
MEMBRANE = {"warp_stiffness": 800.0, "weft_stiffness": 500.0, "coupling_stiffness": 100.0,
            "shear_stiffness": 180.0}
RIGHT_CHART = ((0.0, 0.0), (1.0, 0.0), (0.0, 1.0))


@pytest.mark.parametrize("cls", checkers())
def test_membrane_rest_chart_known_answer(cls):
    """simwing_structure_test.cpp:256-283: one orthotropic element at its
    rest chart, one fixed corner, 4 iterations without gravity: finite, one
    membrane, zero strain (1e-15)."""
    d = sw.definition_from_arrays([(0.0, 0.0, 0.0, 0.0, True), (1.0, 0.0, 0.0, 1.0, False),
                                   (0.0, 1.0, 0.0, 1.0, False)], triangles=[(0, 1, 2)],
                                  membranes=[(0, RIGHT_CHART, MEMBRANE)])
    s = cls(d)
    diag = s.step(sw.StepSettings(time_step=1 / 60, substeps=1, constraint_iterations=4, gravity=(0, 0, 0),
                                  velocity_damping=0.0))
    assert diag.membrane_count == 1 and diag.finite
    assert abs(diag.maximum_absolute_membrane_strain) <= 1e-15


@pytest.mark.parametrize("cls", checkers())
def test_compressed_membrane_solve_known_answer(cls):
    """softwing_material_test.cpp:74-103: an element compressed to 0.9 of its
    chart along the warp, compression softening 0.05, damping 0.02 s;
    dt 1/60 in 2 substeps of 4 iterations without gravity: finite positions
    and velocities, and the strain moves towards the chart."""
    material = dict(MEMBRANE, damping_seconds=0.02, compression_stiffness_ratio=0.05)
    d = sw.definition_from_arrays([(0.0, 0.0, 0.0, 0.0, True), (0.9, 0.0, 0.0, 1.0, False),
                                   (0.0, 1.0, 0.0, 1.0, False)], triangles=[(0, 1, 2)],
                                  membranes=[(0, RIGHT_CHART, material)])
    s = cls(d)
    diag = s.step(sw.StepSettings(time_step=1 / 60, substeps=2, constraint_iterations=4, gravity=(0, 0, 0),
                                  velocity_damping=0.0))
    st = s.node_states()
    assert diag.finite and np.isfinite(st).all()
    # initial warp strain 0.5 (0.81 - 1) = -0.095
    assert 0.0 < diag.maximum_absolute_membrane_strain < 0.095


@needs_ref
@pytest.mark.parametrize("option,pinned", [(1, 1), (2, 1), (2, 0)])
def test_port_matches_reference_bitwise_on_membrane_patch(option, pinned):
    """Membrane elements on every triangle (linear material; pre-tension,
    damping and compression softening), with the patch pinned and free (the
    free patch also runs the momentum guard): node states and membrane
    diagnostics bit for bit."""
    d = sw.generate_patch(nx=12, ny=12, membranes=option, pin_top_corners=pinned)
    ref, port = O.RefStructure(d), O.PortStructure(d)
    st = step_settings(iterations=12)
    for _ in range(4):
        dr = ref.step(st)
        dp = port.step(st)
    assert np.array_equal(ref.node_states(), port.node_states())
    assert dr.membrane_count == dp.membrane_count == d.view.triangle_count
    assert dr.maximum_absolute_membrane_strain == dp.maximum_absolute_membrane_strain
    assert dr.maximum_membrane_residual == dp.maximum_membrane_residual
    assert dr.maximum_membrane_residual > 0.0


@needs_ref
def test_port_matches_reference_bitwise_on_membrane_wing():
    """The wing with its fabric as membrane elements (the reference scene
    assembly's form), lines and pilot: node states, pilot and membrane
    diagnostics bit for bit."""
    d = sw.generate_wing(cells=6, chordwise=12, spanwise_per_cell=2, rib_layers=3, fabric=1)
    assert d.view.membrane_count == d.view.triangle_count
    ref, port = O.RefStructure(d), O.PortStructure(d)
    st = step_settings()
    for _ in range(3):
        dr = ref.step(st)
        dp = port.step(st)
    assert np.array_equal(ref.node_states(), port.node_states())
    assert dr.maximum_absolute_membrane_strain == dp.maximum_absolute_membrane_strain
    assert dr.maximum_membrane_residual == dp.maximum_membrane_residual


def test_float_vector_port_rounds_to_fp32_and_stays_close():
    """The FP32-rounding build of the port (the tests' sensitivity measure)
    stores FP32-representable positions and stays within FP32 agreement of
    the FP64 port on a well-conditioned membrane patch."""
    d = sw.generate_patch(membranes=2)
    f64, f32 = O.PortStructure(d), O.PortStructure(d, float_vectors=True)
    st = step_settings()
    for _ in range(3):
        f64.step(st)
        f32.step(st)
    a, b = f32.node_states()[:, 0, :], f64.node_states()[:, 0, :]
    assert np.array_equal(a, a.astype(np.float32).astype(np.float64))
    diff = float(np.abs(a - b).max())
    assert 0.0 < diff <= 1e-5 * max(1.0, float(np.abs(b).max()))


def test_golden_trajectories():
    """Committed FP64 fixtures produced by the reference build
    (tests/golden/make_golden.py)."""
    path = os.path.join(GOLDEN, "trajectories.npz")
    g = np.load(path)
    for name in ("patch", "wing", "membrane_patch"):
        d = _golden_definition(name)
        port = O.PortStructure(d)
        st = step_settings()
        for k in range(g[f"{name}_steps"].item()):
            port.step(st)
        np.testing.assert_array_equal(port.node_states()[:, 0, :], g[f"{name}_positions"])


def _golden_definition(name):
    if name == "patch":
        return sw.generate_patch(nx=17, ny=17, seed=7)
    if name == "membrane_patch":
        return sw.generate_patch(nx=12, ny=12, seed=9, membranes=2)
    return sw.generate_wing(cells=4, chordwise=10, spanwise_per_cell=2, rib_layers=2, seed=3)
