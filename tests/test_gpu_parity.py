"""Device parity: the sm_100a solver against the FP64 oracle, through the
C-ABI.

The oracle runs the reference algorithm (the C restatement pinned bit for
bit to the reference build in test_oracle.py) on the definition permuted
into the device sweep order, so both sides perform the same Gauss-Seidel
sweep.  Tolerances:
  * one step from an identical state: max position error / max |position|
    <= 1e-5 (FP32 device vs FP64 oracle);
  * 600 steps of the cloth patch: settled shape and max distance error
    within 1e-3 m.
"""
import numpy as np
import pytest

import simwing_b200 as sw
from oracle import oracle as O
from tests.conftest import step_settings

pytestmark = pytest.mark.gpu

REL_TOL = 1e-5


def rel_error(device_states, oracle_states):
    scale = max(1.0, float(np.abs(oracle_states[:, 0, :]).max()))
    return float(np.abs(device_states[:, 0, :] - oracle_states[:, 0, :]).max()) / scale


def sync_oracle_to_device(dev, orc):
    orc.write_node_states(dev.node_states())
    if dev._segments:
        s = dev.suspension_state()
        import simwing_b200.abi as abi
        orc.write_payload(abi.PayloadState(abi.Vec3(*s.center_of_mass), abi.Quat(*s.body_to_world),
                                           abi.Vec3(*s.linear_velocity), abi.Vec3(*s.angular_velocity)))


def per_step_errors(definition, steps, settings, options=None, sync=True):
    dev = sw.Structure(definition, options)
    orc = O.PortStructure(dev.oracle_definition())
    errs = []
    for _ in range(steps):
        if sync:
            sync_oracle_to_device(dev, orc)
        dev.step(settings, diagnostics=False)
        orc.step(settings)
        errs.append(rel_error(dev.node_states(), orc.node_states()))
    return errs, dev, orc


def test_known_answers_on_device(cuda_device):
    d = sw.definition_from_arrays([(0.0, 0.0, 0.0, 2.0, False)])
    s = sw.Structure(d)
    s.add_external_force(0, (4.0, 0.0, 0.0))
    diag = s.step(sw.StepSettings(time_step=0.25, substeps=1, constraint_iterations=0, gravity=(0, 0, -2.0),
                                  velocity_damping=0.0))
    st = s.node_states()
    assert st[0, 2, 0] == pytest.approx(0.5, abs=1e-7)
    assert st[0, 0, 2] == pytest.approx(-0.125, abs=1e-7)
    assert diag.last_applied_external_force.x == 4.0
    assert diag.pending_external_force.x == 0.0
    for kind, length, expected in [(1, 2.0, 1.0), (2, 0.5, 0.5), (2, 2.0, 1.0), (3, 2.0, 1.0)]:
        d = sw.definition_from_arrays([(0.0, 0.0, 0.0, 0.0, True), (length, 0.0, 0.0, 1.0, False)],
                                      constraints=[(kind, 0, 1, 1.0, 0.0)])
        s = sw.Structure(d)
        s.step(sw.StepSettings(time_step=1 / 60, substeps=1, constraint_iterations=1, gravity=(0, 0, 0),
                               velocity_damping=0.0))
        assert s.node_states()[1, 0, 0] == pytest.approx(expected, abs=1e-6)


@pytest.mark.parametrize("ctas", [1, 4, 16])
def test_patch_per_step_parity_cluster(cuda_device, ctas):
    d = sw.generate_patch()
    dev = sw.Structure(d, sw.SolverOptions(cluster_ctas=ctas))
    assert dev.schedule_report().cluster_ctas == ctas
    errs, _, _ = per_step_errors(d, 6, step_settings(), sw.SolverOptions(cluster_ctas=ctas))
    assert max(errs) <= REL_TOL, errs


@pytest.mark.parametrize("blocks,levels", [(1, 1), (8, 1), (8, 3), (148, 3)])
def test_patch_per_step_parity_grid(cuda_device, blocks, levels):
    errs, _, _ = per_step_errors(sw.generate_patch(), 6, step_settings(),
                                 sw.SolverOptions(blocks=blocks, partition_levels=levels, flags=sw.abi.OPT_GRID))
    assert max(errs) <= REL_TOL, errs


def test_patch_global_only_parity(cuda_device):
    errs, _, _ = per_step_errors(sw.generate_patch(nx=17, ny=17), 4, step_settings(),
                                 sw.SolverOptions(blocks=16, flags=sw.abi.OPT_GLOBAL_ONLY))
    assert max(errs) <= REL_TOL, errs


@pytest.mark.parametrize("options", [dict(), dict(cluster_ctas=4), dict(flags=sw.abi.OPT_GRID),
                                     dict(cluster_ctas=4, flags=sw.abi.OPT_SPLIT_STAGES)])
def test_wing_per_step_parity_small(cuda_device, options):
    d = sw.generate_wing(cells=8, chordwise=20, spanwise_per_cell=2, rib_layers=3)
    errs, dev, orc = per_step_errors(d, 4, step_settings(), sw.SolverOptions(**options))
    assert max(errs) <= REL_TOL, errs
    s = dev.suspension_state()
    p, w, _ = orc.payload()
    assert np.abs(s.center_of_mass - [p.center_of_mass.x, p.center_of_mass.y, p.center_of_mass.z]).max() < 1e-4


@pytest.mark.parametrize("options", [dict(), dict(flags=sw.abi.OPT_GRID), dict(flags=sw.abi.OPT_SPLIT_STAGES)])
def test_full_wing_one_step_parity(cuda_device, options):
    errs, dev, _ = per_step_errors(sw.generate_wing(), 2, step_settings(), sw.SolverOptions(**options))
    assert max(errs) <= REL_TOL, errs
    if not options:
        assert dev.schedule_report().cluster_ctas == 16


@pytest.mark.parametrize("case,ctas", [("patch", 1), ("patch", 4), ("patch", 16), ("wing without pilot", 4)])
def test_free_structure_momentum_guard_parity(cuda_device, case, ctas):
    """Structures with no fixed node and no suspension (a patch with no pin,
    a wing without its pilot): the reference restores the predicted linear
    and angular momentum after every substep (soft_body.cpp:152-190,
    1192-1202).  The correction changes velocities only, so velocities and
    the momentum are compared as well as positions.  Tolerances: a velocity
    is a position difference over dt, so the per-step position bound (1e-5
    of the largest coordinate) over dt; the linear and angular momentum of
    the structure within 1e-5 relative (the guard sets both to the predicted
    state's, which FP32 and FP64 compute alike)."""
    d = sw.generate_patch(pin_top_corners=0) if case == "patch" else \
        sw.generate_wing(cells=8, chordwise=16, spanwise_per_cell=2, rib_layers=3, pilot=0)
    options = sw.SolverOptions(cluster_ctas=ctas)
    dev = sw.Structure(d, options)
    orc = O.PortStructure(dev.oracle_definition())
    st = step_settings()
    mass = d.nodes()["mass"].astype(np.float64)

    def momenta(states):
        x, v = states[:, 0, :], states[:, 2, :]
        p = (mass[:, None] * v).sum(axis=0)
        com = (mass[:, None] * x).sum(axis=0) / mass.sum()
        L = (mass[:, None] * np.cross(x - com, v)).sum(axis=0)
        return p, L

    for _ in range(6):
        sync_oracle_to_device(dev, orc)
        dev.step(st, diagnostics=False)
        orc.step(st)
        a, b = dev.node_states(), orc.node_states()
        assert rel_error(a, b) <= REL_TOL
        scale = max(1.0, float(np.abs(b[:, 0, :]).max()))
        assert np.abs(a[:, 2, :] - b[:, 2, :]).max() <= REL_TOL * scale / st.time_step
        (pa, La), (pb, Lb) = momenta(a), momenta(b)
        assert np.abs(pa - pb).max() <= 1e-5 * max(1.0, np.abs(pb).max())
        assert np.abs(La - Lb).max() <= 1e-5 * max(1.0, np.abs(Lb).max())


def test_free_structures_are_refused_where_the_guard_is_not_built(cuda_device):
    d = sw.generate_patch(pin_top_corners=0)
    s = sw.Structure(d)
    with pytest.raises(sw.Unsupported):
        sw.Rollout(s, 4)
    with pytest.raises(sw.Unsupported):
        sw.Structure(d, sw.SolverOptions(flags=sw.abi.OPT_GRID))


@pytest.mark.parametrize("pairs,pilot", [(8, 1), (96, 0)])
def test_wing_cable_pairs_per_step_parity(cuda_device, pairs, pilot):
    """Load-path cable sweeps (soft_body.cpp:528-629, 1265-1388): the
    device's level-scheduled passes against the serial sweeps of the oracle
    on the same depth order (taken from the definition permuted into the
    device sweep order), one step at a time."""
    d = sw.generate_wing(cells=6, chordwise=12, spanwise_per_cell=2, rib_layers=3, pilot=pilot)
    st = step_settings()
    st.cable_sweep_pairs = pairs
    errs, dev, orc = per_step_errors(d, 3, st)
    assert max(errs) <= REL_TOL, errs


def test_cable_pairs_are_refused_where_they_are_not_built(cuda_device):
    d = sw.generate_wing(cells=6, chordwise=12, spanwise_per_cell=2, rib_layers=3)
    st = step_settings()
    st.cable_sweep_pairs = 4
    with pytest.raises(sw.Unsupported):
        sw.Structure(d, sw.SolverOptions(flags=sw.abi.OPT_GRID)).step(st)
    with sw.Batch([d]) as batch:
        with pytest.raises(sw.Unsupported):
            batch.step(st, 1)
    r = sw.Rollout(sw.Structure(d), 4)
    with pytest.raises(sw.Unsupported):
        r.forward(st, np.zeros((d.node_count, 3)), np.ones(d.node_count))


def test_patch_600_steps_settled_shape(cuda_device):
    d = sw.generate_patch()
    dev = sw.Structure(d)
    orc = O.PortStructure(dev.oracle_definition())
    st = step_settings()
    dev.step_many(st, 600)
    for _ in range(600):
        orc.step(st)
    a, b = dev.node_states(), orc.node_states()
    assert np.abs(a[:, 0, :] - b[:, 0, :]).max() <= 1e-3
    da, db = dev.diagnostics(), orc.diagnostics()
    assert abs(da.maximum_distance_error - db.maximum_distance_error) <= 1e-3
    assert dev.accepted_step_count() == 600


def test_checkpoint_replay_is_bitwise(cuda_device):
    d = sw.generate_wing(cells=6, chordwise=12, spanwise_per_cell=2, rib_layers=3)
    s = sw.Structure(d)
    st = step_settings()
    for _ in range(2):
        s.step(st)
    image = s.checkpoint()
    for _ in range(3):
        s.step(st)
    first = s.node_states()
    first_pay = s.suspension_state()
    s.restore(image)
    assert s.accepted_step_count() == 2
    for _ in range(3):
        s.step(st)
    assert np.array_equal(first, s.node_states())
    assert np.array_equal(first_pay.center_of_mass, s.suspension_state().center_of_mass)
    # tampered and foreign images are rejected, state untouched
    bad = bytearray(image)
    bad[100] ^= 0xFF
    with pytest.raises(sw.InvalidArgument):
        s.restore(bytes(bad))
    other = sw.Structure(sw.generate_patch(nx=5, ny=5))
    with pytest.raises(sw.InvalidArgument):
        other.restore(image)
    assert np.array_equal(first, s.node_states())


def test_failed_step_rolls_back_state_and_loads(cuda_device):
    s = sw.Structure(sw.generate_patch(nx=9, ny=9))
    s.add_external_force(3, (1.0, 2.0, 3.0))
    before = s.node_states()
    with pytest.raises(sw.InvalidArgument):
        s.step(sw.StepSettings(time_step=0.0))
    assert np.array_equal(before, s.node_states())
    assert s.diagnostics().pending_external_force.z == 3.0
    with pytest.raises(sw.OutOfRange):
        s.add_external_force(10**6, (0.0, 0.0, 1.0))
    with pytest.raises(sw.InvalidArgument):
        s.add_external_force(0, (float("nan"), 0.0, 0.0))


def test_non_finite_trial_is_rejected_and_rolled_back(cuda_device):
    s = sw.Structure(sw.generate_patch(nx=9, ny=9))
    st = step_settings()
    s.step(st)
    before = s.node_states()
    s.add_external_force(40, (3.0e38, 3.0e38, 3.0e38))
    with pytest.raises(sw.NonFiniteState):
        s.step(st)
    assert np.array_equal(before, s.node_states())
    assert s.accepted_step_count() == 1


def test_suspension_certification_failure_rolls_back(cuda_device):
    d = sw.generate_wing(cells=4, chordwise=10, spanwise_per_cell=2, rib_layers=2)
    d.view.suspension.contents.maximum_line_residual = 0.0
    s = sw.Structure(d)
    before = s.node_states()
    # a zero residual bound fails certification once the risers load
    with pytest.raises(sw.SuspensionError) as err:
        for _ in range(20):
            s.step(step_settings())
    assert s.accepted_step_count() < 20
    # SuspensionError::phase() / entity() as the reference's certifySubstep
    # raises them (suspension.cpp:2350-2358)
    assert (err.value.phase, err.value.entity) == ("Certification", "line-residual")
    if O.ref_available():
        ref = O.RefStructure(d)
        with pytest.raises(O.OracleError) as ref_err:
            for _ in range(20):
                ref.step(step_settings())
        assert (ref_err.value.phase, ref_err.value.entity) == (err.value.phase, err.value.entity)


def test_barrier_timeout_reports_and_restores(cuda_device):
    s = sw.Structure(sw.generate_patch(), sw.SolverOptions(blocks=8, sync_budget_cycles=1, flags=sw.abi.OPT_GRID))
    before = s.node_states()
    with pytest.raises(sw.SyncTimeout):
        s.step(step_settings())
    assert np.array_equal(before, s.node_states())


def test_multi_substep_step_and_rollback(cuda_device):
    d = sw.generate_patch(nx=12, ny=12)
    s = sw.Structure(d)
    orc = O.PortStructure(s.oracle_definition())
    st = step_settings(substeps=3, iterations=16)
    s.step(st)
    orc.step(st)
    assert rel_error(s.node_states(), orc.node_states()) <= REL_TOL


@pytest.mark.parametrize("case", ["patch", "small wing"])
def test_autotuned_structure_keeps_parity(cuda_device, case):
    """SWB_OPT_AUTOTUNE: the candidates are reported, the fastest is kept,
    every candidate's schedule passed the verifier on construction, and the
    chosen one steps like the oracle in its own sweep order."""
    d = sw.generate_patch() if case == "patch" else \
        sw.generate_wing(cells=8, chordwise=20, spanwise_per_cell=2, rib_layers=3)
    opts = sw.SolverOptions(flags=sw.abi.OPT_AUTOTUNE)
    dev = sw.Structure(d, opts)
    report = dev.autotune_report()
    assert len(report) >= 2 and sum(c["chosen"] for c in report) == 1
    chosen = next(c for c in report if c["chosen"])
    assert chosen["ms_per_substep"] == min(c["ms_per_substep"] for c in report)
    r = dev.schedule_report()
    assert (r.cluster_ctas, r.block_threads) == (chosen["cluster_ctas"], chosen["block_threads"])
    orc = O.PortStructure(dev.oracle_definition())
    st = step_settings()
    for _ in range(3):
        sync_oracle_to_device(dev, orc)
        dev.step(st, diagnostics=False)
        orc.step(st)
        assert rel_error(dev.node_states(), orc.node_states()) <= REL_TOL
    assert sw.Structure(d).autotune_report() == []
