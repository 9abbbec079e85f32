"""Steps with fabric self-contact on the device against the reference build.

The reference's Structure (oracle/_ref/libswref.so, with softwing's contact
code) steps the definition permuted into the device sweep order; both start
from the definition and run freely.  Contact keys are ordered alike on both
sides, so the contact projections run in the same order.  Tolerances as for
the other per-step tests: positions within 1e-5 of the largest coordinate
(at least 1 m), velocities within that over the step; the largest
penetration within the position bound; the active contact counts equal.

Hard (zero-compliance) resting contact is decided at a finer scale than an
FP32 state resolves: the swept query calls a feature in contact when its gap
is within 1e-10 m (CcdSettings::distanceTolerance), while FP32 positions of
a sheet 0.35 m from the origin resolve 3e-8 m.  A resting feature is then
in contact (a record with friction) on one side and not on the other, and
which of two redundant features ends with a multiplier of 1e-12 rather than
zero depends on the same rounding; the reference itself moves from 160 to
157 active features when its input is rounded to FP32.  Hard contact is
therefore compared without friction and on whether any feature is active;
compliant contact (1e-3 m/N: resting features sit 1e-5 m inside the
envelope) is compared exactly, friction, active counts and the step at which
the reference's query gives up included.
"""
import numpy as np
import pytest

import simwing_b200 as sw
from oracle import oracle as O
from tests.conftest import step_settings

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not O.ref_available(), reason="reference build not present")]

REL_TOL = 1e-5


def two_sheets():
    """The reference's contact checkpoint fixture (simwing_structure_test.cpp:
    297-329): two disconnected triangles 1 cm apart, half thickness 1 cm."""
    nodes = [(-1, -1, 0, 1.0, 0), (1, -1, 0, 1.0, 0), (0, 1, 0, 1.0, 0),
             (-1, -1, 0.01, 1.0, 0), (0, 1, 0.01, 1.0, 0), (1, -1, 0.01, 1.0, 0)]
    return sw.definition_from_arrays(nodes, [(0, 1, 2), (3, 4, 5)], contact=(0.01, 0.0, 0.0, 0.0))


def stacked_sheets(**kw):
    """A free sheet resting 1 mm inside the contact envelope of a pinned sheet
    below it (simwing_b200.stacked_sheets)."""
    return sw.stacked_sheets(**kw)


SLIDE = step_settings(iterations=8, gravity=(2.0, 0.0, -9.81))  # tilted gravity: static and dynamic friction
# (make, settings, steps, exact active count, step at which the reference
# raises ContactStepError: its swept query cannot certify the resting
# contact, contact.cpp:1318-1325)
CASES = {
    "two_sheets": (two_sheets, step_settings(iterations=4), 6, False, None),
    "stacked_hard": (lambda: stacked_sheets(friction=(0.0, 0.0)), SLIDE, 3, False, None),
    "stacked_compliant": (lambda: stacked_sheets(compliance=1e-3), SLIDE, 4, True, 3),
}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("ctas", [1, 4])
def test_contact_steps_match_the_reference(cuda_device, name, ctas):
    make, st, steps, exact_count, fails_at = CASES[name]
    d = make()
    dev = sw.Structure(d, sw.SolverOptions(cluster_ctas=ctas))
    ref = O.RefStructure(dev.oracle_definition())
    saw_contact = False
    for k in range(steps):
        if k == fails_at:
            before = dev.node_states().copy()
            with pytest.raises(O.OracleError) as err:
                ref.step(st)
            assert err.value.status == sw.abi.CONTACT_ERROR
            with pytest.raises(sw.ContactStepError) as dev_err:
                dev.step(st)
            # both report a feature of the free sheet resting on the pinned
            # one; which resting feature's swept query gives up first
            # depends on the last bits of the positions (FP32 here, FP64
            # there), so the keys are compared only where the failure is
            # not that fine (test_unresolvable_contact...)
            assert dev_err.value.key is not None and dev_err.value.key[1] == err.value.key[1]
            np.testing.assert_array_equal(dev.node_states(), before)
            break
        da = dev.step(st)
        db = ref.step(st)
        a, b = dev.node_states(), ref.node_states()
        scale = max(1.0, float(np.abs(b[:, 0, :]).max()))
        assert float(np.abs(a[:, 0, :] - b[:, 0, :]).max()) <= REL_TOL * scale
        assert float(np.abs(a[:, 2, :] - b[:, 2, :]).max()) <= REL_TOL * scale / st.time_step
        assert da.contact_pair_count == db.contact_pair_count == 1
        if exact_count:
            assert da.active_contact_count == db.active_contact_count
        else:
            assert (da.active_contact_count > 0) == (db.active_contact_count > 0)
        assert abs(da.maximum_contact_penetration - db.maximum_contact_penetration) <= REL_TOL * scale
        assert da.finite and db.finite
        saw_contact = saw_contact or db.active_contact_count > 0
    assert saw_contact


def test_unresolvable_contact_fails_the_step_and_rolls_back(cuda_device):
    """Two pinned sheets inside each other's envelope: no movable or
    compliant response (contact.cpp:1366-1372).  Both solvers raise
    ContactStepError; the device keeps the pre-step state."""
    nodes = [(-1, -1, 0, 1.0, 1), (1, -1, 0, 1.0, 1), (0, 1, 0, 1.0, 1),
             (-1, -1, 0.005, 1.0, 1), (0, 1, 0.005, 1.0, 1), (1, -1, 0.005, 1.0, 1),
             (3, 3, 3, 1.0, 0)]
    d = sw.definition_from_arrays(nodes, [(0, 1, 2), (3, 4, 5)], contact=(0.01, 0.0, 0.0, 0.0))
    st = step_settings(iterations=4)
    dev = sw.Structure(d)
    ref = O.RefStructure(dev.oracle_definition())
    before = dev.node_states().copy()
    with pytest.raises(sw.ContactStepError) as dev_err:
        dev.step(st)
    with pytest.raises(O.OracleError) as err:
        ref.step(st)
    assert err.value.status == sw.abi.CONTACT_ERROR
    # ContactStepError::key(): the feature the reference's key-ordered
    # projection throws at
    assert dev_err.value.key == err.value.key
    np.testing.assert_array_equal(dev.node_states(), before)
    assert dev.accepted_step_count() == 0


def test_contact_is_refused_where_it_is_not_built(cuda_device):
    d = two_sheets()
    with pytest.raises(sw.Unsupported):
        sw.Structure(d, sw.SolverOptions(flags=sw.abi.OPT_GRID))
    with pytest.raises(sw.Unsupported):
        sw.Batch([d, two_sheets()])
    s = sw.Structure(d)
    with pytest.raises(sw.Unsupported):
        sw.Rollout(s, 4)
    with pytest.raises(sw.Unsupported):
        sw.contact_sweep(sw.abi.FEATURE_SEGMENT_TRIANGLE, np.zeros((1, 9)), np.zeros((1, 9)), np.zeros((1, 9)),
                         np.zeros((1, 9)), 0.0)


def key_tuple(k):
    return (k.pair, k.kind, tuple(k.first), tuple(k.second))


@pytest.mark.parametrize("make", [lambda: sw.stacked_sheets(n=16, compliance=1e-3),
                                  lambda: sw.stacked_sheets(n=12, gap=0.001, half_thickness=0.003)])
def test_binned_broadphase_equals_the_exhaustive_list(cuda_device, make):
    """The step's broadphase bins the columns along one axis; its list (the
    certification's, for the last step's start and end positions) must be
    the exhaustive one (swb_contact_candidates), key for key."""
    d = make()
    dev = sw.Structure(d)
    st = SLIDE
    dev.step(st)
    states = dev.node_states()
    keys = dev.contact_candidates()
    h = d.view.fabric_self_contact.contents.half_thickness
    full, _, _ = sw.contact_candidates(d, h, states[:, 1, :], states[:, 0, :])
    assert [key_tuple(k) for k in keys] == [key_tuple(k) for k in full]
    assert len(keys) > 1000


def pilot_sheets():
    """The compliant stacked sheets with a light rigid pilot hanging from
    two nodes of the free sheet by two risers (the payload's line damping
    precedes contact friction, friction precedes the payload's
    certification: soft_body.cpp:1447-1457)."""
    n, spacing = 8, 0.05
    a, b = n * n + 2 * n + 2, n * n + 5 * n + 5
    pa = np.array([2 * spacing + 0.013, 2 * spacing + 0.007, 0.003])
    pb = np.array([5 * spacing + 0.013, 5 * spacing + 0.007, 0.003])
    com = np.array([0.5 * (pa[0] + pb[0]), 0.5 * (pa[1] + pb[1]), -0.6])
    ha, hb = np.array([-0.05, 0.0, 0.2]), np.array([0.05, 0.0, 0.2])
    ra, rb = float(np.linalg.norm(pa - (com + ha))), float(np.linalg.norm(pb - (com + hb)))
    susp = dict(pilot_mass=0.05, pilot_com_world=tuple(com), pilot_inertia=(0.002, 0.002, 0.001),
                attachments=[(1, a), (2, b)], harness=[(1, tuple(ha)), (2, tuple(hb))],
                segments=[(1, (1, 1), (3, 1), ra, 1e3, 0.5), (2, (1, 2), (3, 2), rb, 1e3, 0.5)],
                solver_iterations=8, maximum_line_residual=1e-2)
    return sw.stacked_sheets(n=n, compliance=1e-3, suspension=susp)


@pytest.mark.parametrize("ctas", [1, 4])
def test_contact_with_a_pilot_matches_the_reference(cuda_device, ctas):
    d = pilot_sheets()
    dev = sw.Structure(d, sw.SolverOptions(cluster_ctas=ctas))
    ref = O.RefStructure(dev.oracle_definition())
    da = dev.step(SLIDE)
    db = ref.step(SLIDE)
    a, b = dev.node_states(), ref.node_states()
    assert float(np.abs(a[:, 0, :] - b[:, 0, :]).max()) <= REL_TOL
    assert float(np.abs(a[:, 2, :] - b[:, 2, :]).max()) <= REL_TOL / SLIDE.time_step
    assert da.active_contact_count == db.active_contact_count > 0
    assert abs(da.maximum_contact_penetration - db.maximum_contact_penetration) <= REL_TOL
    pd, pr = dev.suspension_state(), ref.payload()[0]
    np.testing.assert_allclose(pd.center_of_mass, [pr.center_of_mass.x, pr.center_of_mass.y, pr.center_of_mass.z],
                               atol=REL_TOL)
    np.testing.assert_allclose(pd.linear_velocity,
                               [pr.linear_velocity.x, pr.linear_velocity.y, pr.linear_velocity.z],
                               atol=REL_TOL / SLIDE.time_step)
    assert abs(da.maximum_suspension_residual - db.maximum_suspension_residual) <= REL_TOL
    # the resting contact the pilot presses: the reference's swept query gives up
    before = dev.node_states().copy()
    with pytest.raises(O.OracleError) as err:
        ref.step(SLIDE)
    assert err.value.status == sw.abi.CONTACT_ERROR
    with pytest.raises(sw.ContactStepError):
        dev.step(SLIDE)
    np.testing.assert_array_equal(dev.node_states(), before)


def test_candidate_inspection_needs_contact(cuda_device):
    s = sw.Structure(sw.generate_patch(nx=8, ny=8))
    with pytest.raises(sw.Unsupported):
        s.contact_candidates()


@pytest.mark.parametrize("name,warm,replay", [("two_sheets", 0, 3), ("stacked_hard", 2, 1)])
def test_contact_checkpoint_replay_is_bitwise(cuda_device, name, warm, replay):
    """The checkpoint image carries the contact multiplier table (the warm
    starts and the record book that carry over between steps, as
    SoftBodyCheckpoint::State holds contactMultipliers and contactRecords)
    and the contact diagnostics: replay after a restore is bit for bit.  The
    reference's own contact checkpoint fixture (two sheets inside each
    other's envelope, simwing_structure_test.cpp:297-329), whose contact is
    active in the first step, checkpointed before it; and the resting
    stacked sheets, checkpointed after two steps, whose third step (the last
    of the steps the parity test above runs) has active contacts with
    multipliers warm-started from the table the image carries."""
    make, st, _, _, _ = CASES[name]
    d = make()
    s = sw.Structure(d)
    for _ in range(warm):
        s.step(st)
    image = s.checkpoint()
    first = [s.step(st) for _ in range(replay)]
    states = s.node_states()
    s.restore(image)
    assert s.checkpoint() == image
    again = [s.step(st) for _ in range(replay)]
    np.testing.assert_array_equal(s.node_states(), states)
    for a, b in zip(first, again):
        assert a.active_contact_count == b.active_contact_count
        assert a.maximum_contact_penetration == b.maximum_contact_penetration
    assert first[0].active_contact_count > 0 if warm == 0 else all(a.active_contact_count > 0 for a in first)
    # a tampered image is refused, the state untouched
    bad = bytearray(image)
    bad[-60] ^= 0x40
    with pytest.raises(sw.InvalidArgument):
        s.restore(bytes(bad))
    np.testing.assert_array_equal(s.node_states(), states)


@pytest.mark.parametrize("failure", ["contact", "non_finite"])
def test_failed_contact_step_restores_the_multiplier_table(cuda_device, failure):
    """A failed step rolls the contact multiplier table back with the nodes
    (soft_body.cpp:1090-1112): afterwards the structure is byte for byte the
    one that never tried the step."""
    d = stacked_sheets(compliance=1e-3)
    tried, twin = sw.Structure(d), sw.Structure(d)
    steps = 3 if failure == "contact" else 2
    for _ in range(steps):
        tried.step(SLIDE)
        twin.step(SLIDE)
    if failure == "non_finite":
        last = d.node_count - 1  # a node of the free sheet
        for s in (tried, twin):
            s.add_external_force(last, (3.0e38, 3.0e38, 3.0e38))
    before = tried.checkpoint()
    # the compliant stacked sheets' fourth step fails in the swept query, as
    # the reference's does (see CASES)
    # a non-finite prediction is refused by the contact broadphase (its
    # inputs must be finite) or by the finite-state check, whichever reads it
    # first; either way the step fails as a whole
    with pytest.raises(sw.ContactStepError if failure == "contact" else (sw.NonFiniteState, sw.ContactStepError)):
        tried.step(SLIDE)
    assert tried.checkpoint() == before == twin.checkpoint()


@pytest.mark.parametrize("name", ["two_sheets", "stacked_hard", "stacked_compliant"])
def test_helper_clusters_change_nothing(cuda_device, name):
    """The detection phases (broadphase, swept queries) run over helper
    clusters beside the structure's cluster by default; the candidate lists
    and queries, and so the steps, are bit for bit those of the structure's
    cluster alone (SWB_OPT_CONTACT_ONE_CLUSTER)."""
    make, st, steps, _, fails_at = CASES[name]
    d = make()
    a = sw.Structure(d)
    b = sw.Structure(d, sw.SolverOptions(flags=sw.abi.OPT_CONTACT_ONE_CLUSTER))
    for k in range(steps if fails_at is None else fails_at):
        ga, gb = a.step(st), b.step(st)
        assert ga.active_contact_count == gb.active_contact_count
        assert ga.maximum_contact_penetration == gb.maximum_contact_penetration
        np.testing.assert_array_equal(a.node_states(), b.node_states())


def test_helper_clusters_on_a_large_scene(cuda_device):
    """The same on 48 x 48 stacked sheets (a candidate list of about 100,000
    features spread over every cluster), three consecutive steps."""
    d = stacked_sheets(n=48, compliance=1e-3)
    a = sw.Structure(d)
    b = sw.Structure(d, sw.SolverOptions(flags=sw.abi.OPT_CONTACT_ONE_CLUSTER))
    for _ in range(3):
        ga, gb = a.step(SLIDE), b.step(SLIDE)
        assert ga.active_contact_count == gb.active_contact_count
    np.testing.assert_array_equal(a.node_states(), b.node_states())
