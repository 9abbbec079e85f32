"""Coupling callers with device-resident loads (swb_coupling_*): the
structural side of ConservativeMacroStepCoupling::advanceStructure and
advanceStructureWithEndpointLoads (coupling.cpp:806-911).

The reference converts each binding's load to an average force
(impulse x (1 / duration), or the mean of the endpoint loads), adds it to
its structure node with addExternalForce in binding order, and steps.  The
device path gathers the same sums from device memory into the step's force
buffer, so both paths must give the same state bit for bit.
"""
import numpy as np
import pytest

import simwing_b200 as sw
from tests.conftest import step_settings

pytestmark = pytest.mark.gpu


def case(seed=3):
    d = sw.generate_patch(nx=12, ny=12, seed=seed)
    n = d.view.node_count
    rng = np.random.default_rng(seed)
    # 300 interface nodes; several load the same structure node
    nodes = rng.integers(0, n, size=300).astype(np.uint64)
    return d, nodes, rng


def pair(d):
    return sw.Structure(d, sw.SolverOptions(cluster_ctas=4)), sw.Structure(d, sw.SolverOptions(cluster_ctas=4))


def test_impulses_from_device_memory_equal_the_add_external_force_path(cuda_device):
    import torch

    d, nodes, rng = case()
    st = step_settings(iterations=16)
    host, dev = pair(d)
    coupling = sw.Coupling(dev, nodes)
    # loads already pending before the macro-step
    for node in (3, 17, 17, 40):
        f = rng.normal(size=3)
        host.add_external_force(node, f)
        dev.add_external_force(node, f)
    for _ in range(3):
        impulses = rng.normal(scale=1e-3, size=(len(nodes), 3))
        scale = 1.0 / st.time_step
        for node, imp in zip(nodes, impulses):
            host.add_external_force(int(node), imp * scale)
        da = host.step(st)
        db = coupling.advance_impulses(torch.tensor(impulses, dtype=torch.float64, device="cuda"), st.time_step, st)
        np.testing.assert_array_equal(dev.node_states(), host.node_states())
        for f in ("x", "y", "z"):
            assert getattr(db.last_applied_external_force, f) == pytest.approx(
                getattr(da.last_applied_external_force, f), rel=1e-12, abs=1e-15)
        assert db.pending_external_force.x == da.pending_external_force.x == 0.0
    coupling.close()


def test_endpoint_loads_from_device_memory(cuda_device):
    import torch

    d, nodes, rng = case(5)
    st = step_settings(iterations=16)
    host, dev = pair(d)
    coupling = sw.Coupling(dev, nodes)
    start = rng.normal(size=(len(nodes), 3))
    end = rng.normal(size=(len(nodes), 3))
    for node, a, b in zip(nodes, start, end):
        host.add_external_force(int(node), 0.5 * (a + b))
    host.step(st)
    coupling.advance_endpoint_loads(torch.tensor(start, device="cuda"), torch.tensor(end, device="cuda"), st)
    np.testing.assert_array_equal(dev.node_states(), host.node_states())


def test_invalid_transfers_are_refused_and_keep_the_pending_loads(cuda_device):
    import torch

    d, nodes, rng = case(7)
    st = step_settings(iterations=16)
    host, dev = pair(d)
    coupling = sw.Coupling(dev, nodes)
    for s in (host, dev):
        s.add_external_force(5, (0.0, 0.0, 2.0))
    before = dev.node_states().copy()
    bad = rng.normal(size=(len(nodes), 3))
    bad[17, 1] = np.nan
    with pytest.raises(sw.InvalidArgument):
        coupling.advance_impulses(torch.tensor(bad, device="cuda"), st.time_step, st)
    with pytest.raises(sw.InvalidArgument):  # the duration must be the step's
        coupling.advance_impulses(torch.zeros((len(nodes), 3), dtype=torch.float64, device="cuda"),
                                  0.5 * st.time_step, st)
    np.testing.assert_array_equal(dev.node_states(), before)
    assert dev.accepted_step_count() == 0
    # the loads pending before the refused calls still apply on the next step
    host.step(st)
    dev.step(st)
    np.testing.assert_array_equal(dev.node_states(), host.node_states())
    with pytest.raises(sw.OutOfRange):
        sw.Coupling(dev, [d.view.node_count])


def test_a_batch_structure_is_not_coupled(cuda_device):
    """A structure of a batch steps with its batch's launches."""
    defs = [sw.generate_patch(nx=8, ny=8, seed=1), sw.generate_patch(nx=9, ny=9, seed=2)]
    with sw.Batch(defs) as batch:
        with pytest.raises(sw.Unsupported):
            sw.Coupling(batch.structure(0), [0, 1, 2])
