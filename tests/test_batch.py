"""Batched structures (swb_batch_*): many structures of uneven sizes in one
packed cluster launch per substep, blocks of steps in a CUDA graph.

Pinning: every structure of a batch must step bit for bit like a plain
structure built with the same cluster rank count (same schedule, same
arithmetic), and through that like the FP64 oracle within the plain
solver's 1e-5 per-step tolerance.  A failure in one structure must leave
the others committed and the failed one at its state before the block."""
import numpy as np
import pytest

import simwing_b200 as sw
from simwing_b200 import abi
from oracle import oracle as O
from tests.conftest import step_settings
from tests.test_gpu_parity import sync_oracle_to_device

pytestmark = pytest.mark.gpu


def mixed_definitions():
    """Uneven sizes, with and without pilot, a cloth patch among wings."""
    return [
        sw.generate_wing(cells=8, chordwise=16, spanwise_per_cell=2, rib_layers=3, seed=1),
        sw.generate_patch(nx=20, ny=20, seed=2),
        sw.generate_wing(cells=12, chordwise=20, spanwise_per_cell=2, rib_layers=3, seed=3, pilot=0),
        sw.generate_wing(cells=6, chordwise=12, spanwise_per_cell=2, rib_layers=2, seed=4, compliance_jitter=0.2),
        sw.generate_patch(nx=33, ny=33, seed=5),
        sw.generate_wing(cells=20, chordwise=30, seed=6),
    ]


def plain_twin(batch, i, definition):
    ranks = batch.structure(i).schedule_report().cluster_ctas
    return sw.Structure(definition, sw.SolverOptions(cluster_ctas=ranks))


@pytest.mark.parametrize("flags", [0, abi.OPT_NO_GRAPH])
def test_batch_matches_plain_structures_bitwise(cuda_device, flags):
    defs = mixed_definitions()
    st = step_settings()
    with sw.Batch(defs, sw.BatchOptions(target_patch_nodes=512, graph_steps=2, flags=flags)) as batch:
        rep = batch.report()
        assert rep.structures == len(defs) and rep.clusters >= 1
        statuses = batch.step(st, 5)  # blocks of 2, 2, 1 steps
        assert not statuses.any()
        for i, d in enumerate(defs):
            plain = plain_twin(batch, i, d)
            for _ in range(5):
                plain.step(st, diagnostics=False)
            got = batch.structure(i).node_states()
            np.testing.assert_array_equal(got, plain.node_states())
            assert batch.structure(i).accepted_step_count() == 5
            if d.has_suspension:
                a, b = batch.structure(i).suspension_state(), plain.suspension_state()
                np.testing.assert_array_equal(a.center_of_mass, b.center_of_mass)
            plain.close()


def test_batch_structures_match_the_oracle_per_step(cuda_device):
    defs = mixed_definitions()[:4]
    st = step_settings()
    with sw.Batch(defs, sw.BatchOptions(target_patch_nodes=512)) as batch:
        oracles = [O.PortStructure(batch.structure(i).oracle_definition()) for i in range(len(defs))]
        for _ in range(3):
            for i, orc in enumerate(oracles):
                sync_oracle_to_device(batch.structure(i), orc)
            batch.step(st, 1)
            for i, orc in enumerate(oracles):
                orc.step(st)
                ref = orc.node_states()
                got = batch.structure(i).node_states()
                scale = max(1.0, float(np.abs(ref[:, 0, :]).max()))
                err = float(np.abs(got[:, 0, :] - ref[:, 0, :]).max()) / scale
                assert err <= 1e-5, (i, err)


def test_batch_failure_is_isolated_and_rolled_back(cuda_device):
    defs = mixed_definitions()[:3]
    st = step_settings()
    with sw.Batch(defs, sw.BatchOptions(target_patch_nodes=512, graph_steps=3)) as batch:
        batch.step(st, 1)
        before = [batch.structure(i).node_states() for i in range(len(defs))]
        counts = [batch.structure(i).accepted_step_count() for i in range(len(defs))]
        # a load that overflows FP32 makes structure 1's trial state non-finite
        forces = np.zeros((batch.structure(1).node_count, 3))
        forces[5] = (0.0, 0.0, 1e38)
        batch.structure(1).set_external_forces(forces)
        with pytest.raises(sw.NonFiniteState) as e:
            batch.step(st, 3)
        assert e.value.statuses[1] == abi.NON_FINITE
        assert e.value.statuses[0] == abi.OK and e.value.statuses[2] == abi.OK
        np.testing.assert_array_equal(batch.structure(1).node_states(), before[1])
        assert batch.structure(1).accepted_step_count() == counts[1]
        assert batch.structure(1).diagnostics().pending_external_force.z == 1e38  # load kept
        for i in (0, 2):
            assert batch.structure(i).accepted_step_count() == counts[i] + 3
            plain = plain_twin(batch, i, defs[i])
            for _ in range(4):
                plain.step(st, diagnostics=False)
            np.testing.assert_array_equal(batch.structure(i).node_states(), plain.node_states())
            plain.close()


def test_batch_autotune_times_candidates(cuda_device):
    """The batch autotuner times three patch sizes, each with two block
    sizes (enough threads for the widest stage, and 512), and keeps the
    fastest pair."""
    defs = mixed_definitions()[:3]
    with sw.Batch(defs, sw.BatchOptions(flags=abi.BATCH_AUTOTUNE)) as batch:
        rep = batch.report()
        n = rep.autotune_candidates
        assert n == 6
        pairs = {(rep.candidate_patch_nodes[k], rep.candidate_block_threads[k]) for k in range(n)}
        assert pairs == {(p, t) for p in (1024, 2048, 4096) for t in (0, 512)}
        ms = [rep.candidate_ms_per_step[k] for k in range(n)]
        assert all(m > 0 for m in ms)
        best = min(range(n), key=lambda k: ms[k])
        assert rep.target_patch_nodes == rep.candidate_patch_nodes[best]
        if rep.candidate_block_threads[best]:
            assert rep.block_threads == rep.candidate_block_threads[best]
        batch.step(step_settings(), 2)
        assert all(batch.structure(i).accepted_step_count() == 2 for i in range(len(defs)))
