"""Membrane elements on the device (the orthotropic XPBD element of
soft_body.cpp:1822-1929) against the FP64 oracle, whose membrane
restatement is pinned bit for bit to the reference build in test_oracle.py.

The oracle runs the definition permuted into the device sweep order
(distance, membrane and dihedral lists alike), from the device's state, so
both take the same Gauss-Seidel sweep.  Tolerances:
  * positions after one step: 1e-5 of the largest coordinate (FP32 device);
  * the largest membrane strain: the strain is Lipschitz in the corner
    positions with constant about 2 / (shortest chart edge), so the bound is
    4 x (largest position difference) / (shortest edge) + 1e-7;
  * the largest normalized residual: 5 % of the oracle's plus the same
    position term (the residual is a difference of terms of the size of the
    strain, computed in FP32).
"""
import numpy as np
import pytest

import simwing_b200 as sw
from oracle import oracle as O
from tests.conftest import step_settings

pytestmark = pytest.mark.gpu

REL_TOL = 1e-5


def sync(dev, orc):
    orc.write_node_states(dev.node_states())


@pytest.mark.parametrize("option,pinned,ctas", [(1, 1, 1), (1, 1, 4), (2, 1, 16), (2, 0, 4)])
def test_membrane_patch_per_step_parity(cuda_device, option, pinned, ctas):
    """Linear material (1); pre-tension, damping and compression softening
    (2); pinned and free (the free patch also runs the momentum guard)."""
    d = sw.generate_patch(membranes=option, pin_top_corners=pinned)
    dev = sw.Structure(d, sw.SolverOptions(cluster_ctas=ctas))
    assert dev.schedule_report().cluster_ctas == ctas
    orc = O.PortStructure(dev.oracle_definition())
    st = step_settings()
    edge = 1.0 / 32.0  # shortest chart edge of the 33 x 33 sheet
    for _ in range(4):
        sync(dev, orc)
        da = dev.step(st)
        db = orc.step(st)
        a, b = dev.node_states(), orc.node_states()
        scale = max(1.0, float(np.abs(b[:, 0, :]).max()))
        dx = float(np.abs(a[:, 0, :] - b[:, 0, :]).max())
        assert dx <= REL_TOL * scale
        assert da.membrane_count == db.membrane_count == d.view.triangle_count
        assert da.finite and db.finite
        lip = 4.0 * dx / edge
        assert abs(da.maximum_absolute_membrane_strain - db.maximum_absolute_membrane_strain) <= lip + 1e-7
        assert abs(da.maximum_membrane_residual - db.maximum_membrane_residual) <= \
            0.05 * db.maximum_membrane_residual + lip + 1e-7
        assert db.maximum_membrane_residual > 0.0


def test_batch_with_membranes_matches_plain_structures_bitwise(cuda_device):
    defs = [sw.generate_patch(nx=20, ny=20, membranes=2, seed=3),
            sw.generate_wing(cells=6, chordwise=12, spanwise_per_cell=2, rib_layers=2, seed=4),
            sw.generate_patch(nx=24, ny=24, membranes=1, pin_top_corners=0, seed=5)]
    st = step_settings()
    with sw.Batch(defs, sw.BatchOptions(target_patch_nodes=512, graph_steps=2)) as batch:
        statuses = batch.step(st, 3)
        assert not statuses.any()
        for i, d in enumerate(defs):
            ranks = batch.structure(i).schedule_report().cluster_ctas
            plain = sw.Structure(d, sw.SolverOptions(cluster_ctas=ranks))
            for _ in range(3):
                plain.step(st, diagnostics=False)
            np.testing.assert_array_equal(batch.structure(i).node_states(), plain.node_states())
            plain.close()


def test_membranes_are_refused_where_they_are_not_built(cuda_device):
    d = sw.generate_patch(nx=12, ny=12, membranes=1)
    with pytest.raises(sw.Unsupported):
        sw.Structure(d, sw.SolverOptions(flags=sw.abi.OPT_GRID))
    s = sw.Structure(d)
    with pytest.raises(sw.Unsupported):
        sw.Rollout(s, 4)
