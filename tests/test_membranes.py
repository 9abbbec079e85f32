"""Membrane elements on the device (the orthotropic XPBD element of
soft_body.cpp:1822-1929) against the FP64 oracle, whose membrane
restatement is pinned bit for bit to the reference build in test_oracle.py.

The oracle runs the definition permuted into the device sweep order
(distance, membrane and dihedral lists alike), from the device's state, so
both take the same Gauss-Seidel sweep.  Tolerances:
  * positions after one step: 1e-5 of the largest coordinate (FP32 device).
    On the full fabric wing the first step from rest inflates the canopy by
    about 20 mm against 1.6 mm elements of 5e-7 kg nodes at the tip's
    trailing-edge closure, and the reference algorithm itself amplifies FP32
    rounding there: the oracle with every vector result rounded to FP32
    (PortStructure(float_vectors=True)) leaves the FP64 oracle by up to
    7.5e-5 m at two nodes while 99 % of nodes agree to 1.2e-6 m.  A second
    measure of the same sensitivity is the FP64 oracle started from the
    device state with every position moved by N(0, 1e-7 m), the rounding of
    an FP32 coordinate of a metre.  The wing test bounds the device by the
    larger of 1e-5 relative and four times the larger of the two measured
    sensitivities, and requires 99.9 % of the nodes to meet 1e-5 relative;
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
import simwing_b200.abi as abi
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


def shortest_chart_edge(definition):
    chart = np.ctypeslib.as_array(definition.view.membranes, shape=(definition.view.membrane_count,))["chart"]
    edges = [np.linalg.norm(chart[:, (k + 1) % 3] - chart[:, k], axis=1) for k in range(3)]
    return float(np.min(edges))


@pytest.mark.parametrize("size,ctas,steps", [("small", 4, 4), ("full", 16, 2)])
def test_membrane_wing_per_step_parity(cuda_device, size, ctas, steps):
    """The wing with membrane fabric, lines and the rigid pilot."""
    d = sw.generate_wing(fabric=1) if size == "full" else \
        sw.generate_wing(cells=8, chordwise=20, spanwise_per_cell=2, rib_layers=3, fabric=1)
    dev = sw.Structure(d, sw.SolverOptions(cluster_ctas=ctas))
    orc = O.PortStructure(dev.oracle_definition())
    st = step_settings()
    edge = shortest_chart_edge(d)
    f32 = O.PortStructure(dev.oracle_definition(), float_vectors=True)
    moved = O.PortStructure(dev.oracle_definition())
    rng = np.random.default_rng(7)
    for _ in range(steps):
        s = dev.suspension_state()
        payload = abi.PayloadState(abi.Vec3(*s.center_of_mass), abi.Quat(*s.body_to_world),
                                   abi.Vec3(*s.linear_velocity), abi.Vec3(*s.angular_velocity))
        for o in (orc, f32, moved):
            sync(dev, o)
            o.write_payload(payload)
        x = moved.node_states()
        x[:, 0, :] += rng.normal(0.0, 1e-7, x[:, 0, :].shape)
        moved.write_node_states(x)
        da = dev.step(st)
        db = orc.step(st)
        f32.step(st)
        moved.step(st)
        a, b = dev.node_states(), orc.node_states()
        scale = max(1.0, float(np.abs(b[:, 0, :]).max()))
        err = np.abs(a[:, 0, :] - b[:, 0, :]).max(axis=1)
        dx = float(err.max())
        sensitivity = max(float(np.abs(f32.node_states()[:, 0, :] - b[:, 0, :]).max()),
                          float(np.abs(moved.node_states()[:, 0, :] - b[:, 0, :]).max()))
        assert dx <= max(REL_TOL * scale, 4.0 * sensitivity)
        assert np.count_nonzero(err > REL_TOL * scale) <= 1e-3 * err.size
        lip = 4.0 * dx / edge
        assert abs(da.maximum_absolute_membrane_strain - db.maximum_absolute_membrane_strain) <= lip + 1e-7
        assert abs(da.maximum_membrane_residual - db.maximum_membrane_residual) <= \
            0.05 * db.maximum_membrane_residual + lip + 1e-7


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
