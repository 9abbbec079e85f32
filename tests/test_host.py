"""Host-side logic without a GPU: the C-ABI library loads and exports every
declared entry point, definition validation mirrors Structure's
validateDefinition (structure.cpp:102-291), the fingerprint and the
reference colouring are bit-exact with the reference, the generators emit
the configured shapes, and the device schedule satisfies its invariants."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import simwing_b200 as sw
from simwing_b200 import abi
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = np.load(os.path.join(ROOT, "tests", "golden", "trajectories.npz"))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "simwing_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(swb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(abi.LIBRARY_PATH)
    names = declared_functions()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(abi.DECLARED_SYMBOLS) <= set(names)
    assert abi.library().swb_abi_version() == 1


def test_default_settings_match_reference():
    s = sw.StepSettings()
    assert s.time_step == 1.0 / 120.0 and s.substeps == 2 and s.constraint_iterations == 12
    assert s.gravity.z == -9.80665 and s.velocity_damping == 0.25 and s.cable_sweep_pairs == 0


@pytest.mark.parametrize("bad", [
    dict(nodes=[(0, 0, 0, 0.0, False)]),                               # dynamic node without mass
    dict(nodes=[(0, 0, 0, -1.0, True)]),                               # negative mass
    dict(nodes=[(float("nan"), 0, 0, 1.0, False)]),                    # non-finite position
    dict(triangles=[(0, 1, 1)]),                                       # repeated node
    dict(triangles=[(0, 1, 9)]),                                       # unknown node
    dict(constraints=[(1, 0, 0, 1.0, 0.0)]),                           # self constraint
    dict(constraints=[(1, 0, 1, -1.0, 0.0)]),                          # negative rest
    dict(constraints=[(4, 0, 1, 0.5, 0.0)]),                           # seam stitch with rest
    dict(constraints=[(9, 0, 1, 1.0, 0.0)]),                           # unknown kind
    dict(dihedrals=[(0, 1, 2, 2, 0.0, 0.0)]),                          # repeated dihedral node
    dict(dihedrals=[(0, 1, 2, 3, 0.0, -1.0)]),                         # negative compliance
])
def test_validation_rejects_like_the_reference(bad):
    base = dict(nodes=[(0, 0, 0, 1.0, False), (1, 0, 0, 1.0, False), (0, 1, 0, 1.0, False), (1, 1, 0, 1.0, False)])
    base.update(bad)
    d = sw.definition_from_arrays(**base)
    with pytest.raises(sw.InvalidArgument):
        d.validate()
    if O.ref_available():
        with pytest.raises(O.OracleError) as e:
            O.RefStructure(d)
        assert e.value.status == abi.INVALID_ARGUMENT


def test_suspension_validation():
    nodes = [(0, 0, 0, 1.0, False), (0, 0, -1, 1.0, False)]
    good = dict(attachments=[(1, 1)], harness=[(1, (0, 0, 0.2))],
                segments=[(1, (1, 1), (3, 1), 0.5, 1e4, 0.0)], pilot_com_world=(0, 0, -1.7))
    sw.definition_from_arrays(nodes, suspension=good).validate()
    for change in (dict(pilot_mass=0.0), dict(segments=[(1, (1, 1), (3, 1), -0.5, 1e4, 0.0)]),
                   dict(attachments=[(0, 1)]), dict(solver_iterations=0)):
        bad = dict(good, **change)
        with pytest.raises(sw.InvalidArgument):
            sw.definition_from_arrays(nodes, suspension=bad).validate()


def golden_definition(name):
    if name == "patch":
        return sw.generate_patch(nx=17, ny=17, seed=7)
    if name == "membrane_patch":
        return sw.generate_patch(nx=12, ny=12, seed=9, membranes=2)
    return sw.generate_wing(cells=4, chordwise=10, spanwise_per_cell=2, rib_layers=2, seed=3)


@pytest.mark.parametrize("name", ["patch", "wing", "membrane_patch"])
def test_fingerprint_matches_reference_golden(name):
    d = golden_definition(name)
    if name == "wing":
        # the reference definition has no face pressure; hash without it
        t = d.triangles()
        t["pressure_difference"] = 0.0
    assert d.fingerprint == int(GOLDEN[f"{name}_fingerprint"])


@pytest.mark.parametrize("name", ["patch", "wing", "membrane_patch"])
def test_reference_colouring_is_bit_exact(name):
    d = golden_definition(name)
    order, offsets, parallel = sw.reference_colouring(d)
    np.testing.assert_array_equal(order, GOLDEN[f"{name}_colour_order"])
    np.testing.assert_array_equal(offsets, GOLDEN[f"{name}_colour_offsets"])
    assert parallel == int(GOLDEN[f"{name}_parallel_colours"])


def test_reference_colouring_on_full_wing_against_reference_build():
    if not O.ref_available():
        pytest.skip("reference build not present")
    d = sw.generate_wing()
    mine = sw.reference_colouring(d)
    ref = O.ref_colouring(d)
    np.testing.assert_array_equal(mine[0], ref[0])
    np.testing.assert_array_equal(mine[1], ref[1])
    assert mine[2] == ref[2]


def test_patch_generator_shape():
    d = sw.generate_patch()
    c = d.counts()
    assert (c["nodes"], c["triangles"], c["distance"], c["dihedrals"]) == (1089, 2048, 3136, 3008)
    n = d.nodes()
    assert int(n["fixed"].sum()) == 2
    total = n["mass"].sum()
    assert total == pytest.approx(0.040, rel=1e-12)  # 40 g/m^2 on 1 m^2
    assert sw.generate_patch().fingerprint == d.fingerprint
    assert sw.generate_patch(seed=2).fingerprint != d.fingerprint


def test_wing_generator_shape():
    d = sw.generate_wing()
    c = d.counts()
    assert 65000 <= c["triangles"] <= 72000
    assert 36000 <= c["nodes"] <= 40000
    assert c["suspension_segments"] == 2
    assert c["seam_stitch"] == 41 * (120 - 2)  # every rib sewn except next to the trailing edge
    assert 2000 <= c["cable"] <= 3000
    assert 95000 <= c["dihedrals"] <= 105000
    assert sw.generate_wing().fingerprint == d.fingerprint


@pytest.mark.parametrize("levels", [1, 2, 3, 4])
@pytest.mark.parametrize("blocks", [1, 7, 148])
def test_schedule_invariants_patch(levels, blocks):
    d = sw.generate_patch(nx=20, ny=20)
    r, do, ho = sw.plan_schedule(d, sw.SolverOptions(blocks=blocks, partition_levels=levels, flags=abi.OPT_GRID))
    assert sorted(do.tolist()) == list(range(d.view.constraint_count))
    assert sorted(ho.tolist()) == list(range(d.view.dihedral_count))
    assert r.blocks == min(blocks, d.node_count)


@pytest.mark.parametrize("split", [False, True])
@pytest.mark.parametrize("ctas", [1, 2, 4, 8, 16])
def test_cluster_schedule_invariants(ctas, split):
    # plan_schedule runs the host verifier: node-disjoint stages, and within
    # every run of stages joined by CTA barriers each node touched by one CTA
    d = sw.generate_wing(cells=8, chordwise=16, spanwise_per_cell=2, rib_layers=3)
    flags = abi.OPT_SPLIT_STAGES if split else 0
    r, do, ho = sw.plan_schedule(d, sw.SolverOptions(cluster_ctas=ctas, flags=flags))
    assert r.cluster_ctas == ctas
    assert sorted(do.tolist()) == list(range(d.view.constraint_count))
    assert sorted(ho.tolist()) == list(range(d.view.dihedral_count))
    if not split or ctas == 1:
        # the last two stages touch no suspension node: the line iteration
        # runs beside them and takes no cluster barrier of its own
        assert r.cluster_barriers_per_iteration == r.local_stages_per_iteration
    else:
        assert r.cluster_barriers_per_iteration < r.local_stages_per_iteration + 1


def test_split_stages_cut_cluster_barriers_on_the_full_wing():
    """Split stages: the stages of records inside one CTA's patch end in CTA
    barriers, so fewer cluster barriers than the classic schedule's one per
    stage (the schedule verifier checks that no node is touched by two CTAs
    between cluster barriers)."""
    d = sw.generate_wing()
    classic, _, _ = sw.plan_schedule(d)
    split, _, _ = sw.plan_schedule(d, sw.SolverOptions(flags=abi.OPT_SPLIT_STAGES))
    assert classic.cluster_barriers_per_iteration == classic.local_stages_per_iteration
    assert split.cluster_barriers_per_iteration < classic.cluster_barriers_per_iteration
    assert split.local_stages_per_iteration > split.cluster_barriers_per_iteration


def test_full_wing_fits_one_cluster():
    r, _, _ = sw.plan_schedule(sw.generate_wing())
    assert r.cluster_ctas == 16 and r.max_patch_nodes <= 4096
    assert r.shared_bytes <= 227 * 1024


def test_schedule_invariants_wing_and_global_only():
    d = sw.generate_wing(cells=8, chordwise=16, spanwise_per_cell=2, rib_layers=3)
    r, _, _ = sw.plan_schedule(d, sw.SolverOptions(blocks=148, flags=abi.OPT_GRID))
    assert r.level_constraints[0] > 0
    r, _, _ = sw.plan_schedule(d, sw.SolverOptions(blocks=32, flags=abi.OPT_GLOBAL_ONLY))
    assert r.partition_levels == 0 and r.global_constraints == d.view.constraint_count + d.view.dihedral_count


def test_full_wing_schedule_invariants():
    d = sw.generate_wing()
    r, do, ho = sw.plan_schedule(d, sw.SolverOptions(blocks=148, flags=abi.OPT_GRID))
    total = d.view.constraint_count + d.view.dihedral_count
    assert sum(r.level_constraints) + r.global_constraints == total
    assert r.max_patch_nodes < 65536


def test_bench_workload_counts_match_the_generator():
    """The bench line names the wing by its counts; they must be the
    generator's."""
    import bench

    c = sw.generate_wing().counts()
    text = bench.wing_config()["workload"]
    assert f"{c['triangles']:,} tri" in text and f"{c['nodes']:,} nodes" in text
