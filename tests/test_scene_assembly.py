"""Scene assembly (swb_assemble_scene) against the reference's
assembleSceneStructure (src/fsi/scene_structure.cpp:894-1284), compiled into
oracle/_ref, on the same scenes.

A small canopy scene: a closed skin sheet swept along the span, a separately
meshed rib sheet at every station sewn to the skin by a seam (coincident
vertex pairs), suspension lines from bottom-skin attachments through
junctions to the harness points of a rigid pilot, entities given in shuffled
order.  The assembled definitions must be identical field for field (the
integer topology and every double, the lumped masses accumulated in long
double as the reference does), the definition fingerprints equal, and the
totals equal.  Without the pilot the lines become nodal cables.  Each
refusal case must fail on both sides with the same first diagnostic
(code, scene validation code, entity kind and ID)."""
import copy

import numpy as np
import pytest

import simwing_b200 as sw
from simwing_b200 import abi
from oracle import oracle as O

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference build not present")


def chart_of(p):
    """The triangle's own rest shape in its plane: positive area by
    construction."""
    a, b, c = p
    u = (b - a) / np.linalg.norm(b - a)
    n = np.cross(b - a, c - a)
    n /= np.linalg.norm(n)
    v = np.cross(n, u)
    return [(0.0, 0.0), (float(np.dot(b - a, u)), float(np.dot(b - a, v))),
            (float(np.dot(c - a, u)), float(np.dot(c - a, v)))]


def canopy(stations=4, loop=10, pilot=True, seed=0):
    """Scene items (lists of abi records) of the small canopy."""
    rng = np.random.default_rng(seed)
    ids = iter(rng.permutation(np.arange(1000, 100000)).tolist())
    items = {k: [] for k, _, _ in abi.SCENE_ARRAYS}
    pos = {}

    def vertex(p):
        i = next(ids)
        pos[i] = np.asarray(p, dtype=float)
        items["vertex"].append(abi.SceneVertex(i, abi.Vec3(*p)))
        return i

    def fabric(bending, warp=4e4):
        i = next(ids)
        items["fabric"].append(abi.SceneFabric(i, warp, 3e4, 1.5e3, bending, 0.045, 0.01, 0.0, 0.0))
        return i

    skin_mat, rib_mat = fabric(1e-3), fabric(2e-3, warp=5e4)

    def triangle(a, b, c, mat, sheet):
        chart = tuple(tuple(x) for x in chart_of([pos[a], pos[b], pos[c]]))
        items["triangle"].append(abi.SceneTriangle(next(ids), (a, b, c), chart, mat, sheet))

    ring = []
    for s in range(stations):
        y = 0.6 * s
        ring.append([vertex((0.5 * np.cos(2 * np.pi * k / loop) + 0.01 * rng.normal(), y,
                             0.12 * np.sin(2 * np.pi * k / loop) + 0.01 * rng.normal())) for k in range(loop)])
    skin_sheet = next(ids)
    for s in range(stations - 1):
        for k in range(loop):
            a, b = ring[s][k], ring[s][(k + 1) % loop]
            c, d = ring[s + 1][(k + 1) % loop], ring[s + 1][k]
            triangle(a, b, c, skin_mat, skin_sheet)
            triangle(a, c, d, skin_mat, skin_sheet)
    seam_mat = next(ids)
    items["seam_material"].append(abi.SceneSeamMaterial(seam_mat, 0.02, 1e5))
    for s in range(stations):
        # rib: its own boundary vertices at the skin's, a fan from its centre
        rib = [vertex(pos[v]) for v in ring[s]]
        centre = vertex(np.mean([pos[v] for v in rib], axis=0))
        sheet = next(ids)
        for k in range(loop):
            triangle(centre, rib[k], rib[(k + 1) % loop], rib_mat, sheet)
        begin = len(items["seam_vertex_id"])
        items["seam_vertex_id"] += rib + ring[s]
        items["seam"].append(abi.SceneSeam(next(ids), seam_mat, begin, begin + loop, loop))
    line_mat = next(ids)
    items["line_material"].append(abi.SceneLineMaterial(line_mat, 0.002, 0.005, 2e4, 1.0))
    pilot_id = next(ids) if pilot else 0
    if pilot:
        items["pilot"].append(abi.ScenePilot(pilot_id, 90.0, abi.Vec3(0.0, 0.9, -5.0), abi.Vec3(0.0, 0.0, 0.0),
                                             abi.Quat(1.0, 0.0, 0.0, 0.0), abi.Vec3(12.0, 10.0, 6.0)))

    def attach(kind, vertex_id=0, junction=0, local=(0.0, 0.0, 0.0)):
        i = next(ids)
        items["attachment"].append(abi.SceneAttachment(i, kind, 0, vertex_id, pilot_id if kind == 2 else 0,
                                                       junction, abi.Vec3(*local)))
        return i

    def line(a, b, rest):
        items["line"].append(abi.SceneLine(next(ids), a, b, line_mat, rest, 1, 0))

    bottom = loop * 3 // 4  # a bottom-skin vertex of each ring
    for side, stations_of_side in enumerate((range(0, stations // 2), range(stations // 2, stations))):
        j = next(ids)
        jp = np.array([0.0, 0.3 + 1.2 * side, -3.0])
        items["junction"].append(abi.SceneJunction(j, abi.Vec3(*jp), 0.01, 0, 0))
        ja = attach(3, junction=j)
        for s in stations_of_side:
            for k in (bottom - 1, bottom + 1):
                v = ring[s][k]
                line(attach(1, vertex_id=v), ja, float(np.linalg.norm(pos[v] - jp)))
        if pilot:
            line(ja, attach(2, local=(0.0, 0.2 * (2 * side - 1), 0.35)), 1.5)
    # shuffled input order (the assembly sorts by stable ID)
    for k in ("vertex", "triangle", "attachment", "line", "fabric", "junction"):
        order = rng.permutation(len(items[k]))
        items[k] = [items[k][i] for i in order]
    return items


def fields(view):
    """Every array of a definition view as numpy records, for exact
    comparison."""
    out = {}
    for count, field, ctype in (("node_count", "nodes", abi.NodeDef), ("triangle_count", "triangles", abi.TriangleDef),
                                ("constraint_count", "constraints", abi.ConstraintDef),
                                ("membrane_count", "membranes", abi.MembraneDef),
                                ("dihedral_count", "dihedrals", abi.DihedralDef)):
        n = getattr(view, count)
        out[field] = bytes((ctype * n).from_address(C_addr(getattr(view, field)))) if n else b""
    if view.suspension:
        s = view.suspension.contents
        out["suspension"] = bytes(s)[:s.__class__.attachment_count.offset]
        for count, field, ctype in (("attachment_count", "attachments", abi.SuspensionAttachment),
                                    ("junction_count", "junctions", abi.SuspensionJunction),
                                    ("harness_count", "harness_points", abi.PilotHarness),
                                    ("segment_count", "segments", abi.SuspensionSegment)):
            n = getattr(s, count)
            out["suspension_" + field] = bytes((ctype * n).from_address(C_addr(getattr(s, field)))) if n else b""
        out["suspension_solver"] = (s.solver_iterations, s.attachment_tolerance, s.minimum_line_length,
                                    s.maximum_line_residual, s.maximum_control_work)
    out["contact"] = bytes(view.fabric_self_contact.contents) if view.fabric_self_contact else None
    return out


def C_addr(ptr):
    import ctypes

    return ctypes.cast(ptr, ctypes.c_void_p).value


def both(items, settings=None):
    scene = sw.SceneArrays(**items)
    st = settings or sw.SceneSettings()
    mine, report = sw.assemble_scene(scene, st)
    ref = O.RefAssembly(scene, st)
    return mine, report, ref


@pytest.mark.parametrize("pilot", [True, False])
@pytest.mark.parametrize("seed", [0, 1])
def test_assembly_equals_the_reference(pilot, seed):
    items = canopy(pilot=pilot, seed=seed)
    settings = sw.SceneSettings(has_fabric_self_contact=1,
                                fabric_self_contact=abi.FabricContactDef(0.002, 1e-3, 0.4, 0.25))
    mine, report, ref = both(items, settings)
    assert ref.status == 0, ref.report.first_message
    assert mine is not None and report.assembled
    a, b = fields(mine.view), fields(ref.view)
    assert a.keys() == b.keys()
    for k in a:
        assert a[k] == b[k], k
    assert report.total_fabric_mass == ref.report.total_fabric_mass
    assert report.total_seam_mass == ref.report.total_seam_mass
    assert mine.fingerprint == abi.library().swb_definition_fingerprint(ref.pointer)
    counts = mine.counts()
    assert counts["dihedrals"] > 0 and counts["seam_stitch"] > 0 and counts["membranes"] == counts["triangles"]
    if pilot:
        assert counts["suspension_segments"] > 0 and counts["cable"] == 0
    else:
        assert counts["cable"] > 0 and not mine.has_suspension
    mine.validate()  # a valid structure definition


def refusal_cases():
    base = canopy(seed=3)
    cases = {}

    def case(name, edit):
        items = copy.deepcopy(base)
        edit(items)
        cases[name] = items

    def move_seam_vertex(it):
        v = it["seam_vertex_id"][it["seam"][0].first_begin + 1]
        for x in it["vertex"]:
            if x.id == v:
                x.position.x += 1e-3
    case("seam not coincident", move_seam_vertex)
    case("zero bending rigidity", lambda it: setattr(it["fabric"][0], "bending_stiffness", 0.0))
    case("degenerate chart", lambda it: setattr(it["triangle"][3], "chart", ((0, 0), (1, 0), (2, 0))))
    case("missing vertex", lambda it: it["triangle"][5].vertex_ids.__setitem__(0, 7))
    case("duplicate id", lambda it: setattr(it["line"][1], "id", it["line"][0].id))
    case("two pilots", lambda it: it["pilot"].append(abi.ScenePilot(3, 80.0, abi.Vec3(0, 0, -5), abi.Vec3(0, 0, 0),
                                                                     abi.Quat(1, 0, 0, 0), abi.Vec3(1, 1, 1))))
    case("pilot orientation", lambda it: setattr(it["pilot"][0].body_to_world, "w", 2.0))
    case("fixed junction", lambda it: setattr(it["junction"][0], "fixed", 1))

    def non_leaf(it):
        # a second line on one surface attachment: not a leaf of the tree
        surface = [a for a in it["attachment"] if a.kind == 1][0]
        junction = [a for a in it["attachment"] if a.kind == 3][0]
        it["line"].append(abi.SceneLine(5, surface.id, junction.id, it["line_material"][0].id, 1.0, 1, 0))
    case("surface attachment not a leaf", non_leaf)

    def non_manifold(it):
        t = it["triangle"][0]
        apex = abi.SceneVertex(11, abi.Vec3(5.0, 5.0, 5.0))
        it["vertex"].append(apex)
        it["triangle"].append(abi.SceneTriangle(12, (t.vertex_ids[1], t.vertex_ids[0], 11),
                                                ((0, 0), (1, 0), (0, 1)), t.material_id, t.sheet_id))
    case("non-manifold sheet edge", non_manifold)
    case("line rest length", lambda it: setattr(it["line"][2], "rest_length", -1.0))
    case("ill-conditioned fabric", lambda it: setattr(it["fabric"][1], "shear_stiffness", 1e-300))
    return cases


@pytest.mark.parametrize("name", sorted(refusal_cases()))
def test_refusals_match_the_reference(name):
    mine, report, ref = both(refusal_cases()[name])
    if name == "zero bending rigidity":
        # not a refusal: the hinges of that material are left out alike
        assert mine is not None and ref.status == 0
        assert fields(mine.view) == fields(ref.view)
        return
    assert ref.status != 0 and mine is None
    assert not report.assembled and report.diagnostic_count > 0
    got = (report.first_code, report.first_validation_code, report.first_entity_kind, report.first_entity_id)
    want = (ref.report.first_code, ref.report.first_validation_code, ref.report.first_entity_kind,
            ref.report.first_entity_id)
    assert got == want, (report.first_message, ref.report.first_message)
