"""B200 XPBD structural solver: Python mirror of SimWing's structural adapter.

`Structure` follows `simwing::fsi::Structure` (src/fsi/structure.h:273-309):
the same calls, argument meaning and error behaviour, over the library's
C-ABI (include/simwing_b200.h).  Reference exception types map to Python
ones: std::invalid_argument -> InvalidArgument (ValueError),
std::out_of_range -> OutOfRange (IndexError), softwing::SuspensionError ->
SuspensionError, softwing::ContactStepError -> ContactStepError.  A failed
step restores the pre-step state before raising, as the reference does.

There is no CPU fallback: importing the solver requires the built CUDA
library (simwing_b200/libsimwing_b200.so) and a CUDA device to run.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import abi
from .abi import Vec3

__all__ = [
    "Structure", "Definition", "StepSettings", "SolverOptions", "generate_patch", "generate_wing",
    "SimwingError", "InvalidArgument", "OutOfRange", "SuspensionError", "ContactStepError",
    "port_mass_flows",
    "NonFiniteState", "SyncTimeout", "CudaError", "Unsupported", "reference_colouring",
    "definition_from_arrays", "plan_schedule",
]


class SimwingError(RuntimeError):
    status = -1


class InvalidArgument(SimwingError, ValueError):
    status = abi.INVALID_ARGUMENT


class OutOfRange(SimwingError, IndexError):
    status = abi.OUT_OF_RANGE


class SuspensionError(SimwingError):
    """softwing::SuspensionError: `phase` (a SuspensionPhase name) and
    `entity`, as its phase() and entity() give them."""
    status = abi.SUSPENSION_ERROR
    phase = None
    entity = None


class ContactStepError(SimwingError):
    """softwing::ContactStepError: `key`, its ContactFeatureKey as (pair,
    kind, first, second) -- the default key (0, 0, (0, 0, 0), (0, 0, 0))
    when the failure belongs to no feature."""
    status = abi.CONTACT_ERROR
    key = None


class NonFiniteState(SimwingError):
    status = abi.NON_FINITE


class SyncTimeout(SimwingError):
    status = abi.SYNC_TIMEOUT


class CudaError(SimwingError):
    status = abi.CUDA_ERROR


class Unsupported(SimwingError):
    status = abi.UNSUPPORTED


class OutOfMemory(SimwingError, MemoryError):
    status = abi.OUT_OF_MEMORY


_ERRORS = {cls.status: cls for cls in (InvalidArgument, OutOfRange, SuspensionError, ContactStepError,
                                        NonFiniteState, SyncTimeout, CudaError, Unsupported, OutOfMemory)}


def _check(status: int) -> None:
    if status != abi.OK:
        lib = abi.library()
        message = lib.swb_last_error().decode(errors="replace")
        error = _ERRORS.get(status, SimwingError)(message)
        if status in (abi.SUSPENSION_ERROR, abi.CONTACT_ERROR):
            d = abi.ErrorDetail()
            lib.swb_last_error_detail(C.byref(d))
            if d.status == status and status == abi.SUSPENSION_ERROR:
                error.phase = abi.SUSPENSION_PHASES[d.suspension_phase]
                error.entity = d.suspension_entity.decode(errors="replace")
            elif d.status == status:
                k = d.contact_key
                error.key = (int(k.pair), int(k.kind), tuple(int(x) for x in k.first),
                             tuple(int(x) for x in k.second))
        raise error


def StepSettings(**overrides) -> abi.StepSettings:
    """StructureStepSettings with the reference defaults (structure.h:208-219)."""
    s = abi.StepSettings()
    abi.library().swb_default_step_settings(C.byref(s))
    for key, value in overrides.items():
        if key in ("gravity", "damping_reference_velocity"):
            value = Vec3(*value)
        setattr(s, key, value)
    return s


def SolverOptions(**overrides) -> abi.SolverOptions:
    o = abi.SolverOptions()
    abi.library().swb_default_solver_options(C.byref(o))
    for key, value in overrides.items():
        setattr(o, key, value)
    return o


def _array(ptr, count, ctype):
    if count == 0:
        return np.zeros(0, dtype=np.dtype(ctype))
    return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ctype)), shape=(count,))


class Definition:
    """An owned StructureDefinition (swb_definition handle)."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)
        self._lib = abi.library()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and h.value:
            self._lib.swb_definition_destroy(h)
            self._h = C.c_void_p()

    @property
    def view(self) -> abi.StructureDefinition:
        return self._lib.swb_definition_view(self._h).contents

    @property
    def pointer(self):
        return self._lib.swb_definition_view(self._h)

    def copy(self) -> "Definition":
        out = C.c_void_p()
        _check(self._lib.swb_definition_copy(self.pointer, C.byref(out)))
        return Definition(out.value)

    def permuted(self, constraint_order=None, dihedral_order=None, membrane_order=None) -> "Definition":
        d = self.copy()
        co = None if constraint_order is None else np.ascontiguousarray(constraint_order, dtype=np.uint64)
        ho = None if dihedral_order is None else np.ascontiguousarray(dihedral_order, dtype=np.uint64)
        _check(self._lib.swb_definition_permute(
            d._h, None if co is None else co.ctypes.data, None if ho is None else ho.ctypes.data))
        if membrane_order is not None:
            mo = np.ascontiguousarray(membrane_order, dtype=np.uint64)
            _check(self._lib.swb_definition_permute_membranes(d._h, mo.ctypes.data))
        return d

    def set_contact(self, contact) -> None:
        """Fabric self-contact of all triangles: (half_thickness,
        normal_compliance, static_friction, dynamic_friction), or None."""
        fc = None if contact is None else abi.FabricContactDef(*[float(x) for x in contact])
        _check(abi.library().swb_definition_set_contact(self._h, None if fc is None else C.byref(fc)))

    def scale_rest(self, index: int, factor: float) -> None:
        _check(self._lib.swb_definition_scale_rest(self._h, index, factor))

    @property
    def fingerprint(self) -> int:
        return int(self._lib.swb_definition_fingerprint(self.pointer))

    def validate(self) -> None:
        _check(self._lib.swb_validate_definition(self.pointer))

    # numpy views (valid while the definition lives)
    @property
    def node_count(self) -> int:
        return int(self.view.node_count)

    def positions(self) -> np.ndarray:
        v = self.view
        raw = _array(v.nodes, v.node_count, abi.NodeDef)
        return np.stack([raw["position"]["x"], raw["position"]["y"], raw["position"]["z"]], axis=1)

    def nodes(self):
        v = self.view
        return _array(v.nodes, v.node_count, abi.NodeDef)

    def triangles(self):
        v = self.view
        return _array(v.triangles, v.triangle_count, abi.TriangleDef)

    def constraints(self):
        v = self.view
        return _array(v.constraints, v.constraint_count, abi.ConstraintDef)

    def dihedrals(self):
        v = self.view
        return _array(v.dihedrals, v.dihedral_count, abi.DihedralDef)

    @property
    def has_suspension(self) -> bool:
        return bool(self.view.suspension)

    def counts(self) -> dict:
        v = self.view
        out = {"nodes": int(v.node_count), "triangles": int(v.triangle_count),
               "constraints": int(v.constraint_count), "dihedrals": int(v.dihedral_count),
               "membranes": int(v.membrane_count)}
        if v.suspension:
            out["suspension_segments"] = int(v.suspension.contents.segment_count)
        c = self.constraints()
        for name, kind in (("distance", abi.DISTANCE), ("cable", abi.CABLE), ("seam_stitch", abi.SEAM_STITCH),
                           ("suspension_tie", abi.SUSPENSION_TIE)):
            out[name] = int(np.count_nonzero(c["kind"] == kind))
        return out


def definition_from_arrays(nodes, triangles=(), constraints=(), dihedrals=(), suspension=None,
                           membranes=(), contact=None) -> Definition:
    """Builds an owned Definition from plain Python records.

    nodes:       [(x, y, z, mass, fixed), ...]
    triangles:   [(a, b, c[, pressure]), ...]
    constraints: [(kind, a, b, rest, compliance), ...]
    dihedrals:   [(a, b, c, d, rest_angle, compliance), ...]
    membranes:   [(triangle, ((u0, v0), (u1, v1), (u2, v2)), material[, role]), ...]
                 material = dict of MembraneMaterial fields (warp_stiffness,
                 weft_stiffness, coupling_stiffness, shear_stiffness,
                 warp_pretension, weft_pretension, damping_seconds,
                 compression_stiffness_ratio; the last defaults to 1)
    suspension:  dict with pilot_mass, pilot_com_world, pilot_inertia,
                 attachments [(id, node)], harness [(id, (x, y, z))],
                 segments [(id, (kind, id), (kind, id), rest, stiffness,
                 damping)], solver_iterations, maximum_line_residual.
    contact:     (half_thickness, normal_compliance, static_friction,
                 dynamic_friction): fabric self-contact of all triangles.
    """
    lib = abi.library()
    n = (abi.NodeDef * max(len(nodes), 1))()
    for i, (x, y, z, m, fixed) in enumerate(nodes):
        n[i] = abi.NodeDef(Vec3(x, y, z), m, 1 if fixed else 0, 0)
    t = (abi.TriangleDef * max(len(triangles), 1))()
    for i, tri in enumerate(triangles):
        t[i].nodes[:] = [int(tri[0]), int(tri[1]), int(tri[2])]
        t[i].pressure_difference = float(tri[3]) if len(tri) > 3 else 0.0
    c = (abi.ConstraintDef * max(len(constraints), 1))()
    for i, (kind, a, b, rest, comp) in enumerate(constraints):
        c[i] = abi.ConstraintDef(kind, 0, a, b, rest, comp)
    h = (abi.DihedralDef * max(len(dihedrals), 1))()
    for i, (a, b, cc, d, rest, comp) in enumerate(dihedrals):
        h[i].nodes[:] = [a, b, cc, d]
        h[i].rest_angle = rest
        h[i].compliance = comp
    view = abi.StructureDefinition()
    view.node_count, view.nodes = len(nodes), n
    view.triangle_count, view.triangles = len(triangles), t
    view.constraint_count, view.constraints = len(constraints), c
    view.dihedral_count, view.dihedrals = len(dihedrals), h
    mb = (abi.MembraneDef * max(len(membranes), 1))()
    for i, rec in enumerate(membranes):
        tri, chart, material = rec[0], rec[1], rec[2]
        mb[i].triangle = int(tri)
        for k in range(3):
            mb[i].chart[k][0], mb[i].chart[k][1] = float(chart[k][0]), float(chart[k][1])
        fields = {"compression_stiffness_ratio": 1.0}
        fields.update(material)
        for name, value in fields.items():
            setattr(mb[i].material, name, float(value))
        mb[i].role = int(rec[3]) if len(rec) > 3 else abi.ROLE_BULK
    view.membrane_count, view.membranes = len(membranes), mb
    keep = [n, t, c, h, mb]
    if suspension is not None:
        s = abi.SuspensionDef()
        s.pilot_stable_id = 1
        s.pilot_mass = suspension.get("pilot_mass", 90.0)
        s.pilot_initial_com_world = Vec3(*suspension.get("pilot_com_world", (0.0, 0.0, 0.0)))
        s.pilot_initial_body_to_world = abi.Quat(*suspension.get("pilot_orientation", (1.0, 0.0, 0.0, 0.0)))
        s.pilot_principal_inertia = Vec3(*suspension.get("pilot_inertia", (10.0, 10.0, 5.0)))
        s.pilot_initial_linear_velocity = Vec3(*suspension.get("pilot_velocity", (0.0, 0.0, 0.0)))
        s.pilot_initial_angular_velocity = Vec3(*suspension.get("pilot_angular_velocity", (0.0, 0.0, 0.0)))
        att = suspension.get("attachments", [])
        a = (abi.SuspensionAttachment * max(len(att), 1))(*[abi.SuspensionAttachment(i, nd) for i, nd in att])
        jun = suspension.get("junctions", [])
        j = (abi.SuspensionJunction * max(len(jun), 1))(*[abi.SuspensionJunction(i, nd) for i, nd in jun])
        har = suspension.get("harness", [])
        hp = (abi.PilotHarness * max(len(har), 1))(*[abi.PilotHarness(i, Vec3(*p)) for i, p in har])
        seg = suspension.get("segments", [])
        sg = (abi.SuspensionSegment * max(len(seg), 1))()
        for k, (sid, fr, to, rest, stiff, damp) in enumerate(seg):
            sg[k] = abi.SuspensionSegment(sid, abi.SuspensionEndpoint(fr[0], 0, fr[1]),
                                          abi.SuspensionEndpoint(to[0], 0, to[1]), rest, stiff, damp, 1, 0)
        s.attachment_count, s.attachments = len(att), a
        s.junction_count, s.junctions = len(jun), j
        s.harness_count, s.harness_points = len(har), hp
        s.segment_count, s.segments = len(seg), sg
        s.solver_iterations = suspension.get("solver_iterations", 12)
        s.attachment_tolerance = 1e-10
        s.minimum_line_length = 1e-10
        s.maximum_line_residual = suspension.get("maximum_line_residual", 2e-4)
        s.maximum_control_work = 1e6
        view.suspension = C.pointer(s)
        keep += [s, a, j, hp, sg]
    if contact is not None:
        fc = abi.FabricContactDef(*[float(x) for x in contact])
        view.fabric_self_contact = C.pointer(fc)
        keep.append(fc)
    out = C.c_void_p()
    _check(lib.swb_definition_copy(C.byref(view), C.byref(out)))
    del keep
    return Definition(out.value)


def stacked_sheets(n: int = 8, gap: float = 0.003, half_thickness: float = 0.002, friction=(0.4, 0.25),
                   spacing: float = 0.05, compliance: float = 0.0, mass: float = 0.001,
                   suspension=None) -> Definition:
    """Fabric self-contact scene: a free n x n sheet (distance constraints on
    its edges, compliance 1e-7) `gap` above a pinned n x n sheet, shifted by
    (13 mm, 7 mm) so that vertices, edges and faces of the two meet in every
    feature configuration; contact (half_thickness, compliance, static and
    dynamic friction) over all triangles.  `suspension` as for
    definition_from_arrays (node indices: the pinned sheet first)."""
    nodes, tris, cons = [], [], []
    for layer, z in ((0, 0.0), (1, gap)):
        off = len(nodes)
        for j in range(n):
            for i in range(n):
                x, y = i * spacing, j * spacing
                if layer:
                    x, y = x + 0.013, y + 0.007
                nodes.append((x, y, z, mass, layer == 0))
        for j in range(n - 1):
            for i in range(n - 1):
                a = off + j * n + i
                b, c, d = a + 1, a + n, a + n + 1
                tris += [(a, b, d), (a, d, c)]
                if layer:
                    for u, v in ((a, b), (a, c), (a, d)):
                        rest = float(np.linalg.norm(np.subtract(nodes[u][:3], nodes[v][:3])))
                        cons.append((1, u, v, rest, 1e-7))
        if layer:
            for j in range(n - 1):
                a = off + j * n + n - 1
                cons.append((1, a, a + n, spacing, 1e-7))
            for i in range(n - 1):
                a = off + (n - 1) * n + i
                cons.append((1, a, a + 1, spacing, 1e-7))
    return definition_from_arrays(nodes, tris, cons, suspension=suspension,
                                  contact=(half_thickness, compliance, friction[0], friction[1]))


def generate_patch(**overrides) -> Definition:
    """The hanging cloth patch (33 x 33 on 1 m x 1 m by default)."""
    lib = abi.library()
    p = abi.PatchParams()
    lib.swb_default_patch_params(C.byref(p))
    for k, v in overrides.items():
        setattr(p, k, v)
    out = C.c_void_p()
    _check(lib.swb_generate_patch(C.byref(p), C.byref(out)))
    return Definition(out.value)


def generate_wing(**overrides) -> Definition:
    """The ram-air wing with cascaded lines and rigid pilot (40 cells by default)."""
    lib = abi.library()
    p = abi.WingParams()
    lib.swb_default_wing_params(C.byref(p))
    for k, v in overrides.items():
        setattr(p, k, v)
    out = C.c_void_p()
    _check(lib.swb_generate_wing(C.byref(p), C.byref(out)))
    return Definition(out.value)


# The adjoint calibration wing: 20 cells x 30 chordwise (13,338 triangles)
# with two line attachment stations per cell and row (266 line rest
# lengths).
CALIBRATION_WING = dict(cells=20, chordwise=30, attachments_per_cell=2)


def generate_calibration_wing(**overrides) -> Definition:
    """The adjoint calibration wing (CALIBRATION_WING)."""
    return generate_wing(**dict(CALIBRATION_WING, **overrides))


class SceneArrays:
    """A swb_scene over ctypes arrays (kept alive here): `items` maps each
    array name of abi.SCENE_ARRAYS to a list of its ctypes records (or, for
    seam_vertex_id, of IDs)."""

    def __init__(self, **items):
        self.view = abi.Scene()
        self._keep = []
        for name, ctype, field in abi.SCENE_ARRAYS:
            values = items.get(name, [])
            arr = (ctype * max(len(values), 1))(*values)
            self._keep.append(arr)
            setattr(self.view, name + "_count", len(values))
            setattr(self.view, field, C.cast(arr, C.POINTER(ctype)))


def SceneSettings(**overrides) -> abi.SceneSettings:
    s = abi.SceneSettings()
    abi.library().swb_default_scene_settings(C.byref(s))
    for key, value in overrides.items():
        setattr(s, key, value)
    return s


def assemble_scene(scene: SceneArrays, settings: abi.SceneSettings | None = None):
    """simwing::fsi::assembleSceneStructure (scene_structure.cpp:894-1284):
    returns (Definition or None when refused, the report)."""
    report = abi.SceneReport()
    out = C.c_void_p()
    st = settings if settings is not None else SceneSettings()
    status = abi.library().swb_assemble_scene(C.byref(scene.view), C.byref(st), C.byref(out), C.byref(report))
    if status == abi.INVALID_ARGUMENT and not report.assembled and report.diagnostic_count:
        return None, report
    _check(status)
    return Definition(out.value), report


def wing_batch_parameters(count: int = 64, seed: int = 2024):
    """Seeded uneven wing sizes of the batched workload: cells ~ U{20..60},
    chordwise in {30, 45, 60}, aspect ratio ~ U(4.5, 7), per-wing compliance
    multiplier lognormal(0, 0.2) (drawn by the generator from its seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        out.append(dict(cells=int(rng.integers(20, 61)), chordwise=int(rng.choice([30, 45, 60])),
                        aspect_ratio=float(rng.uniform(4.5, 7.0)), compliance_jitter=0.2,
                        seed=int(seed) * 1000 + i))
    return out


def generate_wing_batch(count: int = 64, seed: int = 2024, **overrides) -> list:
    """Definitions of the batched workload (see wing_batch_parameters)."""
    return [generate_wing(**dict(p, **overrides)) for p in wing_batch_parameters(count, seed)]


def line_groups(definition: Definition) -> list:
    """The suspension lines of a definition as groups of cable constraints:
    maximal chains of cables through nodes that exactly two cables share (a
    line's particles, or a junction where one line continues into one
    other).  Returns a list of constraint-index arrays."""
    cons = definition.constraints()
    cables = np.where(cons["kind"] == abi.CABLE)[0]
    a = cons["first_node"][cables].astype(np.int64)
    b = cons["second_node"][cables].astype(np.int64)
    degree = np.bincount(np.concatenate([a, b]), minlength=definition.node_count)
    parent = np.arange(len(cables))

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    first_at = {}
    for j, (u, v) in enumerate(zip(a, b)):
        for node in (int(u), int(v)):
            if degree[node] != 2:
                continue
            if node in first_at:
                parent[find(j)] = find(first_at[node])
            else:
                first_at[node] = j
    groups = {}
    for j in range(len(cables)):
        groups.setdefault(find(j), []).append(int(cables[j]))
    return [np.array(g, dtype=np.int64) for g in groups.values()]


def reference_colouring(definition: Definition):
    """Bit-exact restatement of SoftBody::constraintColouringView."""
    lib = abi.library()
    m = definition.view.constraint_count
    order = np.zeros(max(m, 1), dtype=np.uint64)
    offsets = np.zeros(4096, dtype=np.uint64)
    colours = C.c_uint64()
    parallel = C.c_uint64()
    _check(lib.swb_reference_colouring(definition.pointer, order.ctypes.data, offsets.ctypes.data,
                                       offsets.size, C.byref(colours), C.byref(parallel)))
    return order[:m], offsets[: colours.value + 1 if m else 0], int(parallel.value)


def CcdSettings(**overrides) -> abi.CcdSettings:
    s = abi.CcdSettings()
    abi.library().swb_default_ccd_settings(C.byref(s))
    for k, v in overrides.items():
        setattr(s, k, v)
    return s


def contact_candidates(definition: Definition, half_thickness: float, previous, current):
    """Candidate features of the definition's fabric self-contact pair on the
    device (swb_contact_candidates); returns (keys, possible, excluded)."""
    lib = abi.library()
    prev = np.ascontiguousarray(previous, dtype=np.float64)
    cur = np.ascontiguousarray(current, dtype=np.float64)
    n, possible, excluded = C.c_uint64(), C.c_uint64(), C.c_uint64()
    status = lib.swb_contact_candidates(definition.pointer, half_thickness, prev.ctypes.data, cur.ctypes.data,
                                        None, 0, C.byref(n), C.byref(possible), C.byref(excluded))
    if status not in (abi.OK, abi.OUT_OF_RANGE):
        _check(status)
    keys = (abi.ContactKey * max(n.value, 1))()
    _check(lib.swb_contact_candidates(definition.pointer, half_thickness, prev.ctypes.data, cur.ctypes.data, keys,
                                      n.value, C.byref(n), C.byref(possible), C.byref(excluded)))
    return list(keys)[: n.value], possible.value, excluded.value


def port_mass_flows(zones, ports, air=(287.05, 1.4)):
    """Mass flow through each pneumatic port between two zones
    (evaluateOrificeMassFlow / evaluateConductanceMassFlow,
    pneumatics.cpp:132-232), one device thread per port.  `zones` are
    (absolute pressure Pa, absolute temperature K) records, `ports` records
    of abi.PORT_DTYPE, `air` (R, gamma).  Returns abi.FLOW_DTYPE records.
    Raises InvalidArgument where the reference throws, with the first
    refusing port in the exception's `port`."""
    z = np.array(zones, dtype=abi.ZONE_DTYPE).reshape(-1)
    p = np.array(ports, dtype=abi.PORT_DTYPE).reshape(-1)
    out = np.zeros(len(p), dtype=abi.FLOW_DTYPE)
    failed = C.c_uint64(0)
    a = abi.AirProperties(*air)
    status = abi.library().swb_port_mass_flows(C.byref(a), z.ctypes.data, len(z), p.ctypes.data, len(p),
                                               out.ctypes.data, C.byref(failed))
    try:
        _check(status)
    except InvalidArgument as e:
        e.port = failed.value
        raise
    return out


def contact_closest(kind: int, first, second, separation: float):
    """closestVertexTriangle / closestEdgeEdge on the device, 9 doubles per
    feature and side (swb_contact_closest)."""
    f = np.ascontiguousarray(first, dtype=np.float64).reshape(-1, 9)
    s = np.ascontiguousarray(second, dtype=np.float64).reshape(-1, 9)
    out = (abi.ClosestResult * max(len(f), 1))()
    _check(abi.library().swb_contact_closest(kind, len(f), f.ctypes.data, s.ctypes.data, separation, out))
    return list(out)[: len(f)]


def contact_sweep(kind: int, first_previous, first_current, second_previous, second_current, separation: float,
                  settings: abi.CcdSettings | None = None):
    """sweptContact on the device (swb_contact_sweep)."""
    arrays = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1, 9)
              for a in (first_previous, first_current, second_previous, second_current)]
    n = len(arrays[0])
    out = (abi.CcdResult * max(n, 1))()
    _check(abi.library().swb_contact_sweep(kind, n, *[a.ctypes.data for a in arrays], separation,
                                           C.byref(settings or CcdSettings()), out))
    return list(out)[:n]


def plan_schedule(definition: Definition, options: abi.SolverOptions | None = None):
    """Host-only schedule build + invariant check; returns (report,
    distance sweep order, dihedral sweep order)."""
    lib = abi.library()
    v = definition.view
    r = abi.ScheduleReport()
    do = np.zeros(max(v.constraint_count, 1), dtype=np.uint64)
    ho = np.zeros(max(v.dihedral_count, 1), dtype=np.uint64)
    _check(lib.swb_plan_schedule(definition.pointer, None if options is None else C.byref(options), C.byref(r),
                                 do.ctypes.data, ho.ctypes.data))
    return r, do[: v.constraint_count], ho[: v.dihedral_count]


def plan_membrane_order(definition: Definition, options: abi.SolverOptions | None = None) -> np.ndarray:
    """The membrane sweep order of the host-built schedule (as
    Structure.sweep_order(SWEEP_MEMBRANE) gives it on the device)."""
    n = definition.view.membrane_count
    out = np.zeros(max(n, 1), dtype=np.uint64)
    _check(abi.library().swb_plan_membrane_order(definition.pointer, None if options is None else C.byref(options),
                                                 out.ctypes.data))
    return out[:n]


@dataclass
class SuspensionState:
    center_of_mass: np.ndarray
    body_to_world: np.ndarray  # w, x, y, z
    linear_velocity: np.ndarray
    angular_velocity: np.ndarray
    segments: list
    line_force: np.ndarray
    line_moment: np.ndarray


def _vec(v) -> np.ndarray:
    return np.array([v.x, v.y, v.z])


class Structure:
    """simwing::fsi::Structure on the device (src/fsi/structure.h:273-309)."""

    def __init__(self, definition: Definition, options: abi.SolverOptions | None = None, *, _borrowed=None):
        self._lib = abi.library()
        self._definition = definition
        self._owner = None
        if _borrowed is not None:
            # a structure owned by a Batch: the batch keeps it alive
            h, self._owner = _borrowed
        else:
            h = C.c_void_p()
            _check(self._lib.swb_structure_create(definition.pointer, None if options is None else C.byref(options),
                                                  C.byref(h)))
        self._h = h
        self.node_count = int(self._lib.swb_structure_node_count(h))
        self._segments = int(definition.view.suspension.contents.segment_count) if definition.has_suspension else 0

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            if getattr(self, "_owner", None) is None:
                self._lib.swb_structure_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def definition_fingerprint(self) -> int:
        return int(self._lib.swb_structure_fingerprint(self._h))

    def accepted_step_count(self) -> int:
        return int(self._lib.swb_structure_accepted_steps(self._h))

    def simulation_time_seconds(self) -> float:
        return float(self._lib.swb_structure_simulation_time(self._h))

    def clear_external_forces(self) -> None:
        _check(self._lib.swb_structure_clear_external_forces(self._h))

    def add_external_force(self, node: int, force) -> None:
        if node < 0:
            raise OutOfRange("Structure force node is out of range")
        _check(self._lib.swb_structure_add_external_force(self._h, int(node), C.byref(Vec3(*force))))

    def set_external_forces(self, forces) -> None:
        f = np.ascontiguousarray(forces, dtype=np.float64)
        if f.ndim != 2 or f.shape[1] != 3:
            raise InvalidArgument("Structure forces must be an (n, 3) array")
        _check(self._lib.swb_structure_set_external_forces(self._h, f.ctypes.data, f.shape[0]))

    def set_face_pressure(self, triangle: int, pressure: float) -> None:
        _check(self._lib.swb_structure_set_face_pressure(self._h, int(triangle), float(pressure)))

    def set_uniform_pressure(self, pressure: float) -> None:
        _check(self._lib.swb_structure_set_uniform_pressure(self._h, float(pressure)))

    def set_ground(self, normal=(0.0, 0.0, 1.0), offset: float = 0.0, friction: float = 0.0,
                   enabled: bool = True) -> None:
        """A ground plane normal . x >= offset (swb_structure_set_ground);
        enabled=False removes it."""
        g = abi.Ground(Vec3(*normal), float(offset), float(friction), 1 if enabled else 0, 0)
        _check(self._lib.swb_structure_set_ground(self._h, C.byref(g)))

    def set_line_contact(self, radius: float, margin: float = 0.0, enabled: bool = True) -> None:
        """Line-line contact of the cable segments, kept 2 x radius apart
        (swb_structure_set_line_contact); enabled=False removes it."""
        lc = abi.LineContact(float(radius), float(margin), 1 if enabled else 0, 0)
        _check(self._lib.swb_structure_set_line_contact(self._h, C.byref(lc)))

    def step(self, settings: abi.StepSettings | None = None, diagnostics: bool = True):
        s = settings if settings is not None else StepSettings()
        d = abi.Diagnostics()
        _check(self._lib.swb_structure_step(self._h, C.byref(s), C.byref(d) if diagnostics else None))
        return d if diagnostics else None

    def step_many(self, settings: abi.StepSettings, steps: int, diagnostics: bool = False):
        d = abi.Diagnostics()
        _check(self._lib.swb_structure_step_many(self._h, C.byref(settings), int(steps),
                                                 C.byref(d) if diagnostics else None))
        return d if diagnostics else None

    def diagnostics(self) -> abi.Diagnostics:
        d = abi.Diagnostics()
        _check(self._lib.swb_structure_diagnostics(self._h, C.byref(d)))
        return d

    def node_states(self) -> np.ndarray:
        """(n, 3, 3) array: position, previous position, velocity."""
        out = np.zeros((self.node_count, 3, 3), dtype=np.float64)
        _check(self._lib.swb_structure_read_nodes(self._h, out.ctypes.data, self.node_count))
        return out

    def positions(self) -> np.ndarray:
        return self.node_states()[:, 0, :]

    def write_node_states(self, states: np.ndarray) -> None:
        s = np.ascontiguousarray(states, dtype=np.float64)
        if s.shape != (self.node_count, 3, 3):
            raise InvalidArgument("node states must be (n, 3, 3)")
        _check(self._lib.swb_structure_write_nodes(self._h, s.ctypes.data, self.node_count))

    def suspension_state(self) -> SuspensionState | None:
        if not self._segments:
            return None
        p = abi.PayloadState()
        segs = (abi.SegmentState * self._segments)()
        w = abi.Wrench()
        _check(self._lib.swb_structure_read_suspension(self._h, C.byref(p), segs, self._segments, C.byref(w)))
        q = p.body_to_world
        return SuspensionState(_vec(p.center_of_mass), np.array([q.w, q.x, q.y, q.z]), _vec(p.linear_velocity),
                               _vec(p.angular_velocity),
                               [(s.stable_id, s.current_length, s.commanded_rest_length, s.tension) for s in segs],
                               _vec(w.force), _vec(w.moment))

    def write_payload_state(self, com, q_wxyz, v, w) -> None:
        p = abi.PayloadState(Vec3(*com), abi.Quat(*q_wxyz), Vec3(*v), Vec3(*w))
        _check(self._lib.swb_structure_write_payload(self._h, C.byref(p)))

    def checkpoint(self) -> bytes:
        n = C.c_uint64()
        _check(self._lib.swb_structure_checkpoint_size(self._h, C.byref(n)))
        buf = (C.c_uint8 * n.value)()
        _check(self._lib.swb_structure_checkpoint(self._h, buf, n.value))
        return bytes(buf)

    def restore(self, image: bytes) -> None:
        buf = (C.c_uint8 * len(image)).from_buffer_copy(image)
        _check(self._lib.swb_structure_restore(self._h, buf, len(image)))

    def sweep_order(self, which: int) -> np.ndarray:
        v = self._definition.view
        n = v.constraint_count if which == abi.SWEEP_DISTANCE else (
            v.dihedral_count if which == abi.SWEEP_DIHEDRAL else v.membrane_count)
        out = np.zeros(max(n, 1), dtype=np.uint64)
        _check(self._lib.swb_structure_sweep_order(self._h, which, out.ctypes.data, n))
        return out[:n]

    def oracle_definition(self) -> Definition:
        """The definition with its constraint lists permuted into the device
        sweep order: the reference serial solver run on it performs exactly
        the device's Gauss-Seidel sweep."""
        return self._definition.permuted(self.sweep_order(abi.SWEEP_DISTANCE),
                                         self.sweep_order(abi.SWEEP_DIHEDRAL),
                                         self.sweep_order(abi.SWEEP_MEMBRANE) if self._definition.view.membrane_count
                                         else None)

    def contact_candidates(self) -> list:
        """Candidate features of the last step's contact certification, in
        key order (swb_structure_contact_candidates)."""
        n = C.c_uint64()
        status = self._lib.swb_structure_contact_candidates(self._h, None, 0, C.byref(n))
        if status not in (abi.OK, abi.OUT_OF_RANGE):
            _check(status)
        keys = (abi.ContactKey * max(n.value, 1))()
        _check(self._lib.swb_structure_contact_candidates(self._h, keys, n.value, C.byref(n)))
        return list(keys)[: n.value]

    def autotune_report(self) -> list:
        """The autotuner's candidates (SolverOptions flags OPT_AUTOTUNE), each
        a dict with `chosen` set on the one kept; empty when not tuned."""
        r = abi.AutotuneReport()
        _check(self._lib.swb_structure_autotune_report(self._h, C.byref(r)))
        out = []
        for k in range(r.candidates):
            e = r.entries[k]
            out.append({"cluster_ctas": e.cluster_ctas, "block_threads": e.block_threads,
                        "split_stages": bool(e.split_stages), "stages_per_iteration": e.stages_per_iteration,
                        "ms_per_substep": e.ms_per_substep, "chosen": k == r.chosen})
        return out

    def schedule_report(self) -> abi.ScheduleReport:
        r = abi.ScheduleReport()
        _check(self._lib.swb_structure_schedule_report(self._h, C.byref(r)))
        return r

    def last_step_ms(self) -> float:
        return float(self._lib.swb_structure_last_step_ms(self._h))


class Coupling:
    """The structural side of ConservativeMacroStepCoupling
    (src/fsi/coupling.cpp:806-911) with device-resident loads: interface node
    i loads structure node structure_nodes[i].  The load arrays are device
    addresses (integers) or CUDA tensors of bindings x 3 doubles."""

    def __init__(self, structure: "Structure", structure_nodes):
        self._lib = abi.library()
        self._structure = structure  # keep alive
        nodes = np.ascontiguousarray(structure_nodes, dtype=np.uint64)
        h = C.c_void_p()
        _check(self._lib.swb_coupling_create(structure.handle, nodes.ctypes.data, nodes.size, C.byref(h)))
        self._h = h

    @staticmethod
    def _ptr(a):
        return a.data_ptr() if hasattr(a, "data_ptr") else int(a)

    def advance_impulses(self, impulses, duration: float, settings: abi.StepSettings) -> abi.Diagnostics:
        d = abi.Diagnostics()
        _check(self._lib.swb_coupling_advance_impulses(self._h, self._ptr(impulses), duration, C.byref(settings),
                                                       C.byref(d)))
        return d

    def advance_endpoint_loads(self, start_loads, end_loads, settings: abi.StepSettings) -> abi.Diagnostics:
        d = abi.Diagnostics()
        _check(self._lib.swb_coupling_advance_endpoint_loads(self._h, self._ptr(start_loads), self._ptr(end_loads),
                                                             C.byref(settings), C.byref(d)))
        return d

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.swb_coupling_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        self.close()


def BatchOptions(**overrides) -> abi.BatchOptions:
    o = abi.BatchOptions()
    abi.library().swb_default_batch_options(C.byref(o))
    for k, v in overrides.items():
        setattr(o, k, v)
    return o


class Batch:
    """Many independent structures stepped together by one packed cluster
    launch per substep (swb_batch_*).  Each structure is reachable as a
    `Structure` through `structure(i)`; it steps exactly as a plain structure
    built with `cluster_ctas` equal to its rank count."""

    def __init__(self, definitions, options: abi.BatchOptions | None = None):
        self._lib = abi.library()
        self._definitions = list(definitions)
        ptrs = (C.c_void_p * len(self._definitions))(*[C.cast(d.pointer, C.c_void_p) for d in self._definitions])
        h = C.c_void_p()
        _check(self._lib.swb_batch_create(ptrs, len(self._definitions),
                                          None if options is None else C.byref(options), C.byref(h)))
        self._h = h
        self._structures = [Structure(d, _borrowed=(C.c_void_p(self._lib.swb_batch_structure(h, i)), self))
                            for i, d in enumerate(self._definitions)]

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            for s in self._structures:
                s.close()
            self._lib.swb_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __len__(self) -> int:
        return len(self._definitions)

    def structure(self, index: int) -> Structure:
        return self._structures[index]

    def set_ground(self, normal=(0.0, 0.0, 1.0), offset: float = 0.0, friction: float = 0.0,
                   enabled: bool = True) -> None:
        """The ground plane of Structure.set_ground for every structure of
        the batch (swb_batch_set_ground)."""
        g = abi.Ground(Vec3(*normal), float(offset), float(friction), 1 if enabled else 0, 0)
        _check(self._lib.swb_batch_set_ground(self._h, C.byref(g)))

    def step(self, settings: abi.StepSettings, steps: int = 1) -> np.ndarray:
        """Steps every structure; returns the per-structure status codes.
        Raises the first failure after the others have committed."""
        statuses = np.zeros(len(self), dtype=np.int32)
        rc = self._lib.swb_batch_step(self._h, C.byref(settings), int(steps),
                                      statuses.ctypes.data_as(C.c_void_p))
        if rc != abi.OK:
            err = _ERRORS.get(rc, SimwingError)(self._lib.swb_last_error().decode())
            err.statuses = statuses
            raise err
        return statuses

    def report(self) -> abi.BatchReport:
        r = abi.BatchReport()
        _check(self._lib.swb_batch_get_report(self._h, C.byref(r)))
        return r

    def last_step_ms(self) -> float:
        return float(self._lib.swb_batch_last_step_ms(self._h))


class Rollout:
    """Differentiable rollout of a structure (swb_rollout_*): `forward`
    steps it `steps` times from its committed state (left unchanged) and
    returns the loss sum_i w_i |x_i(T) - target_i|^2 / sum w; `backward`
    returns the loss gradient with respect to every constraint's rest length
    and compliance, every dihedral's compliance, every suspension segment's
    rest length and the pilot mass (definition order)."""

    def __init__(self, structure: Structure, steps: int, checkpoint_interval: int = 16):
        self._lib = abi.library()
        self._structure = structure
        h = C.c_void_p()
        _check(self._lib.swb_rollout_create(structure.handle, int(steps), int(checkpoint_interval), C.byref(h)))
        self._h = h
        self.steps = int(steps)

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.swb_rollout_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def forward(self, settings: abi.StepSettings, target, weights) -> float:
        n = self._structure.node_count
        t = np.ascontiguousarray(target, dtype=np.float64).reshape(n, 3)
        w = np.ascontiguousarray(weights, dtype=np.float64).reshape(n)
        loss = C.c_double()
        _check(self._lib.swb_rollout_forward(self._h, C.byref(settings), t.ctypes.data, w.ctypes.data,
                                             C.byref(loss)))
        return loss.value

    def _gradient_buffers(self):
        v = self._structure._definition.view
        m, h = v.constraint_count, v.dihedral_count
        ns = v.suspension.contents.segment_count if v.suspension else 0
        out = {"d_rest": np.zeros(max(m, 1)), "d_comp": np.zeros(max(m, 1)),
               "d_dihedral_comp": np.zeros(max(h, 1)), "d_segment_rest": np.zeros(max(ns, 1)), "mass": np.zeros(1)}
        g = abi.RolloutGradient(out["d_rest"].ctypes.data, out["d_comp"].ctypes.data,
                                out["d_dihedral_comp"].ctypes.data, out["d_segment_rest"].ctypes.data,
                                out["mass"].ctypes.data)
        return out, g, (m, h, ns)

    @staticmethod
    def _gradient_result(out, sizes) -> dict:
        m, h, ns = sizes
        out["d_rest"], out["d_comp"] = out["d_rest"][:m], out["d_comp"][:m]
        out["d_dihedral_comp"], out["d_segment_rest"] = out["d_dihedral_comp"][:h], out["d_segment_rest"][:ns]
        out["d_mass"] = float(out.pop("mass")[0])
        return out

    def backward(self) -> dict:
        out, g, sizes = self._gradient_buffers()
        _check(self._lib.swb_rollout_backward(self._h, C.byref(g)))
        return self._gradient_result(out, sizes)

    def final_positions(self) -> np.ndarray:
        n = self._structure.node_count
        out = np.zeros((n, 3))
        _check(self._lib.swb_rollout_final_positions(self._h, out.ctypes.data, n))
        return out

    def forward_ms(self) -> float:
        return float(self._lib.swb_rollout_forward_ms(self._h))

    def backward_ms(self) -> float:
        return float(self._lib.swb_rollout_backward_ms(self._h))


def rollout_forward_many(rollouts, settings: abi.StepSettings, targets, weights) -> np.ndarray:
    """The forwards of several rollouts at once (swb_rollout_forward_many):
    their structures run side by side on the device.  Returns the losses."""
    lib = abi.library()
    k = len(rollouts)
    ts = [np.ascontiguousarray(t, dtype=np.float64).reshape(r._structure.node_count, 3)
          for r, t in zip(rollouts, targets)]
    ws = [np.ascontiguousarray(w, dtype=np.float64).reshape(r._structure.node_count) for r, w in zip(rollouts, weights)]
    handles = (C.c_void_p * k)(*[r._h for r in rollouts])
    tp = (C.c_void_p * k)(*[t.ctypes.data for t in ts])
    wp = (C.c_void_p * k)(*[w.ctypes.data for w in ws])
    losses = np.zeros(k)
    statuses = np.zeros(k, dtype=np.int32)
    _check(lib.swb_rollout_forward_many(handles, k, C.byref(settings), tp, wp, losses.ctypes.data,
                                        statuses.ctypes.data))
    return losses


def rollout_backward_many(rollouts, statuses: np.ndarray | None = None) -> list:
    """The backwards of several rollouts at once (swb_rollout_backward_many);
    one gradient dict per rollout, as Rollout.backward returns it.  With
    `statuses` (an int32 array, one entry per rollout) the call fills it and
    raises only when it fails as a whole (each rollout's own failure, as
    SWB_NON_FINITE for an overflowed gradient, is left in its entry)."""
    lib = abi.library()
    k = len(rollouts)
    bufs = [r._gradient_buffers() for r in rollouts]
    grads = (abi.RolloutGradient * k)(*[b[1] for b in bufs])
    handles = (C.c_void_p * k)(*[r._h for r in rollouts])
    own = statuses is None
    st = np.zeros(k, dtype=np.int32) if own else statuses
    assert st.dtype == np.int32 and st.shape == (k,)
    status = lib.swb_rollout_backward_many(handles, k, grads, st.ctypes.data)
    if own or not (st != abi.OK).any():
        _check(status)
    return [Rollout._gradient_result(out, sizes) for out, _, sizes in bufs]
