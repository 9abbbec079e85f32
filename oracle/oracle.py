"""ORACLE / TEST INFRASTRUCTURE ONLY.

ctypes loaders for the CPU checkers:
  * PortStructure -- oracle/liboracle.so, the plain-C FP64 restatement of
    the reference step (oracle/xpbd_oracle.c); with float_vectors=True,
    oracle/liboracle_f32.so, the same step with every vector result rounded
    to FP32 (the tests' measure of a configuration's FP32 sensitivity);
  * RefStructure  -- oracle/_ref/libswref.so, the reference's own
    softwing core + Structure adapter compiled from source
    (oracle/ref_shim.cpp, oracle/Makefile);
  * rollout_gradient -- oracle/libadjoint.so, the FP64 reference gradient
    of a rollout loss (oracle/xpbd_adjoint.cpp).
All take the product's swb_structure_definition, so the device solver and
the checkers run on identical inputs.  Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from simwing_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_PATH = os.path.join(HERE, "liboracle.so")
PORT_F32_PATH = os.path.join(HERE, "liboracle_f32.so")
REF_PATH = os.path.join(HERE, "_ref", "libswref.so")
ADJOINT_PATH = os.path.join(HERE, "libadjoint.so")

P = C.POINTER
_PORT = {
    "swo_last_error": (C.c_char_p, []),
    "swo_create": (C.c_int, [P(abi.StructureDefinition), P(C.c_void_p)]),
    "swo_destroy": (None, [C.c_void_p]),
    "swo_set_external_forces": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "swo_add_external_force": (C.c_int, [C.c_void_p, C.c_uint64, P(abi.Vec3)]),
    "swo_step": (C.c_int, [C.c_void_p, P(abi.StepSettings)]),
    "swo_diagnostics": (C.c_int, [C.c_void_p, P(abi.Diagnostics)]),
    "swo_read_nodes": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "swo_write_nodes": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "swo_read_payload": (C.c_int, [C.c_void_p, P(abi.PayloadState), P(abi.Wrench), P(C.c_double)]),
    "swo_write_payload": (C.c_int, [C.c_void_p, P(abi.PayloadState)]),
    "swo_read_segment_lambdas": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "swo_evaluate_dihedral": (None, [C.c_void_p, C.c_void_p]),
    "swo_set_ground": (C.c_int, [C.c_void_p, C.c_void_p]),
    "swo_set_line_contact": (C.c_int, [C.c_void_p, C.c_void_p]),
}
_REF = {
    "swref_last_error": (C.c_char_p, []),
    "swref_physical_cores": (C.c_uint, []),
    "swref_last_error_detail": (C.c_int, [P(abi.ErrorDetail)]),
    "swref_assemble_scene": (C.c_int, [P(abi.Scene), P(abi.SceneSettings), P(C.c_void_p), P(abi.SceneReport)]),
    "swref_assembly_view": (P(abi.StructureDefinition), [C.c_void_p]),
    "swref_assembly_destroy": (None, [C.c_void_p]),
    "swref_create": (C.c_int, [P(abi.StructureDefinition), P(C.c_void_p)]),
    "swref_destroy": (None, [C.c_void_p]),
    "swref_fingerprint": (C.c_uint64, [C.c_void_p]),
    "swref_set_external_forces": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "swref_add_external_force": (C.c_int, [C.c_void_p, C.c_uint64, P(abi.Vec3)]),
    "swref_step": (C.c_int, [C.c_void_p, P(abi.StepSettings), P(abi.Diagnostics)]),
    "swref_last_step_seconds": (C.c_double, [C.c_void_p]),
    "swref_diagnostics": (C.c_int, [C.c_void_p, P(abi.Diagnostics)]),
    "swref_read_nodes": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "swref_read_suspension": (C.c_int, [C.c_void_p, P(abi.PayloadState), C.c_void_p, C.c_uint64]),
    "swref_colouring": (C.c_int, [P(abi.StructureDefinition), C.c_void_p, C.c_void_p, C.c_uint64,
                                  P(C.c_uint64), P(C.c_uint64)]),
    "swref_contact_candidates": (C.c_int, [P(abi.StructureDefinition), C.c_double, C.c_void_p, C.c_void_p,
                                           P(abi.ContactKey), C.c_uint64, P(C.c_uint64), P(C.c_uint64),
                                           P(C.c_uint64)]),
    "swref_port_mass_flows": (C.c_int, [P(abi.AirProperties), C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64,
                                        C.c_void_p, P(C.c_uint64)]),
    "swref_contact_closest": (C.c_int, [C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p, C.c_double,
                                        P(abi.ClosestResult)]),
    "swref_contact_sweep": (C.c_int, [C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_double, P(abi.CcdSettings), P(abi.CcdResult)]),
}

_ADJ = {
    "swa_last_error": (C.c_char_p, []),
    "swa_rollout_gradient": (C.c_int, [P(abi.StructureDefinition), P(abi.StepSettings), C.c_int, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       P(C.c_double), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       P(C.c_double), C.c_void_p, C.c_void_p]),
}

_libs = {}


def port_available() -> bool:
    return os.path.exists(PORT_PATH)


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def port_library(float_vectors: bool = False) -> C.CDLL:
    key = "port_f32" if float_vectors else "port"
    if key not in _libs:
        _libs[key] = abi.bind(C.CDLL(PORT_F32_PATH if float_vectors else PORT_PATH), _PORT)
    return _libs[key]


def ref_library() -> C.CDLL:
    if "ref" not in _libs:
        _libs["ref"] = abi.bind(C.CDLL(REF_PATH), _REF)
    return _libs["ref"]


class OracleError(RuntimeError):
    """A checker's failure; for the reference build's SuspensionError and
    ContactStepError also `phase`/`entity` or `key`, as the product's
    exceptions carry them."""

    def __init__(self, status, message, phase=None, entity=None, key=None):
        super().__init__(f"status {status}: {message}")
        self.status = status
        self.phase, self.entity, self.key = phase, entity, key


class _Base:
    _prefix = ""

    def _lib(self):
        raise NotImplementedError

    def _check(self, status):
        if status != 0:
            message = getattr(self._lib(), self._prefix + "last_error")().decode()
            phase = entity = key = None
            if self._prefix == "swref_" and status in (abi.SUSPENSION_ERROR, abi.CONTACT_ERROR):
                d = abi.ErrorDetail()
                ref_library().swref_last_error_detail(C.byref(d))
                if status == abi.SUSPENSION_ERROR:
                    phase = abi.SUSPENSION_PHASES[d.suspension_phase]
                    entity = d.suspension_entity.decode(errors="replace")
                else:
                    k = d.contact_key
                    key = (int(k.pair), int(k.kind), tuple(int(x) for x in k.first), tuple(int(x) for x in k.second))
            raise OracleError(status, message, phase, entity, key)

    def __init__(self, definition):
        self._definition = definition  # keep alive
        h = C.c_void_p()
        self._check(getattr(self._lib(), self._prefix + "create")(definition.pointer, C.byref(h)))
        self._h = h
        self.node_count = int(definition.view.node_count)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            getattr(self._lib(), self._prefix + "destroy")(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        self.close()

    def set_external_forces(self, forces):
        f = np.ascontiguousarray(forces, dtype=np.float64)
        self._check(getattr(self._lib(), self._prefix + "set_external_forces")(self._h, f.ctypes.data, f.shape[0]))

    def add_external_force(self, node, force):
        self._check(getattr(self._lib(), self._prefix + "add_external_force")(self._h, node, C.byref(abi.Vec3(*force))))

    def node_states(self):
        out = np.zeros((self.node_count, 3, 3), dtype=np.float64)
        self._check(getattr(self._lib(), self._prefix + "read_nodes")(self._h, out.ctypes.data, self.node_count))
        return out

    def positions(self):
        return self.node_states()[:, 0, :]

    def diagnostics(self):
        d = abi.Diagnostics()
        self._check(getattr(self._lib(), self._prefix + "diagnostics")(self._h, C.byref(d)))
        return d


class PortStructure(_Base):
    """The C restatement (FP64; float_vectors=True rounds every vector
    result to FP32)."""
    _prefix = "swo_"

    def __init__(self, definition, float_vectors: bool = False):
        self._float_vectors = float_vectors
        super().__init__(definition)

    def _lib(self):
        return port_library(self._float_vectors)

    def step(self, settings):
        """One structure step; returns the diagnostics after it (as the
        reference adapter's step does)."""
        self._check(self._lib().swo_step(self._h, C.byref(settings)))
        return self.diagnostics()

    def write_node_states(self, states):
        s = np.ascontiguousarray(states, dtype=np.float64)
        self._check(self._lib().swo_write_nodes(self._h, s.ctypes.data, self.node_count))

    def payload(self):
        p = abi.PayloadState()
        w = abi.Wrench()
        r = C.c_double()
        self._check(self._lib().swo_read_payload(self._h, C.byref(p), C.byref(w), C.byref(r)))
        return p, w, r.value

    def write_payload(self, p):
        self._check(self._lib().swo_write_payload(self._h, C.byref(p)))

    def set_ground(self, normal=(0.0, 0.0, 1.0), offset=0.0, friction=0.0, enabled=True):
        g = abi.Ground(abi.Vec3(*normal), float(offset), float(friction), 1 if enabled else 0, 0)
        self._check(self._lib().swo_set_ground(self._h, C.byref(g)))

    def set_line_contact(self, radius, margin=0.0, enabled=True):
        lc = abi.LineContact(float(radius), float(margin), 1 if enabled else 0, 0)
        self._check(self._lib().swo_set_line_contact(self._h, C.byref(lc)))

    def segment_lambdas(self, n):
        out = np.zeros(n)
        self._check(self._lib().swo_read_segment_lambdas(self._h, out.ctypes.data, n))
        return out


class RecentredF32:
    """The FP32-rounded restatement (PortStructure(float_vectors=True)) in
    the frame the device keeps: FP32 coordinates relative to an FP64 origin
    on a 1/256 m grid, which starts at the pilot's centre of mass (the
    centre of the nodes' bounding box without a pilot) and moves to the
    pilot's grid point after every step in which the pilot has left the
    origin by more than a quarter metre.  Its long runs show how far FP32
    arithmetic of the reference algorithm itself drifts from the FP64
    run.  positions() and the diagnostics' centre of mass are in world
    coordinates."""

    def __init__(self, definition):
        self._s = PortStructure(definition, float_vectors=True)
        v = definition.view
        if v.suspension:
            c = v.suspension.contents.pilot_initial_com_world
            o = np.array([c.x, c.y, c.z])
        else:
            x = self._s.positions()
            o = 0.5 * (x.min(axis=0) + x.max(axis=0))
        self.origin = np.zeros(3)
        self._has_pilot = bool(v.suspension)
        self._shift(np.round(o * 256.0) / 256.0)

    def _shift(self, d):
        s = self._s.node_states()
        s[:, 0:2, :] -= d
        self._s.write_node_states(s)
        if self._has_pilot:
            p = self._s.payload()[0]
            c = p.center_of_mass
            self._s.write_payload(abi.PayloadState(abi.Vec3(c.x - d[0], c.y - d[1], c.z - d[2]), p.body_to_world,
                                                   p.linear_velocity, p.angular_velocity))
        self.origin = self.origin + d

    def write_state(self, states, payload=None):
        """Node states (and the pilot's state) in world coordinates; the
        origin moves to the pilot's grid point (to the bounding-box centre
        without a pilot)."""
        s = np.array(states, dtype=np.float64)
        if payload is not None:
            c = payload.center_of_mass
            o = np.array([c.x, c.y, c.z])
        else:
            o = 0.5 * (s[:, 0, :].min(axis=0) + s[:, 0, :].max(axis=0))
        o = np.round(o * 256.0) / 256.0
        # as the device stores them: FP32 offsets and velocities
        s[:, 0:2, :] = (s[:, 0:2, :] - o).astype(np.float32)
        s[:, 2, :] = s[:, 2, :].astype(np.float32)
        self._s.write_node_states(s)
        if payload is not None:
            c = payload.center_of_mass
            self._s.write_payload(abi.PayloadState(abi.Vec3(c.x - o[0], c.y - o[1], c.z - o[2]), payload.body_to_world,
                                                   payload.linear_velocity, payload.angular_velocity))
        self.origin = o

    def step(self, settings):
        g = self._s.step(settings)
        c = g.center_of_mass
        g.center_of_mass = abi.Vec3(c.x + self.origin[0], c.y + self.origin[1], c.z + self.origin[2])
        if self._has_pilot:
            pc = self._s.payload()[0].center_of_mass
            pc = np.array([pc.x, pc.y, pc.z])
            if np.abs(pc).max() > 0.25:
                self._shift(np.round(pc * 256.0) / 256.0)
        return g

    def positions(self):
        return self._s.positions() + self.origin

    def close(self):
        self._s.close()


class RefStructure(_Base):
    """The reference's own Structure adapter (FP64, compiled from source)."""
    _prefix = "swref_"

    def _lib(self):
        return ref_library()

    def step(self, settings):
        d = abi.Diagnostics()
        self._check(ref_library().swref_step(self._h, C.byref(settings), C.byref(d)))
        return d

    def last_step_seconds(self):
        return float(ref_library().swref_last_step_seconds(self._h))

    def fingerprint(self):
        return int(ref_library().swref_fingerprint(self._h))

    def payload(self, segments=0):
        p = abi.PayloadState()
        segs = (abi.SegmentState * max(segments, 1))()
        self._check(ref_library().swref_read_suspension(self._h, C.byref(p), segs, segments))
        return p, list(segs)[:segments]


def evaluate_dihedral(points12):
    out = np.zeros(14)
    p = np.ascontiguousarray(points12, dtype=np.float64)
    port_library().swo_evaluate_dihedral(p.ctypes.data, out.ctypes.data)
    return out[0], out[1:13].reshape(4, 3), bool(out[13])


def ref_colouring(definition):
    lib = ref_library()
    m = definition.view.constraint_count
    order = np.zeros(max(m, 1), dtype=np.uint64)
    offsets = np.zeros(4096, dtype=np.uint64)
    colours = C.c_uint64()
    parallel = C.c_uint64()
    status = lib.swref_colouring(definition.pointer, order.ctypes.data, offsets.ctypes.data, offsets.size,
                                 C.byref(colours), C.byref(parallel))
    if status != 0:
        raise OracleError(status, lib.swref_last_error().decode())
    return order[:m], offsets[: colours.value + 1 if m else 0], int(parallel.value)


def adjoint_library() -> C.CDLL:
    if "adjoint" not in _libs:
        _libs["adjoint"] = abi.bind(C.CDLL(ADJOINT_PATH), _ADJ)
    return _libs["adjoint"]


def rollout_gradient(definition, settings, steps, target, weights, forces=None, state=None, payload=None,
                     trajectory=None, trajectory_payloads=None, ground=None, lines=None):
    """FP64 loss and gradient of sum_i w_i |x_i(T) - target_i|^2 / sum w over
    `steps` steps (the definition's insertion order is the sweep order) from
    `state` (N x 3 x 3 node states as read_nodes returns: position, previous,
    velocity; default: the definition at rest) and `payload` (13 values: com,
    orientation wxyz, linear and angular velocity; default: the definition's
    pilot).  `trajectory` (steps x N x 3 x 3) and `trajectory_payloads`
    (steps x 13), when given, restart every step s > 0 from that state, so
    the reverse sweep is evaluated along another solver's trajectory.
    `ground` = (normal xyz, offset) adds the frictionless ground plane;
    `lines` = (radius, margin) adds line-line contact of the cable segments.
    Returns a dict: loss, final (N x 3), d_rest and d_comp
    (per constraint), d_dihedral_comp (per dihedral), d_segment_rest (per
    suspension segment, definition order), d_mass."""
    lib = adjoint_library()
    v = definition.view
    n, m, h = v.node_count, v.constraint_count, v.dihedral_count
    ns = v.suspension.contents.segment_count if v.suspension else 0
    target = np.ascontiguousarray(target, dtype=np.float64).reshape(n, 3)
    weights = np.ascontiguousarray(weights, dtype=np.float64).reshape(n)
    f = None if forces is None else np.ascontiguousarray(forces, dtype=np.float64).reshape(n, 3)
    x0 = None
    if state is not None:
        st = np.asarray(state, dtype=np.float64).reshape(n, 3, 3)
        x0 = np.ascontiguousarray(np.concatenate([st[:, 0, :], st[:, 2, :]], axis=1))
    p0 = None if payload is None else np.ascontiguousarray(payload, dtype=np.float64).reshape(13)
    traj = None
    if trajectory is not None:
        tr = np.asarray(trajectory, dtype=np.float64).reshape(steps, n, 3, 3)
        traj = np.ascontiguousarray(np.concatenate([tr[:, :, 0, :], tr[:, :, 2, :]], axis=2))
    tpay = None if trajectory_payloads is None else \
        np.ascontiguousarray(trajectory_payloads, dtype=np.float64).reshape(steps, 13)
    out = {"final": np.zeros((n, 3)), "d_rest": np.zeros(max(m, 1)), "d_comp": np.zeros(max(m, 1)),
           "d_dihedral_comp": np.zeros(max(h, 1)), "d_segment_rest": np.zeros(max(ns, 1))}
    loss, mass = C.c_double(), C.c_double()
    g = None if ground is None else np.ascontiguousarray([*ground[0], ground[1]], dtype=np.float64)
    lc = None if lines is None else np.ascontiguousarray(lines, dtype=np.float64)
    rc = lib.swa_rollout_gradient(definition.pointer, C.byref(settings), int(steps),
                                  None if x0 is None else x0.ctypes.data, None if p0 is None else p0.ctypes.data,
                                  None if traj is None else traj.ctypes.data,
                                  None if tpay is None else tpay.ctypes.data,
                                  None if f is None else f.ctypes.data, target.ctypes.data, weights.ctypes.data,
                                  C.byref(loss), out["final"].ctypes.data, out["d_rest"].ctypes.data,
                                  out["d_comp"].ctypes.data, out["d_dihedral_comp"].ctypes.data,
                                  out["d_segment_rest"].ctypes.data, C.byref(mass),
                                  None if g is None else g.ctypes.data,
                                  None if lc is None else lc.ctypes.data)
    if rc != 0:
        raise OracleError(abi.INVALID_ARGUMENT, lib.swa_last_error().decode())
    out["d_rest"], out["d_comp"] = out["d_rest"][:m], out["d_comp"][:m]
    out["d_dihedral_comp"], out["d_segment_rest"] = out["d_dihedral_comp"][:h], out["d_segment_rest"][:ns]
    out["loss"], out["d_mass"] = loss.value, mass.value
    return out


def _ref_check(status):
    if status != 0:
        raise OracleError(status, ref_library().swref_last_error().decode())


def ref_contact_candidates(definition, half_thickness, previous, current):
    """The reference's candidate keys of the fabric self-contact pair (one
    SoftBody contact iteration, read through its audit hook); returns
    (keys, possible, excluded)."""
    lib = ref_library()
    prev = np.ascontiguousarray(previous, dtype=np.float64)
    cur = np.ascontiguousarray(current, dtype=np.float64)
    n, possible, excluded = C.c_uint64(), C.c_uint64(), C.c_uint64()
    status = lib.swref_contact_candidates(definition.pointer, half_thickness, prev.ctypes.data, cur.ctypes.data,
                                          None, 0, C.byref(n), C.byref(possible), C.byref(excluded))
    if status not in (abi.OK, abi.OUT_OF_RANGE):
        _ref_check(status)
    keys = (abi.ContactKey * max(n.value, 1))()
    _ref_check(lib.swref_contact_candidates(definition.pointer, half_thickness, prev.ctypes.data, cur.ctypes.data,
                                            keys, n.value, C.byref(n), C.byref(possible), C.byref(excluded)))
    return list(keys)[: n.value], possible.value, excluded.value


def ref_contact_closest(kind, first, second, separation):
    f = np.ascontiguousarray(first, dtype=np.float64).reshape(-1, 9)
    s = np.ascontiguousarray(second, dtype=np.float64).reshape(-1, 9)
    out = (abi.ClosestResult * max(len(f), 1))()
    _ref_check(ref_library().swref_contact_closest(kind, len(f), f.ctypes.data, s.ctypes.data, separation, out))
    return list(out)[: len(f)]


def ref_contact_sweep(kind, first_previous, first_current, second_previous, second_current, separation, settings):
    arrays = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1, 9)
              for a in (first_previous, first_current, second_previous, second_current)]
    n = len(arrays[0])
    out = (abi.CcdResult * max(n, 1))()
    _ref_check(ref_library().swref_contact_sweep(kind, n, *[a.ctypes.data for a in arrays], separation,
                                                 C.byref(settings), out))
    return list(out)[:n]


def ref_port_mass_flows(zones, ports, air=(287.05, 1.4)):
    """The reference's flow laws over many ports (swref_port_mass_flows):
    returns (status, flows, first refusing port)."""
    z = np.array(zones, dtype=abi.ZONE_DTYPE).reshape(-1)
    p = np.array(ports, dtype=abi.PORT_DTYPE).reshape(-1)
    out = np.zeros(len(p), dtype=abi.FLOW_DTYPE)
    failed = C.c_uint64(0)
    a = abi.AirProperties(*air)
    status = ref_library().swref_port_mass_flows(C.byref(a), z.ctypes.data, len(z), p.ctypes.data, len(p),
                                                 out.ctypes.data, C.byref(failed))
    return status, out, failed.value


class RefAssembly:
    """The reference build's assembleSceneStructure of a scene: `report`, and
    `pointer`/`view` of its definition (None when refused)."""

    def __init__(self, scene, settings):
        lib = ref_library()
        self.report = abi.SceneReport()
        self._h = C.c_void_p()
        self.status = lib.swref_assemble_scene(C.byref(scene.view), C.byref(settings), C.byref(self._h),
                                               C.byref(self.report))
        self.view = lib.swref_assembly_view(self._h).contents if self._h.value else None

    @property
    def pointer(self):
        return C.pointer(self.view)

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            ref_library().swref_assembly_destroy(self._h)
            self._h = C.c_void_p()
