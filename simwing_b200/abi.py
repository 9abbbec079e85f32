"""ctypes mirror of include/simwing_b200.h (the library's C-ABI).

Only plain C types cross the boundary; this module declares the structs and
function prototypes so Python callers (tests, bench) see the same surface a
C or C++ host binds.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "libsimwing_b200.so")


class Vec3(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


class Quat(C.Structure):
    _fields_ = [("w", C.c_double), ("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


class NodeDef(C.Structure):
    _fields_ = [("position", Vec3), ("mass", C.c_double), ("fixed", C.c_uint32), ("reserved", C.c_uint32)]


class TriangleDef(C.Structure):
    _fields_ = [("nodes", C.c_uint64 * 3), ("pressure_difference", C.c_double)]


class ConstraintDef(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("reserved", C.c_uint32), ("first_node", C.c_uint64),
                ("second_node", C.c_uint64), ("rest_length", C.c_double), ("compliance", C.c_double)]


class MembraneMaterial(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "warp_stiffness", "weft_stiffness", "coupling_stiffness", "shear_stiffness",
        "warp_pretension", "weft_pretension", "damping_seconds", "compression_stiffness_ratio")]


ROLE_BULK, ROLE_SEAM, ROLE_REINFORCEMENT = 1, 2, 3


class MembraneDef(C.Structure):
    _fields_ = [("triangle", C.c_uint64), ("chart", (C.c_double * 2) * 3), ("material", MembraneMaterial),
                ("role", C.c_uint32), ("reserved", C.c_uint32)]


class DihedralDef(C.Structure):
    _fields_ = [("nodes", C.c_uint64 * 4), ("rest_angle", C.c_double), ("compliance", C.c_double)]


class FabricContactDef(C.Structure):
    _fields_ = [("half_thickness", C.c_double), ("normal_compliance", C.c_double),
                ("static_friction", C.c_double), ("dynamic_friction", C.c_double)]


class SuspensionEndpoint(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("reserved", C.c_uint32), ("stable_id", C.c_uint64)]


class SuspensionAttachment(C.Structure):
    _fields_ = [("stable_id", C.c_uint64), ("node", C.c_uint64)]


class SuspensionJunction(C.Structure):
    _fields_ = [("stable_id", C.c_uint64), ("node", C.c_uint64)]


class PilotHarness(C.Structure):
    _fields_ = [("stable_id", C.c_uint64), ("local_position", Vec3)]


class SuspensionSegment(C.Structure):
    _fields_ = [("stable_id", C.c_uint64), ("from_", SuspensionEndpoint), ("to", SuspensionEndpoint),
                ("rest_length", C.c_double), ("axial_stiffness", C.c_double), ("axial_damping", C.c_double),
                ("role", C.c_uint32), ("reserved", C.c_uint32)]


class SuspensionDef(C.Structure):
    _fields_ = [("pilot_stable_id", C.c_uint64), ("pilot_mass", C.c_double), ("pilot_com_local", Vec3),
                ("pilot_initial_com_world", Vec3), ("pilot_initial_linear_velocity", Vec3),
                ("pilot_initial_angular_velocity", Vec3), ("pilot_initial_body_to_world", Quat),
                ("pilot_principal_inertia", Vec3),
                ("attachment_count", C.c_uint64), ("attachments", C.POINTER(SuspensionAttachment)),
                ("junction_count", C.c_uint64), ("junctions", C.POINTER(SuspensionJunction)),
                ("harness_count", C.c_uint64), ("harness_points", C.POINTER(PilotHarness)),
                ("segment_count", C.c_uint64), ("segments", C.POINTER(SuspensionSegment)),
                ("solver_iterations", C.c_int32), ("reserved", C.c_int32),
                ("attachment_tolerance", C.c_double), ("minimum_line_length", C.c_double),
                ("maximum_line_residual", C.c_double), ("maximum_control_work", C.c_double)]


class StructureDefinition(C.Structure):
    _fields_ = [("node_count", C.c_uint64), ("nodes", C.POINTER(NodeDef)),
                ("triangle_count", C.c_uint64), ("triangles", C.POINTER(TriangleDef)),
                ("constraint_count", C.c_uint64), ("constraints", C.POINTER(ConstraintDef)),
                ("membrane_count", C.c_uint64), ("membranes", C.POINTER(MembraneDef)),
                ("dihedral_count", C.c_uint64), ("dihedrals", C.POINTER(DihedralDef)),
                ("fabric_self_contact", C.POINTER(FabricContactDef)),
                ("suspension", C.POINTER(SuspensionDef))]


FEATURE_VERTEX_TRIANGLE, FEATURE_EDGE_EDGE, FEATURE_SEGMENT_TRIANGLE = 0, 1, 2
GEOMETRY_CERTIFIED, GEOMETRY_DEGENERATE, GEOMETRY_NON_FINITE, GEOMETRY_UNCERTIFIABLE = 0, 1, 2, 3
CCD_NO_IMPACT, CCD_IMPACT, CCD_INITIALLY_PROXIMATE, CCD_INDETERMINATE = 0, 1, 2, 3
CCD_MAX_SUBDIVISIONS = 4096


class ContactKey(C.Structure):
    _fields_ = [("pair", C.c_uint64), ("kind", C.c_uint32), ("reserved", C.c_uint32),
                ("first", C.c_uint64 * 3), ("second", C.c_uint64 * 3)]


# Scene assembly (swb_assemble_scene)
class SceneVertex(C.Structure):
    _fields_ = [("id", C.c_uint64), ("position", Vec3)]


class SceneFabric(C.Structure):
    _fields_ = [("id", C.c_uint64)] + [(n, C.c_double) for n in (
        "warp_stiffness", "weft_stiffness", "shear_stiffness", "bending_stiffness", "areal_density",
        "damping_seconds", "porosity", "permeability")]


class SceneTriangle(C.Structure):
    _fields_ = [("id", C.c_uint64), ("vertex_ids", C.c_uint64 * 3), ("chart", (C.c_double * 2) * 3),
                ("material_id", C.c_uint64), ("sheet_id", C.c_uint64)]


class SceneSeamMaterial(C.Structure):
    _fields_ = [("id", C.c_uint64), ("linear_density", C.c_double), ("axial_stiffness", C.c_double)]


class SceneSeam(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("id", "material_id", "first_begin", "second_begin", "count")]


class SceneLineMaterial(C.Structure):
    _fields_ = [("id", C.c_uint64)] + [(n, C.c_double) for n in (
        "diameter", "linear_density", "axial_stiffness", "drag_coefficient")]


class ScenePilot(C.Structure):
    _fields_ = [("id", C.c_uint64), ("mass", C.c_double), ("center_of_mass", Vec3), ("linear_velocity", Vec3),
                ("body_to_world", Quat), ("principal_inertia", Vec3)]


class SceneJunction(C.Structure):
    _fields_ = [("id", C.c_uint64), ("position", Vec3), ("mass", C.c_double), ("fixed", C.c_uint32),
                ("reserved", C.c_uint32)]


ATTACH_SURFACE_VERTEX, ATTACH_PILOT_HARNESS, ATTACH_JUNCTION = 1, 2, 3


class SceneAttachment(C.Structure):
    _fields_ = [("id", C.c_uint64), ("kind", C.c_uint32), ("reserved", C.c_uint32), ("vertex_id", C.c_uint64),
                ("pilot_id", C.c_uint64), ("junction_id", C.c_uint64), ("pilot_local_position", Vec3)]


class SceneLine(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("id", "start_attachment_id", "end_attachment_id", "material_id")] + \
               [("rest_length", C.c_double), ("role", C.c_uint32), ("reserved", C.c_uint32)]


SCENE_ARRAYS = (("vertex", SceneVertex, "vertices"), ("fabric", SceneFabric, "fabrics"),
                ("triangle", SceneTriangle, "triangles"), ("seam_material", SceneSeamMaterial, "seam_materials"),
                ("seam", SceneSeam, "seams"), ("seam_vertex_id", C.c_uint64, "seam_vertex_ids"),
                ("line_material", SceneLineMaterial, "line_materials"), ("pilot", ScenePilot, "pilots"),
                ("junction", SceneJunction, "junctions"), ("attachment", SceneAttachment, "attachments"),
                ("line", SceneLine, "lines"))


class Scene(C.Structure):
    _fields_ = [f for name, ctype, field in SCENE_ARRAYS for f in ((name + "_count", C.c_uint64),
                                                                   (field, C.POINTER(ctype)))]


class SceneSettings(C.Structure):
    _fields_ = [("seam_coincidence_tolerance", C.c_double), ("suspension_solver_iterations", C.c_int32),
                ("has_fabric_self_contact", C.c_uint32), ("suspension_attachment_tolerance", C.c_double),
                ("suspension_minimum_line_length", C.c_double), ("suspension_maximum_line_residual", C.c_double),
                ("suspension_maximum_control_work", C.c_double), ("fabric_self_contact", FabricContactDef)]


class SceneReport(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("assembled", "diagnostic_count", "first_code", "first_validation_code",
                                           "first_entity_kind", "reserved")] + \
               [("first_entity_id", C.c_uint64), ("total_fabric_mass", C.c_double), ("total_seam_mass", C.c_double),
                ("first_message", C.c_char * 160)]


# softwing::SuspensionPhase in declaration order (suspension.h:27-38)
SUSPENSION_PHASES = ("Parse", "Validation", "AttachmentResolution", "GraphConstruction", "Control", "Prediction",
                     "LineSolve", "GroundSolve", "Certification", "Diagnostics")


class ErrorDetail(C.Structure):
    _fields_ = [("status", C.c_uint32), ("suspension_phase", C.c_uint32), ("suspension_entity", C.c_char * 128),
                ("has_contact_key", C.c_uint32), ("reserved", C.c_uint32), ("contact_key", ContactKey)]


class AirProperties(C.Structure):
    _fields_ = [("specific_gas_constant", C.c_double), ("heat_capacity_ratio", C.c_double)]


# swb_flow_zone_state, swb_port_def and swb_mass_flow as numpy records
ZONE_DTYPE = np.dtype([("absolute_pressure", "<f8"), ("absolute_temperature", "<f8")])
PORT_DTYPE = np.dtype([("kind", "<u4"), ("reserved", "<u4"), ("first", "<u8"), ("second", "<u8"),
                       ("discharge_coefficient", "<f8"), ("effective_area", "<f8"), ("mass_conductance", "<f8"),
                       ("opening_fraction", "<f8")])
FLOW_DTYPE = np.dtype([("signed_mass_rate", "<f8"), ("magnitude", "<f8"), ("pressure_ratio", "<f8"),
                       ("critical_pressure_ratio", "<f8"), ("direction", "<u4"), ("choked", "<u4")])
PORT_ORIFICE, PORT_CONDUCTANCE = 0, 1
FLOW_EQUILIBRIUM, FLOW_FIRST_TO_SECOND, FLOW_SECOND_TO_FIRST = 0, 1, 2


class CcdSettings(C.Structure):
    _fields_ = [("conservative_iterations", C.c_int32), ("interval_subdivisions", C.c_int32),
                ("time_tolerance", C.c_double), ("distance_tolerance", C.c_double)]


class ClosestResult(C.Structure):
    _fields_ = [("status", C.c_uint32), ("first_feature", C.c_uint32), ("second_feature", C.c_uint32),
                ("reserved", C.c_uint32)] + [(n, C.c_double * 3) for n in (
                    "first_point", "second_point", "first_weights", "second_weights", "normal")] + [
                ("distance", C.c_double), ("gap", C.c_double)]


class CcdResult(C.Structure):
    _fields_ = [("state", C.c_uint32), ("conservative_iterations", C.c_int32), ("interval_subdivisions", C.c_int32),
                ("used_interval_fallback", C.c_uint32), ("time_of_impact", C.c_double),
                ("bracket_lower", C.c_double), ("bracket_upper", C.c_double), ("geometry", ClosestResult)]


class StepSettings(C.Structure):
    _fields_ = [("time_step", C.c_double), ("substeps", C.c_int32), ("constraint_iterations", C.c_int32),
                ("cable_sweep_pairs", C.c_int32), ("worker_threads", C.c_uint32), ("gravity", Vec3),
                ("velocity_damping", C.c_double), ("damping_reference_velocity", Vec3)]


class Diagnostics(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "node_count", "dynamic_node_count", "triangle_count", "constraint_count", "membrane_count",
        "dihedral_count", "contact_pair_count", "active_contact_count", "suspension_segment_count")] + [
        ("total_dynamic_mass", C.c_double), ("center_of_mass", Vec3), ("linear_momentum", Vec3),
        ("kinetic_energy", C.c_double), ("maximum_distance_error", C.c_double),
        ("maximum_cable_extension", C.c_double), ("maximum_absolute_membrane_strain", C.c_double),
        ("maximum_membrane_residual", C.c_double), ("maximum_contact_penetration", C.c_double),
        ("maximum_suspension_residual", C.c_double), ("pending_external_force", Vec3),
        ("last_applied_external_force", Vec3), ("finite", C.c_uint32), ("reserved", C.c_uint32)]


class NodeState(C.Structure):
    _fields_ = [("position", Vec3), ("previous_position", Vec3), ("velocity", Vec3)]


class PayloadState(C.Structure):
    _fields_ = [("center_of_mass", Vec3), ("body_to_world", Quat), ("linear_velocity", Vec3),
                ("angular_velocity", Vec3)]


class SegmentState(C.Structure):
    _fields_ = [("stable_id", C.c_uint64), ("current_length", C.c_double),
                ("commanded_rest_length", C.c_double), ("tension", C.c_double)]


class Ground(C.Structure):
    _fields_ = [("normal", Vec3), ("offset", C.c_double), ("friction", C.c_double), ("enabled", C.c_uint32),
                ("reserved", C.c_uint32)]


class LineContact(C.Structure):
    _fields_ = [("radius", C.c_double), ("margin", C.c_double), ("enabled", C.c_uint32), ("reserved", C.c_uint32)]


class Wrench(C.Structure):
    _fields_ = [("force", Vec3), ("moment", Vec3)]


class SolverOptions(C.Structure):
    _fields_ = [("device", C.c_int32), ("blocks", C.c_int32), ("block_threads", C.c_int32),
                ("partition_levels", C.c_int32), ("cluster_ctas", C.c_int32), ("flags", C.c_uint32),
                ("sync_budget_cycles", C.c_int64)]


class ScheduleReport(C.Structure):
    _fields_ = [("blocks", C.c_int32), ("block_threads", C.c_int32), ("partition_levels", C.c_int32),
                ("device_phases_per_iteration", C.c_int32), ("local_stages_per_iteration", C.c_int32),
                ("global_colours_per_iteration", C.c_int32), ("max_patch_nodes", C.c_int32),
                ("shared_bytes", C.c_int32), ("level_constraints", C.c_uint64 * 4),
                ("global_constraints", C.c_uint64), ("cluster_ctas", C.c_int32),
                ("cluster_barriers_per_iteration", C.c_int32)]


class BatchOptions(C.Structure):
    _fields_ = [("device", C.c_int32), ("cluster_ctas", C.c_int32), ("target_patch_nodes", C.c_int32),
                ("block_threads", C.c_int32), ("graph_steps", C.c_int32), ("flags", C.c_uint32),
                ("autotune_iterations", C.c_int32), ("reserved", C.c_int32)]


class BatchReport(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "structures", "clusters", "cluster_ctas", "idle_ctas", "block_threads", "target_patch_nodes",
        "shared_bytes", "max_cluster_stages", "resident_clusters", "colours_per_sync", "autotune_candidates",
        "reserved")] + [("candidate_patch_nodes", C.c_int32 * 8), ("candidate_ms_per_step", C.c_double * 8),
                        ("candidate_block_threads", C.c_int32 * 8)]


class RolloutGradient(C.Structure):
    _fields_ = [("d_rest", C.c_void_p), ("d_compliance", C.c_void_p), ("d_dihedral_compliance", C.c_void_p),
                ("d_segment_rest", C.c_void_p), ("d_pilot_mass", C.c_void_p)]


class PatchParams(C.Structure):
    _fields_ = [("nx", C.c_uint32), ("ny", C.c_uint32), ("width", C.c_double), ("height", C.c_double),
                ("areal_density", C.c_double), ("distance_compliance", C.c_double),
                ("bend_compliance", C.c_double), ("jitter", C.c_double), ("seed", C.c_uint64),
                ("pin_top_corners", C.c_uint32), ("membranes", C.c_uint32)]


class WingParams(C.Structure):
    _fields_ = [("cells", C.c_uint32), ("chordwise", C.c_uint32), ("spanwise_per_cell", C.c_uint32),
                ("rib_layers", C.c_uint32), ("span", C.c_double), ("root_chord", C.c_double),
                ("thickness", C.c_double), ("areal_density", C.c_double), ("skin_compliance", C.c_double),
                ("bend_rigidity", C.c_double), ("line_compliance_scale", C.c_double), ("pressure", C.c_double),
                ("line_levels", C.c_uint32), ("line_particles", C.c_uint32), ("line_rows", C.c_uint32),
                ("pilot", C.c_uint32), ("pilot_mass", C.c_double), ("aspect_ratio", C.c_double),
                ("compliance_jitter", C.c_double), ("seed", C.c_uint64), ("fabric", C.c_uint32),
                ("attachments_per_cell", C.c_uint32)]


FAST_ATAN2, FAST_RCP = 0, 1

# status codes
OK, INVALID_ARGUMENT, OUT_OF_RANGE, SUSPENSION_ERROR, CONTACT_ERROR, NON_FINITE, SYNC_TIMEOUT, \
    CUDA_ERROR, UNSUPPORTED, OUT_OF_MEMORY = range(10)

DISTANCE, CABLE, SUSPENSION_TIE, SEAM_STITCH = 1, 2, 3, 4
OPT_GLOBAL_ONLY, OPT_NO_GRAPH, OPT_GRID, OPT_SPLIT_STAGES, OPT_AUTOTUNE, OPT_CONTACT_ONE_CLUSTER = 1, 2, 4, 8, 16, 32


class AutotuneCandidate(C.Structure):
    _fields_ = [("cluster_ctas", C.c_int32), ("block_threads", C.c_int32), ("split_stages", C.c_uint32),
                ("stages_per_iteration", C.c_int32), ("ms_per_substep", C.c_double)]


class AutotuneReport(C.Structure):
    _fields_ = [("candidates", C.c_uint32), ("chosen", C.c_uint32), ("iterations", C.c_uint32),
                ("reserved", C.c_uint32), ("entries", AutotuneCandidate * 16)]
BATCH_AUTOTUNE = 1 << 8
SWEEP_DISTANCE, SWEEP_DIHEDRAL, SWEEP_MEMBRANE = 0, 1, 2

P = C.POINTER
_PROTOTYPES = {
    "swb_last_error": (C.c_char_p, []),
    "swb_last_error_detail": (C.c_int, [C.POINTER(ErrorDetail)]),
    "swb_abi_version": (C.c_uint32, []),
    "swb_default_step_settings": (None, [P(StepSettings)]),
    "swb_default_solver_options": (None, [P(SolverOptions)]),
    "swb_structure_create": (C.c_int, [P(StructureDefinition), P(SolverOptions), P(C.c_void_p)]),
    "swb_structure_destroy": (None, [C.c_void_p]),
    "swb_structure_fingerprint": (C.c_uint64, [C.c_void_p]),
    "swb_structure_accepted_steps": (C.c_uint64, [C.c_void_p]),
    "swb_structure_simulation_time": (C.c_double, [C.c_void_p]),
    "swb_structure_node_count": (C.c_uint64, [C.c_void_p]),
    "swb_structure_clear_external_forces": (C.c_int, [C.c_void_p]),
    "swb_structure_add_external_force": (C.c_int, [C.c_void_p, C.c_uint64, P(Vec3)]),
    "swb_structure_set_external_forces": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "swb_structure_set_face_pressure": (C.c_int, [C.c_void_p, C.c_uint64, C.c_double]),
    "swb_structure_set_uniform_pressure": (C.c_int, [C.c_void_p, C.c_double]),
    "swb_structure_set_ground": (C.c_int, [C.c_void_p, C.c_void_p]),
    "swb_structure_set_line_contact": (C.c_int, [C.c_void_p, C.c_void_p]),
    "swb_structure_step": (C.c_int, [C.c_void_p, P(StepSettings), P(Diagnostics)]),
    "swb_structure_step_many": (C.c_int, [C.c_void_p, P(StepSettings), C.c_int32, P(Diagnostics)]),
    "swb_structure_diagnostics": (C.c_int, [C.c_void_p, P(Diagnostics)]),
    "swb_diagnostics_noalloc": (C.c_int, [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, P(Diagnostics)]),
    "swb_fast_math_eval": (C.c_int, [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64]),
    "swb_structure_read_nodes": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "swb_structure_read_positions_f32": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "swb_structure_write_nodes": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "swb_structure_read_suspension": (C.c_int, [C.c_void_p, P(PayloadState), C.c_void_p, C.c_uint64,
                                                P(Wrench)]),
    "swb_structure_write_payload": (C.c_int, [C.c_void_p, P(PayloadState)]),
    "swb_structure_checkpoint_size": (C.c_int, [C.c_void_p, P(C.c_uint64)]),
    "swb_structure_checkpoint": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "swb_structure_restore": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "swb_structure_sweep_order": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64]),
    "swb_structure_schedule_report": (C.c_int, [C.c_void_p, P(ScheduleReport)]),
    "swb_structure_last_step_ms": (C.c_double, [C.c_void_p]),
    "swb_plan_schedule": (C.c_int, [P(StructureDefinition), P(SolverOptions), P(ScheduleReport), C.c_void_p,
                                    C.c_void_p]),
    "swb_plan_membrane_order": (C.c_int, [P(StructureDefinition), P(SolverOptions), C.c_void_p]),
    "swb_default_scene_settings": (None, [P(SceneSettings)]),
    "swb_assemble_scene": (C.c_int, [P(Scene), P(SceneSettings), P(C.c_void_p), P(SceneReport)]),
    "swb_structure_autotune_report": (C.c_int, [C.c_void_p, P(AutotuneReport)]),
    "swb_default_batch_options": (None, [P(BatchOptions)]),
    "swb_batch_create": (C.c_int, [C.c_void_p, C.c_uint64, P(BatchOptions), P(C.c_void_p)]),
    "swb_batch_destroy": (None, [C.c_void_p]),
    "swb_batch_size": (C.c_uint64, [C.c_void_p]),
    "swb_batch_structure": (C.c_void_p, [C.c_void_p, C.c_uint64]),
    "swb_batch_step": (C.c_int, [C.c_void_p, P(StepSettings), C.c_int32, C.c_void_p]),
    "swb_batch_set_ground": (C.c_int, [C.c_void_p, C.c_void_p]),
    "swb_batch_get_report": (C.c_int, [C.c_void_p, P(BatchReport)]),
    "swb_batch_last_step_ms": (C.c_double, [C.c_void_p]),
    "swb_rollout_create": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, P(C.c_void_p)]),
    "swb_rollout_destroy": (None, [C.c_void_p]),
    "swb_rollout_forward": (C.c_int, [C.c_void_p, P(StepSettings), C.c_void_p, C.c_void_p, P(C.c_double)]),
    "swb_rollout_backward": (C.c_int, [C.c_void_p, P(RolloutGradient)]),
    "swb_rollout_forward_many": (C.c_int, [C.c_void_p, C.c_uint64, P(StepSettings), C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p]),
    "swb_rollout_backward_many": (C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]),
    "swb_rollout_final_positions": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "swb_rollout_forward_ms": (C.c_double, [C.c_void_p]),
    "swb_rollout_backward_ms": (C.c_double, [C.c_void_p]),
    "swb_reference_colouring": (C.c_int, [P(StructureDefinition), C.c_void_p, C.c_void_p, C.c_uint64,
                                          P(C.c_uint64), P(C.c_uint64)]),
    "swb_default_patch_params": (None, [P(PatchParams)]),
    "swb_default_wing_params": (None, [P(WingParams)]),
    "swb_generate_patch": (C.c_int, [P(PatchParams), P(C.c_void_p)]),
    "swb_generate_wing": (C.c_int, [P(WingParams), P(C.c_void_p)]),
    "swb_definition_copy": (C.c_int, [P(StructureDefinition), P(C.c_void_p)]),
    "swb_definition_permute": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "swb_definition_permute_membranes": (C.c_int, [C.c_void_p, C.c_void_p]),
    "swb_definition_scale_rest": (C.c_int, [C.c_void_p, C.c_uint64, C.c_double]),
    "swb_definition_view": (P(StructureDefinition), [C.c_void_p]),
    "swb_definition_destroy": (None, [C.c_void_p]),
    "swb_definition_fingerprint": (C.c_uint64, [P(StructureDefinition)]),
    "swb_validate_definition": (C.c_int, [P(StructureDefinition)]),
    "swb_default_ccd_settings": (None, [P(CcdSettings)]),
    "swb_definition_set_contact": (C.c_int, [C.c_void_p, P(FabricContactDef)]),
    "swb_structure_contact_candidates": (C.c_int, [C.c_void_p, P(ContactKey), C.c_uint64, P(C.c_uint64)]),
    "swb_coupling_create": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, P(C.c_void_p)]),
    "swb_coupling_destroy": (None, [C.c_void_p]),
    "swb_coupling_advance_impulses": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, P(StepSettings), P(Diagnostics)]),
    "swb_coupling_advance_endpoint_loads": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, P(StepSettings),
                                                      P(Diagnostics)]),
    "swb_contact_candidates": (C.c_int, [P(StructureDefinition), C.c_double, C.c_void_p, C.c_void_p, P(ContactKey),
                                         C.c_uint64, P(C.c_uint64), P(C.c_uint64), P(C.c_uint64)]),
    "swb_port_mass_flows": (C.c_int, [P(AirProperties), C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p,
                                      P(C.c_uint64)]),
    "swb_port_mass_flows_device": (C.c_int, [P(AirProperties), C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64,
                                             C.c_void_p, C.c_void_p, C.c_void_p]),
    "swb_cell_volume_plan_create": (C.c_int, [P(StructureDefinition), C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                                              C.c_int, P(C.c_void_p)]),
    "swb_cell_volume_plan_destroy": (None, [C.c_void_p]),
    "swb_cell_volumes_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "swb_structure_cell_volumes": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "swb_contact_closest": (C.c_int, [C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p, C.c_double, P(ClosestResult)]),
    "swb_contact_sweep": (C.c_int, [C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_double, P(CcdSettings), P(CcdResult)]),
}

# Entry points the header declares; tests check the library exports each.
DECLARED_SYMBOLS = sorted(_PROTOTYPES)


def bind(lib: C.CDLL, prototypes=None) -> C.CDLL:
    for name, (restype, argtypes) in (prototypes or _PROTOTYPES).items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    return lib


_LIB = None


def library() -> C.CDLL:
    """Loads the in-tree CUDA library; raises if it has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIBRARY_PATH):
            raise ImportError(
                f"{LIBRARY_PATH} is missing: build it with `make -C simwing_b200` "
                "(or __graft_entry__.build()); there is no CPU fallback")
        _LIB = bind(C.CDLL(LIBRARY_PATH))
    return _LIB
