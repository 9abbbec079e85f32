/*
 * simwing_b200.h -- C-ABI of the B200 XPBD structural solver.
 *
 * The entry points replace SimWing's structural adapter
 * `simwing::fsi::Structure` (src/fsi/structure.h:273-309) and the XPBD core
 * step it drives (`softwing::SoftBody::step` / `stepCoupled`,
 * src/softwing/soft_body.cpp:981-1070). Only plain C types cross this
 * boundary: fixed-width integers, doubles, floats and pointers with explicit
 * sizes. Every function returns an `swb_status`; on a non-OK status a
 * human-readable message is available from `swb_last_error()` (thread-local).
 *
 * Index fields are 64-bit like the reference's std::size_t indices.
 * Doubles are used on the boundary (the reference is FP64); the device state
 * is FP32.
 */
#ifndef SIMWING_B200_H
#define SIMWING_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SWB_ABI_VERSION 1u

/* ------------------------------------------------------------------------ */
/* Status codes.  The reference throws typed exceptions; each maps to one    */
/* status (std::invalid_argument, std::out_of_range, SuspensionError,         */
/* ContactStepError).  A failed step restores the pre-step state before it   */
/* returns, as Structure::step does (src/fsi/structure.cpp:807-831).         */
/* ------------------------------------------------------------------------ */
typedef enum swb_status {
    SWB_OK = 0,
    SWB_INVALID_ARGUMENT = 1,   /* std::invalid_argument                    */
    SWB_OUT_OF_RANGE = 2,       /* std::out_of_range                        */
    SWB_SUSPENSION_ERROR = 3,   /* softwing::SuspensionError                */
    SWB_CONTACT_ERROR = 4,      /* softwing::ContactStepError               */
    SWB_NON_FINITE = 5,         /* device detected NaN/Inf in the trial step */
    SWB_SYNC_TIMEOUT = 6,       /* a bounded device-wide barrier gave up     */
    SWB_CUDA_ERROR = 7,         /* CUDA runtime failure                      */
    SWB_UNSUPPORTED = 8,        /* feature not available in this build       */
    SWB_OUT_OF_MEMORY = 9
} swb_status;

/* Thread-local message of the last failing call on this thread. */
const char* swb_last_error(void);
uint32_t swb_abi_version(void);

/* ------------------------------------------------------------------------ */
/* Definition: mirrors simwing::fsi::StructureDefinition                     */
/* (src/fsi/structure.h:16-172).                                             */
/* ------------------------------------------------------------------------ */
typedef struct swb_vec3 {
    double x, y, z;
} swb_vec3;

typedef struct swb_quat {
    double w, x, y, z;
} swb_quat;

/* StructureNodeDefinition (structure.h:32-36) */
typedef struct swb_node_def {
    swb_vec3 position;
    double mass;
    uint32_t fixed;
    uint32_t reserved;
} swb_node_def;

/* StructureTriangleDefinition (structure.h:38-40) plus the per-face pressure
 * jump of softwing::Triangle::pressureDifference (soft_body.h:60-65).  A
 * positive value pushes along the right-hand normal of (a, b, c). */
typedef struct swb_triangle_def {
    uint64_t nodes[3];
    double pressure_difference;
} swb_triangle_def;

/* StructureConstraintKind (structure.h:42-47) */
enum {
    SWB_CONSTRAINT_DISTANCE = 1,
    SWB_CONSTRAINT_CABLE = 2,
    SWB_CONSTRAINT_SUSPENSION_TIE = 3,
    SWB_CONSTRAINT_SEAM_STITCH = 4
};

/* StructureConstraintDefinition (structure.h:49-55) */
typedef struct swb_constraint_def {
    uint32_t kind;
    uint32_t reserved;
    uint64_t first_node;
    uint64_t second_node;
    double rest_length;
    double compliance;
} swb_constraint_def;

/* StructureMembraneMaterial (structure.h:63-72) */
typedef struct swb_membrane_material {
    double warp_stiffness;
    double weft_stiffness;
    double coupling_stiffness;
    double shear_stiffness;
    double warp_pretension;
    double weft_pretension;
    double damping_seconds;
    double compression_stiffness_ratio;
} swb_membrane_material;

enum {
    SWB_ROLE_BULK = 1,
    SWB_ROLE_SEAM = 2,
    SWB_ROLE_REINFORCEMENT = 3
};

/* StructureMembraneDefinition (structure.h:74-79) */
typedef struct swb_membrane_def {
    uint64_t triangle;
    double chart[3][2];
    swb_membrane_material material;
    uint32_t role;
    uint32_t reserved;
} swb_membrane_def;

/* StructureDihedralDefinition (structure.h:81-85).  nodes = {a, b, c, d}:
 * a-b is the hinge, c belongs to face (a, b, c), d to face (b, a, d). */
typedef struct swb_dihedral_def {
    uint64_t nodes[4];
    double rest_angle;
    double compliance;
} swb_dihedral_def;

/* StructureFabricContactDefinition (structure.h:90-97) */
typedef struct swb_fabric_contact_def {
    double half_thickness;
    double normal_compliance;
    double static_friction;
    double dynamic_friction;
} swb_fabric_contact_def;

/* StructureSuspensionEndpointKind (structure.h:108-112) */
enum {
    SWB_ENDPOINT_SURFACE_ATTACHMENT = 1,
    SWB_ENDPOINT_JUNCTION = 2,
    SWB_ENDPOINT_PILOT_HARNESS = 3
};

typedef struct swb_suspension_endpoint {
    uint32_t kind;
    uint32_t reserved;
    uint64_t stable_id;
} swb_suspension_endpoint;

typedef struct swb_suspension_attachment {
    uint64_t stable_id;
    uint64_t node;
} swb_suspension_attachment;

typedef struct swb_suspension_junction {
    uint64_t stable_id;
    uint64_t node;
} swb_suspension_junction;

typedef struct swb_pilot_harness {
    uint64_t stable_id;
    swb_vec3 local_position;
} swb_pilot_harness;

/* StructureSuspensionSegmentDefinition (structure.h:133-141) */
typedef struct swb_suspension_segment {
    uint64_t stable_id;
    swb_suspension_endpoint from;
    swb_suspension_endpoint to;
    double rest_length;
    double axial_stiffness;
    double axial_damping;
    uint32_t role;
    uint32_t reserved;
} swb_suspension_segment;

/* StructureSuspensionDefinition (structure.h:143-162) */
typedef struct swb_suspension_def {
    uint64_t pilot_stable_id;
    double pilot_mass;
    swb_vec3 pilot_com_local;
    swb_vec3 pilot_initial_com_world;
    swb_vec3 pilot_initial_linear_velocity;
    swb_vec3 pilot_initial_angular_velocity;
    swb_quat pilot_initial_body_to_world;
    swb_vec3 pilot_principal_inertia;
    uint64_t attachment_count;
    const swb_suspension_attachment* attachments;
    uint64_t junction_count;
    const swb_suspension_junction* junctions;
    uint64_t harness_count;
    const swb_pilot_harness* harness_points;
    uint64_t segment_count;
    const swb_suspension_segment* segments;
    int32_t solver_iterations;
    int32_t reserved;
    double attachment_tolerance;
    double minimum_line_length;
    double maximum_line_residual;
    double maximum_control_work;
} swb_suspension_def;

/* StructureDefinition (structure.h:164-172) */
typedef struct swb_structure_definition {
    uint64_t node_count;
    const swb_node_def* nodes;
    uint64_t triangle_count;
    const swb_triangle_def* triangles;
    uint64_t constraint_count;
    const swb_constraint_def* constraints;
    uint64_t membrane_count;
    const swb_membrane_def* membranes;
    uint64_t dihedral_count;
    const swb_dihedral_def* dihedrals;
    const swb_fabric_contact_def* fabric_self_contact; /* nullable */
    const swb_suspension_def* suspension;              /* nullable */
} swb_structure_definition;

/* StructureStepSettings (structure.h:208-219) */
typedef struct swb_step_settings {
    double time_step;
    int32_t substeps;
    int32_t constraint_iterations;
    int32_t cable_sweep_pairs;
    uint32_t worker_threads; /* accepted for source compatibility; ignored */
    swb_vec3 gravity;
    double velocity_damping;
    swb_vec3 damping_reference_velocity;
} swb_step_settings;

/* StructureStepSettings defaults: dt 1/120, 2 substeps, 12 iterations,
 * gravity -9.80665 z, damping 0.25 (structure.h:208-219). */
void swb_default_step_settings(swb_step_settings* out);

/* StructureDiagnostics (structure.h:221-246) */
typedef struct swb_diagnostics {
    uint64_t node_count;
    uint64_t dynamic_node_count;
    uint64_t triangle_count;
    uint64_t constraint_count;
    uint64_t membrane_count;
    uint64_t dihedral_count;
    uint64_t contact_pair_count;
    uint64_t active_contact_count;
    uint64_t suspension_segment_count;
    double total_dynamic_mass;
    swb_vec3 center_of_mass;
    swb_vec3 linear_momentum;
    double kinetic_energy;
    double maximum_distance_error;
    double maximum_cable_extension;
    double maximum_absolute_membrane_strain;
    double maximum_membrane_residual;
    double maximum_contact_penetration;
    double maximum_suspension_residual;
    swb_vec3 pending_external_force;
    swb_vec3 last_applied_external_force;
    uint32_t finite;
    uint32_t reserved;
} swb_diagnostics;

/* StructureNodeState (structure.h:174-180) */
typedef struct swb_node_state {
    swb_vec3 position;
    swb_vec3 previous_position;
    swb_vec3 velocity;
} swb_node_state;

/* StructureRigidPayloadState (structure.h:182-189) */
typedef struct swb_payload_state {
    swb_vec3 center_of_mass;
    swb_quat body_to_world;
    swb_vec3 linear_velocity;
    swb_vec3 angular_velocity;
} swb_payload_state;

/* StructureSuspensionSegmentState (structure.h:191-198) plus the segment's
 * line wrench contribution on the payload (suspension.cpp:2582-2589). */
typedef struct swb_segment_state {
    uint64_t stable_id;
    double current_length;
    double commanded_rest_length;
    double tension;
} swb_segment_state;

/* Payload line wrench of the last accepted substep: the force and moment the
 * risers exert on the rigid pilot (SuspensionPayloadDiagnostics::lineWrench,
 * suspension.cpp:2582-2589). */
typedef struct swb_wrench {
    swb_vec3 force;
    swb_vec3 moment;
} swb_wrench;

/* ------------------------------------------------------------------------ */
/* Solver options (no reference counterpart: launch shape of the persistent  */
/* kernel; zero fields mean "choose automatically").                         */
/* ------------------------------------------------------------------------ */
/* Two device schedules exist.  The cluster schedule (default when the mesh
 * fits: at most 16 x 4096 nodes and the shared-memory budget) keeps every
 * node in the distributed shared memory of one thread-block cluster and
 * separates colour stages with cluster barriers.  The grid schedule spreads
 * patches over a persistent cooperative grid with device-wide barriers and
 * serves meshes that do not fit one cluster. */
typedef struct swb_solver_options {
    int32_t device;          /* CUDA device ordinal                          */
    int32_t blocks;          /* grid schedule: persistent CTAs; 0 = SMs      */
    int32_t block_threads;   /* threads per CTA; 0 = chosen from the mesh    */
    int32_t partition_levels;/* grid schedule: patch levels; 0 = 3           */
    int32_t cluster_ctas;    /* cluster schedule: CTAs per cluster (1..16);
                                0 = smallest power of two that fits          */
    uint32_t flags;          /* SWB_OPT_* bits                               */
    int64_t sync_budget_cycles; /* bounded barrier spin; 0 = default (~2 s)  */
} swb_solver_options;

enum {
    SWB_OPT_GLOBAL_ONLY = 1u << 0, /* grid schedule without shared-memory
                                      patches: every colour is a device-wide
                                      phase (comparison/debug)               */
    SWB_OPT_NO_GRAPH = 1u << 1,    /* batched: launch without CUDA graphs    */
    SWB_OPT_GRID = 1u << 2,        /* force the grid schedule                */
    SWB_OPT_SPLIT_STAGES = 1u << 3, /* cluster schedule with split stages:
                                      stages of records that touch only the
                                      executing CTA's patch behind CTA
                                      barriers, cluster barriers after the
                                      stages of records that span CTAs       */
    SWB_OPT_AUTOTUNE = 1u << 4,    /* swb_structure_create builds the cluster
                                      schedule for several block sizes (the
                                      widest stage, 512, 768 threads), with
                                      and without split stages and on the
                                      smallest and the next wider cluster
                                      that fit, times trial substeps of each
                                      (which leave the state untouched) and
                                      keeps the fastest; the other options
                                      fields fix what they set.  Ignored for
                                      fabric self-contact (the widest cluster
                                      and 768 threads) and with SWB_OPT_GRID.
                                      swb_structure_autotune_report lists
                                      the candidates.                         */
    SWB_OPT_CONTACT_ONE_CLUSTER = 1u << 5 /* fabric self-contact: run the
                                      detection phases (broadphase, swept
                                      queries) on the structure's cluster
                                      alone; by default, on surfaces of
                                      16,384 vertices and edges or more,
                                      clusters beside it join them (a
                                      cooperative launch), with results bit
                                      for bit the same                       */
};

void swb_default_solver_options(swb_solver_options* out);

/* ------------------------------------------------------------------------ */
/* Single structure (replaces simwing::fsi::Structure).                      */
/* ------------------------------------------------------------------------ */
typedef struct swb_structure swb_structure;

/* Structure::Structure(StructureDefinition) (structure.h:275,
 * structure.cpp:687-690): validates, builds the device image.  The
 * definition is copied; the caller's arrays may be freed afterwards. */
swb_status swb_structure_create(const swb_structure_definition* definition,
                                const swb_solver_options* options,
                                swb_structure** out);
void swb_structure_destroy(swb_structure* structure);

/* Structure::definitionFingerprint / acceptedStepCount /
 * simulationTimeSeconds (structure.h:283-287). */
uint64_t swb_structure_fingerprint(const swb_structure* structure);
uint64_t swb_structure_accepted_steps(const swb_structure* structure);
double swb_structure_simulation_time(const swb_structure* structure);
uint64_t swb_structure_node_count(const swb_structure* structure);

/* Structure::clearExternalForces / addExternalForce / setExternalForces
 * (structure.h:291-295, structure.cpp:778-805). */
swb_status swb_structure_clear_external_forces(swb_structure* structure);
swb_status swb_structure_add_external_force(swb_structure* structure,
                                            uint64_t node,
                                            const swb_vec3* force);
swb_status swb_structure_set_external_forces(swb_structure* structure,
                                             const swb_vec3* forces,
                                             uint64_t count);

/* SoftBody::setFacePressureDifference / setUniformPressureDifference
 * (soft_body.h:425-433): per-face pressure jump used by the device pressure
 * gather (soft_body.cpp:1492-1534). */
swb_status swb_structure_set_face_pressure(swb_structure* structure,
                                           uint64_t triangle,
                                           double pressure_difference);
swb_status swb_structure_set_uniform_pressure(swb_structure* structure,
                                              double pressure_difference);

/* Structure::step (structure.h:297-300, structure.cpp:807-831).  Consumes the
 * pending external forces only when the step is accepted; on failure the
 * pre-step state is restored and the status says why.  `out` is nullable. */
swb_status swb_structure_step(swb_structure* structure,
                              const swb_step_settings* settings,
                              swb_diagnostics* out);

/* Runs `steps` accepted steps back to back with the same settings and the
 * same pending loads re-applied each step (the loads are consumed after the
 * last).  Diagnostics are those of the final step.  No reference
 * counterpart: a caller loop over Structure::step with constant loads. */
swb_status swb_structure_step_many(swb_structure* structure,
                                   const swb_step_settings* settings,
                                   int32_t steps,
                                   swb_diagnostics* out);

/* Structure::diagnostics (structure.h:301, structure.cpp:833-959), reduced
 * on the device. */
swb_status swb_structure_diagnostics(const swb_structure* structure,
                                     swb_diagnostics* out);

/* Diagnostics of caller-owned device arrays that allocates no device memory.
 * No counterpart in the reference: it is for callers that cannot call
 * cudaMalloc (a coupled flow solver that reserves the GPU's memory in its own
 * pool and keeps the structural state there; fixed-budget loops that must
 * not let an allocation synchronize the device).  It computes the node and
 * distance-constraint reductions of Structure::diagnostics
 * (structure.cpp:833-959) over:
 *   positions, previous_positions, velocities: device float4[node_count],
 *       xyz in metres (w of positions = inverse mass, 0 = fixed);
 *   first_nodes, second_nodes: device uint32[constraint_count];
 *   rest_lengths: device float[constraint_count];
 *   kinds: device uint8[constraint_count] (SWB_CONSTRAINT_*).
 * Filled: node_count, dynamic_node_count, constraint_count,
 * total_dynamic_mass, center_of_mass, linear_momentum, kinetic_energy,
 * maximum_distance_error, maximum_cable_extension, finite; the rest is 0.
 * Scratch is one fixed static device array shared by every call: at most
 * SWB_NOALLOC_MAX_NODES nodes and SWB_NOALLOC_MAX_CONSTRAINTS constraints,
 * larger inputs are rejected with SWB_INVALID_ARGUMENT.  Calls whose work
 * overlaps on the GPU would race on that array; the function serialises its
 * own calls per device and returns only when its result is on the host.  It
 * runs on the legacy default stream, after the caller's work on blocking
 * streams. */
#define SWB_NOALLOC_MAX_NODES 524288u
#define SWB_NOALLOC_MAX_CONSTRAINTS 524288u
swb_status swb_diagnostics_noalloc(int32_t device,
                                   const void* positions,
                                   const void* previous_positions,
                                   const void* velocities,
                                   uint64_t node_count,
                                   const uint32_t* first_nodes,
                                   const uint32_t* second_nodes,
                                   const float* rest_lengths,
                                   const uint8_t* kinds,
                                   uint64_t constraint_count,
                                   swb_diagnostics* out);

/* A ground plane under the structure (no counterpart in the reference's
 * structural step, which has none: its only plane is the payload's support
 * plane, which the adapter leaves free).  After every constraint iteration
 * each free node is projected back onto the side normal . x >= offset
 * (world coordinates, metres; `normal` of unit length), rigidly; with
 * friction > 0 its motion over the substep along the plane is then
 * resisted by Coulomb friction: stopped while it stays below friction x
 * the depth of the normal correction, else shortened by that length.
 * enabled = 0 (or a null pointer) removes the plane.  Differentiable
 * rollouts take the frictionless plane. */
typedef struct swb_ground {
    swb_vec3 normal;
    double offset;
    double friction;
    uint32_t enabled;
    uint32_t reserved;
} swb_ground;
swb_status swb_structure_set_ground(swb_structure* structure, const swb_ground* ground);

/* Line-line contact (no counterpart in the reference, which rejects segment
 * contact: contact.cpp:2336-2339): the suspension lines' cable segments are
 * kept 2 x radius apart.  Once per substep, at the predicted positions, the
 * pairs of segments that share no node and come within 2 x radius + margin
 * of each other (by their boxes) become candidates; after every constraint
 * iteration the candidates are projected in key order (by segment, the
 * segments ordered by their smaller, then larger definition node index):
 * the closest points of the two segments pushed apart to 2 x radius,
 * rigidly.  enabled = 0 (or a null pointer) removes it.  Single structures
 * and their differentiable rollouts (which tape up to 4,096 candidates per
 * step and fail the backward with SWB_CONTACT_ERROR beyond that); batches
 * refuse it. */
typedef struct swb_line_contact {
    double radius;
    double margin;
    uint32_t enabled;
    uint32_t reserved;
} swb_line_contact;
swb_status swb_structure_set_line_contact(swb_structure* structure, const swb_line_contact* contact);

/* The device forms of the step's two short math functions on host arrays
 * (no counterpart in the reference; for checking them on the GPU they run
 * on): which = SWB_FAST_ATAN2 gives out[i] = atan2(a[i], b[i]) by the
 * device's polynomial form, SWB_FAST_RCP gives out[i] = 1 / a[i] by the
 * approximate reciprocal.  count may be 0. */
#define SWB_FAST_ATAN2 0u
#define SWB_FAST_RCP 1u
swb_status swb_fast_math_eval(uint32_t which, const float* a, const float* b, float* out, uint64_t count);

/* Structure::nodeStates (structure.h:288, structure.cpp:725-734). */
swb_status swb_structure_read_nodes(const swb_structure* structure,
                                    swb_node_state* out,
                                    uint64_t count);
/* Positions only, FP32 xyz triples (3*count floats). */
swb_status swb_structure_read_positions_f32(const swb_structure* structure,
                                            float* out_xyz,
                                            uint64_t count);
/* Overwrites node positions and velocities (previous positions are set to
 * the positions).  No reference counterpart; used to start the device solver
 * from a state produced elsewhere, e.g. another solver's checkpoint. */
swb_status swb_structure_write_nodes(swb_structure* structure,
                                     const swb_node_state* nodes,
                                     uint64_t count);

/* Structure::suspensionState (structure.h:289-290, structure.cpp:736-776).
 * segments may be NULL when segment_capacity is 0. */
swb_status swb_structure_read_suspension(const swb_structure* structure,
                                         swb_payload_state* payload,
                                         swb_segment_state* segments,
                                         uint64_t segment_capacity,
                                         swb_wrench* line_wrench);
swb_status swb_structure_write_payload(swb_structure* structure,
                                       const swb_payload_state* payload);

/* Structure::checkpoint / restore (structure.h:303-304,
 * structure.cpp:961-1027).  The checkpoint is an opaque, checksummed byte
 * image bound to the definition fingerprint; restore rejects a foreign or
 * tampered image with SWB_INVALID_ARGUMENT. */
swb_status swb_structure_checkpoint_size(const swb_structure* structure,
                                         uint64_t* bytes);
swb_status swb_structure_checkpoint(const swb_structure* structure,
                                    void* buffer,
                                    uint64_t bytes);
swb_status swb_structure_restore(swb_structure* structure,
                                 const void* buffer,
                                 uint64_t bytes);

/* Schedule introspection (no reference counterpart).  The device sweeps
 * distance-like constraints and dihedrals in a fixed order; running the
 * reference's serial solver with its constraint lists permuted into this
 * order reproduces the device sweep exactly.  `order` receives a
 * permutation of [0, count): order[k] is the definition index of the k-th
 * constraint swept. */
swb_status swb_structure_sweep_order(const swb_structure* structure,
                                     uint32_t which, /* SWB_SWEEP_* */
                                     uint64_t* order,
                                     uint64_t count);
enum {
    SWB_SWEEP_DISTANCE = 0,
    SWB_SWEEP_DIHEDRAL = 1,
    SWB_SWEEP_MEMBRANE = 2
};

/* Shape of the device schedule for reporting. */
typedef struct swb_schedule_report {
    int32_t blocks;
    int32_t block_threads;
    int32_t partition_levels;
    int32_t device_phases_per_iteration; /* device-wide barriers / iteration */
    int32_t local_stages_per_iteration;  /* CTA-local colour stages          */
    int32_t global_colours_per_iteration;
    int32_t max_patch_nodes;
    int32_t shared_bytes;
    uint64_t level_constraints[4];       /* distance+dihedral per level      */
    uint64_t global_constraints;
    int32_t cluster_ctas;                /* 0 = grid schedule                */
    int32_t cluster_barriers_per_iteration;
} swb_schedule_report;
/* The autotuner's candidates (SWB_OPT_AUTOTUNE) and its choice; zero
 * candidates when the structure was not tuned.  No reference counterpart. */
#define SWB_AUTOTUNE_MAX_CANDIDATES 16
typedef struct swb_autotune_candidate {
    int32_t cluster_ctas;
    int32_t block_threads;
    uint32_t split_stages;          /* 1: SWB_OPT_SPLIT_STAGES               */
    int32_t stages_per_iteration;
    double ms_per_substep;          /* trial substep, device time            */
} swb_autotune_candidate;
typedef struct swb_autotune_report {
    uint32_t candidates;
    uint32_t chosen;                /* index of the kept candidate            */
    uint32_t iterations;            /* constraint iterations of the trials    */
    uint32_t reserved;
    swb_autotune_candidate entries[SWB_AUTOTUNE_MAX_CANDIDATES];
} swb_autotune_report;
swb_status swb_structure_autotune_report(const swb_structure* structure, swb_autotune_report* out);

swb_status swb_structure_schedule_report(const swb_structure* structure,
                                         swb_schedule_report* out);

/* Builds the same schedule on the host alone (no device needed), checks
 * every invariant the device relies on (disjoint patches, node-disjoint
 * stages, each constraint exactly once, complete patch interfaces) and
 * fills the report and, when non-NULL, the sweep orders (constraint_count
 * and dihedral_count entries).  block_threads and shared_bytes are left 0.
 * No reference counterpart. */
swb_status swb_plan_schedule(const swb_structure_definition* definition,
                             const swb_solver_options* options,
                             swb_schedule_report* out,
                             uint64_t* distance_order,
                             uint64_t* dihedral_order);
/* The membrane sweep order of the same host-built schedule (membrane_count
 * entries).  No reference counterpart. */
swb_status swb_plan_membrane_order(const swb_structure_definition* definition,
                                   const swb_solver_options* options,
                                   uint64_t* membrane_order);

/* Device time of the most recent step's kernels in milliseconds, measured
 * with CUDA events on the solver's stream. */
double swb_structure_last_step_ms(const swb_structure* structure);

/* ------------------------------------------------------------------------ */
/* Batched structures.  No reference counterpart: the reference steps one    */
/* Structure per call, and a caller with many wings loops over them.  A      */
/* batch holds many independent structures of uneven sizes and steps all of  */
/* them with one kernel launch per substep: each structure occupies a        */
/* contiguous range of ranks of a thread-block cluster (several small        */
/* structures share one cluster), and the launches of a block of steps are   */
/* captured in one CUDA graph.  Each structure steps exactly as a plain      */
/* structure created with cluster_ctas = its rank count (bit-identical).     */
/* ------------------------------------------------------------------------ */
typedef struct swb_batch swb_batch;

typedef struct swb_batch_options {
    int32_t device;
    int32_t cluster_ctas;        /* CTAs per cluster, 1..16; 0 = 16            */
    int32_t target_patch_nodes;  /* nodes per CTA each structure is split for;
                                    0 = autotune when SWB_BATCH_AUTOTUNE is
                                    set, else 2048                           */
    int32_t block_threads;       /* 0 = widest stage of any structure        */
    int32_t graph_steps;         /* steps per captured graph; 0 = 120        */
    uint32_t flags;              /* SWB_OPT_NO_GRAPH | SWB_BATCH_AUTOTUNE    */
    int32_t autotune_iterations; /* iterations of the timed trial steps; 0 = 48 */
    int32_t reserved;
} swb_batch_options;

enum {
    SWB_BATCH_AUTOTUNE = 1u << 8  /* time candidate patch sizes at creation */
};

void swb_default_batch_options(swb_batch_options* out);

/* Builds every structure (validation as swb_structure_create), splits each
 * into ranks, packs the ranks into clusters and, with SWB_BATCH_AUTOTUNE,
 * keeps the patch size whose trial launches were fastest. */
swb_status swb_batch_create(const swb_structure_definition* const* definitions,
                            uint64_t count,
                            const swb_batch_options* options,
                            swb_batch** out);
void swb_batch_destroy(swb_batch* batch);
uint64_t swb_batch_size(const swb_batch* batch);

/* Borrowed handle of structure `index` (valid until swb_batch_destroy; do
 * not destroy it).  Every swb_structure_* call works on it: loads, pressure,
 * read_nodes, diagnostics, checkpoint/restore, even a single plain step. */
swb_structure* swb_batch_structure(swb_batch* batch, uint64_t index);

/* Steps every structure `steps` times with the same settings and its own
 * pending loads re-applied each step.  Per structure the steps form
 * transactions of up to graph_steps steps: a structure whose block failed
 * keeps its state and loads from before that block and stops; the others
 * commit.  `statuses` (nullable, `count` entries) receives each structure's
 * status; the return value is SWB_OK or the first failure. */
swb_status swb_batch_step(swb_batch* batch,
                          const swb_step_settings* settings,
                          int32_t steps,
                          int32_t* statuses);

/* The ground plane of swb_structure_set_ground for every structure of the
 * batch (one plane for the whole launch); a null pointer or enabled = 0
 * removes it. */
swb_status swb_batch_set_ground(swb_batch* batch, const swb_ground* ground);

typedef struct swb_batch_report {
    int32_t structures;
    int32_t clusters;
    int32_t cluster_ctas;
    int32_t idle_ctas;           /* ranks of clusters no structure uses      */
    int32_t block_threads;
    int32_t target_patch_nodes;
    int32_t shared_bytes;
    int32_t max_cluster_stages;  /* colour stages per iteration, worst cluster */
    int32_t resident_clusters;   /* clusters the device holds at once        */
    int32_t colours_per_sync;    /* colour stages between cluster barriers   */
    int32_t autotune_candidates; /* patch size x block size pairs timed at
                                    creation                                 */
    int32_t reserved;
    int32_t candidate_patch_nodes[8];
    double candidate_ms_per_step[8];
    int32_t candidate_block_threads[8]; /* 0: enough for the widest stage    */
} swb_batch_report;
swb_status swb_batch_get_report(const swb_batch* batch, swb_batch_report* out);

/* Device time of the most recent swb_batch_step, in milliseconds (CUDA
 * events on the batch's stream around its graphs or launches). */
double swb_batch_last_step_ms(const swb_batch* batch);

/* ------------------------------------------------------------------------ */
/* Differentiable rollouts (adjoint).  No reference counterpart: the        */
/* reference has no adjoint.  An autograd-style pair: forward runs `steps`  */
/* steps of the structure from its committed state (left unchanged) with a */
/* checkpoint every `checkpoint_interval` steps and returns the loss        */
/*   L = sum_i w_i |x_i(T) - target_i|^2 / sum_i w_i   (world positions);   */
/* backward returns dL/d(parameter) for every constraint's rest length and  */
/* compliance, every dihedral's compliance, every suspension segment's rest */
/* length and the pilot mass, by a reverse sweep of the discrete step       */
/* (segments recomputed from their checkpoint with a tape).  One substep    */
/* per step; the structure must run on the cluster schedule.  The external */
/* loads and face pressures pending on the structure stay constant.         */
/* ------------------------------------------------------------------------ */
typedef struct swb_rollout swb_rollout;

/* Output arrays of a backward pass; each is nullable.  Arrays are in
 * definition order: d_rest / d_compliance have constraint_count entries
 * (compliance adjoints are with respect to the magnitude of the
 * compliance), d_dihedral_compliance dihedral_count, d_segment_rest
 * segment_count; d_pilot_mass is a single value (0 without a pilot). */
typedef struct swb_rollout_gradient {
    double* d_rest;
    double* d_compliance;
    double* d_dihedral_compliance;
    double* d_segment_rest;
    double* d_pilot_mass;
} swb_rollout_gradient;

swb_status swb_rollout_create(swb_structure* structure,
                              int32_t steps,
                              int32_t checkpoint_interval, /* 0 = 16 */
                              swb_rollout** out);
void swb_rollout_destroy(swb_rollout* rollout);

/* target_xyz: node_count x 3 world positions; weights: node_count, >= 0. */
swb_status swb_rollout_forward(swb_rollout* rollout,
                               const swb_step_settings* settings,
                               const double* target_xyz,
                               const double* weights,
                               double* loss);
/* The gradient of the last forward's loss.  SWB_NON_FINITE when an entry
 * is not finite (the arrays are written all the same): the reverse sweep
 * runs in FP32, and a rollout whose sensitivity to its parameters grows
 * past FP32's range over its length (an unstable flutter of the fabric
 * amplifies the adjoint step by step) overflows; shorter rollouts stay
 * finite. */
swb_status swb_rollout_backward(swb_rollout* rollout,
                                const swb_rollout_gradient* gradient);
/* The forward of `count` rollouts at once (targets_xyz[k], weights[k] and
 * losses[k] as for swb_rollout_forward): every rollout's launches are
 * enqueued first, each on its structure's own stream, so that the
 * structures run side by side on the device, and then each is waited for.
 * `statuses` (nullable, `count` entries) receives each rollout's status;
 * the return value is SWB_OK or the first failure. */
swb_status swb_rollout_forward_many(swb_rollout* const* rollouts,
                                    uint64_t count,
                                    const swb_step_settings* settings,
                                    const double* const* targets_xyz,
                                    const double* const* weights,
                                    double* losses,
                                    int32_t* statuses);
/* The backward of `count` rollouts at once, as swb_rollout_forward_many
 * runs their forwards; gradients[k] (or none with a null array) receives
 * rollout k's gradient. */
swb_status swb_rollout_backward_many(swb_rollout* const* rollouts,
                                     uint64_t count,
                                     const swb_rollout_gradient* gradients,
                                     int32_t* statuses);
/* World positions at the end of the last forward (node_count x 3). */
swb_status swb_rollout_final_positions(const swb_rollout* rollout,
                                       double* xyz,
                                       uint64_t count);
/* Device time of the last forward / backward in milliseconds. */
double swb_rollout_forward_ms(const swb_rollout* rollout);
double swb_rollout_backward_ms(const swb_rollout* rollout);

/* ------------------------------------------------------------------------ */
/* Reference colouring (bit-exact restatement of                             */
/* SoftBody::constraintColouring, soft_body.cpp:1978-2075): greedy first-fit */
/* over the line graph in insertion order, colours ranked by descending      */
/* size.  order has constraint_count entries, offsets colour_count + 1.      */
/* ------------------------------------------------------------------------ */
swb_status swb_reference_colouring(const swb_structure_definition* definition,
                                   uint64_t* order,
                                   uint64_t* offsets,
                                   uint64_t offsets_capacity,
                                   uint64_t* colour_count,
                                   uint64_t* parallel_colours);

/* ------------------------------------------------------------------------ */
/* Synthetic definitions.  Deterministic generators of the cloth patch and   */
/* the ram-air wing; they emit a definition the way the reference's scene    */
/* assembly would (area/3 mass lumping, one dihedral per interior sheet edge */
/* with the series-strip compliance, seam stitches + rails, cable lines, a   */
/* rigid pilot on two risers) -- src/fsi/scene_structure.cpp:278-892.        */
/* ------------------------------------------------------------------------ */
typedef struct swb_definition swb_definition;

typedef struct swb_patch_params {
    uint32_t nx, ny;          /* particles per side (33 x 33)             */
    double width, height;     /* metres (1 x 1)                           */
    double areal_density;     /* kg/m^2 (0.040)                           */
    double distance_compliance; /* m/N (1e-7)                             */
    double bend_compliance;   /* rad/(N m) (1e-3)                         */
    double jitter;            /* std-dev metres of N(0, jitter) (1e-3)    */
    uint64_t seed;
    uint32_t pin_top_corners; /* 1 = two top corners fixed                */
    uint32_t membranes;       /* 0 = none; 1 = one membrane element per
                                 triangle (chart = the unjittered sheet
                                 coordinates), linear orthotropic
                                 material; 2 = the same with pre-tension,
                                 damping and compression softening        */
} swb_patch_params;

typedef struct swb_wing_params {
    uint32_t cells;           /* 40                                        */
    uint32_t chordwise;       /* quads chordwise per surface (60)          */
    uint32_t spanwise_per_cell; /* quads spanwise per cell (4)             */
    uint32_t rib_layers;      /* quads through the rib thickness (6)       */
    double span;              /* metres (11)                               */
    double root_chord;        /* metres (2.6)                              */
    double thickness;         /* fraction of chord (0.15)                  */
    double areal_density;     /* kg/m^2 (0.045)                            */
    double skin_compliance;   /* m/N for skin/rib edges                    */
    double bend_rigidity;     /* N m bending rigidity of the fabric        */
    double line_compliance_scale; /* multiplies L/EA of every line         */
    double pressure;          /* Pa, outward (30)                          */
    uint32_t line_levels;     /* cascade levels (4)                        */
    uint32_t line_particles;  /* particles per line segment (8)            */
    uint32_t line_rows;       /* A/B/C/brake = 4                           */
    uint32_t pilot;           /* 1 = rigid pilot on two risers             */
    double pilot_mass;        /* kg (90)                                   */
    double aspect_ratio;      /* 0 = derive from span and chord            */
    double compliance_jitter; /* sigma of lognormal compliance multiplier  */
    uint64_t seed;
    uint32_t fabric;          /* 0 = one distance constraint per skin and
                                 rib edge; 1 = one orthotropic membrane
                                 element per skin and rib triangle and no
                                 fabric edge constraints, as the reference's
                                 scene assembly builds the canopy
                                 (scene_structure.cpp:1125-1151)           */
    uint32_t attachments_per_cell; /* line attachment stations per cell on
                                 each row (0 or 1 = one per rib; must
                                 divide spanwise_per_cell)                 */
} swb_wing_params;

void swb_default_patch_params(swb_patch_params* out);
void swb_default_wing_params(swb_wing_params* out);
swb_status swb_generate_patch(const swb_patch_params* params,
                              swb_definition** out);
swb_status swb_generate_wing(const swb_wing_params* params,
                             swb_definition** out);
/* ------------------------------------------------------------------------ */
/* Scene assembly: simwing::fsi::assembleSceneStructure                     */
/* (src/fsi/scene_structure.h:127-196, scene_structure.cpp:278-1284) --     */
/* authored scene-v2 geometry (src/fsi/scene.h:77-233) to a definition:     */
/* fabric mass lumped from each triangle's material-chart area, one Bulk    */
/* membrane per triangle, one dihedral per consistently oriented manifold   */
/* edge of one sheet with compliance h0/(2 D0 L0) + h1/(2 D1 L1), seams as  */
/* zero-rest stitches plus half-rigidity rails, and the suspension as       */
/* nodal cables or, with one rigid pilot, a tree oriented from the canopy   */
/* leaves to the harness roots.  Entities are taken in stable-ID order, so  */
/* the input order does not matter.  Stable IDs are non-zero.               */
/* ------------------------------------------------------------------------ */
typedef struct swb_scene_vertex {        /* Vertex                        */
    uint64_t id;
    swb_vec3 position;                   /* m                             */
} swb_scene_vertex;

typedef struct swb_scene_fabric {        /* FabricMaterial                */
    uint64_t id;
    double warp_stiffness, weft_stiffness, shear_stiffness; /* N/m       */
    double bending_stiffness;            /* N m (0: no hinge)             */
    double areal_density;                /* kg/m^2                        */
    double damping_seconds;
    double porosity;                     /* fraction in [0, 1]            */
    double permeability;                 /* m^2                           */
} swb_scene_fabric;

typedef struct swb_scene_triangle {      /* Triangle                      */
    uint64_t id;
    uint64_t vertex_ids[3];
    double chart[3][2];                  /* material coordinates, m       */
    uint64_t material_id;
    uint64_t sheet_id;                   /* hinges only within one sheet   */
} swb_scene_triangle;

typedef struct swb_scene_seam_material { /* SeamMaterial                  */
    uint64_t id;
    double linear_density;               /* kg/m                          */
    double axial_stiffness;              /* N                             */
} swb_scene_seam_material;

typedef struct swb_scene_seam {          /* Seam: two chains of `count`
                                            vertex IDs in seam_vertex_ids */
    uint64_t id;
    uint64_t material_id;
    uint64_t first_begin, second_begin, count;
} swb_scene_seam;

typedef struct swb_scene_line_material { /* LineMaterial                  */
    uint64_t id;
    double diameter, linear_density, axial_stiffness, drag_coefficient;
} swb_scene_line_material;

typedef struct swb_scene_pilot {         /* Pilot                         */
    uint64_t id;
    double mass;
    swb_vec3 center_of_mass, linear_velocity;
    swb_quat body_to_world;
    swb_vec3 principal_inertia;
} swb_scene_pilot;

typedef struct swb_scene_junction {      /* SuspensionJunction            */
    uint64_t id;
    swb_vec3 position;
    double mass;
    uint32_t fixed;
    uint32_t reserved;
} swb_scene_junction;

#define SWB_ATTACH_SURFACE_VERTEX 1u
#define SWB_ATTACH_PILOT_HARNESS 2u
#define SWB_ATTACH_JUNCTION 3u
typedef struct swb_scene_attachment {    /* Attachment: one target by kind */
    uint64_t id;
    uint32_t kind;                       /* SWB_ATTACH_*                  */
    uint32_t reserved;
    uint64_t vertex_id, pilot_id, junction_id;
    swb_vec3 pilot_local_position;
} swb_scene_attachment;

typedef struct swb_scene_line {          /* SuspensionLine                */
    uint64_t id;
    uint64_t start_attachment_id, end_attachment_id, material_id;
    double rest_length;
    uint32_t role;                       /* 1 suspension, 2 riser, 3 brake,
                                            4 harness                     */
    uint32_t reserved;
} swb_scene_line;

typedef struct swb_scene {
    uint64_t vertex_count;          const swb_scene_vertex* vertices;
    uint64_t fabric_count;          const swb_scene_fabric* fabrics;
    uint64_t triangle_count;        const swb_scene_triangle* triangles;
    uint64_t seam_material_count;   const swb_scene_seam_material* seam_materials;
    uint64_t seam_count;            const swb_scene_seam* seams;
    uint64_t seam_vertex_id_count;  const uint64_t* seam_vertex_ids;
    uint64_t line_material_count;   const swb_scene_line_material* line_materials;
    uint64_t pilot_count;           const swb_scene_pilot* pilots;
    uint64_t junction_count;        const swb_scene_junction* junctions;
    uint64_t attachment_count;      const swb_scene_attachment* attachments;
    uint64_t line_count;            const swb_scene_line* lines;
} swb_scene;

typedef struct swb_scene_settings {      /* SceneStructureSettings        */
    double seam_coincidence_tolerance;   /* 1e-9 m                        */
    int32_t suspension_solver_iterations;/* 12                            */
    uint32_t has_fabric_self_contact;
    double suspension_attachment_tolerance;   /* 1e-10                    */
    double suspension_minimum_line_length;    /* 1e-10 m                  */
    double suspension_maximum_line_residual;  /* 2e-4 m                   */
    double suspension_maximum_control_work;   /* 1e6 J                    */
    swb_fabric_contact_def fabric_self_contact;
} swb_scene_settings;

/* The first diagnostic (in the reference's order: entity kind, stable ID,
 * code, message) and the assembly totals. */
typedef struct swb_scene_report {
    uint32_t assembled;
    uint32_t diagnostic_count;
    uint32_t first_code;           /* SceneStructureDiagnosticCode: 1 invalid
                                      scene, 2 mapping overflow, 3 material
                                      incompatible, 4 degenerate material
                                      coordinates, 5 zero-mass dynamic node,
                                      6 unsupported pilot, 7 unsupported pilot
                                      harness, 8 unsupported suspension
                                      topology, 9 unsupported seam,
                                      10 unsupported bending topology      */
    uint32_t first_validation_code;/* scene ValidationCode for code 1, or 0 */
    uint32_t first_entity_kind;    /* EntityKind (scene.h:239-253)         */
    uint32_t reserved;
    uint64_t first_entity_id;
    double total_fabric_mass;      /* kg                                   */
    double total_seam_mass;        /* kg                                   */
    char first_message[160];
} swb_scene_report;

void swb_default_scene_settings(swb_scene_settings* out);
/* Assembles `scene`; on success *out owns the definition (free with
 * swb_definition_destroy).  A scene the reference refuses returns
 * SWB_INVALID_ARGUMENT with *out NULL and the diagnostics in `report`
 * (nullable). */
swb_status swb_assemble_scene(const swb_scene* scene,
                              const swb_scene_settings* settings,
                              swb_definition** out,
                              swb_scene_report* report);

/* Copies an arbitrary definition into an owned one (for permutation). */
swb_status swb_definition_copy(const swb_structure_definition* source,
                               swb_definition** out);
/* Reorders the constraint and dihedral lists (order arrays as returned by
 * swb_structure_sweep_order; NULL keeps a list as is). */
swb_status swb_definition_permute(swb_definition* definition,
                                  const uint64_t* constraint_order,
                                  const uint64_t* dihedral_order);
/* Reorders the membrane list (an order from swb_structure_sweep_order with
 * SWB_SWEEP_MEMBRANE). */
swb_status swb_definition_permute_membranes(swb_definition* definition,
                                            const uint64_t* membrane_order);
/* Sets (or, with NULL, removes) the fabric self-contact of a definition. */
swb_status swb_definition_set_contact(swb_definition* definition,
                                      const swb_fabric_contact_def* contact);
/* Multiplies the rest length of constraint `index` (any kind) or, when
 * index >= constraint_count, of suspension segment index - constraint_count. */
swb_status swb_definition_scale_rest(swb_definition* definition,
                                     uint64_t index,
                                     double factor);
const swb_structure_definition* swb_definition_view(
    const swb_definition* definition);
void swb_definition_destroy(swb_definition* definition);

/* Definition fingerprint of Structure (structure.cpp:463-553 restated:
 * FNV-1a over the definition's fields in declaration order). */
uint64_t swb_definition_fingerprint(const swb_structure_definition* definition);

/* Validation only (structure.cpp:102-455). */
swb_status swb_validate_definition(const swb_structure_definition* definition);

/* ------------------------------------------------------------------------ */
/* Contact building blocks on the device, in FP64 (softwing contact.h).      */
/* The fabric self-contact of a definition (structure.cpp:626-636) is one    */
/* contact surface over all triangles, paired with itself: vertex-triangle   */
/* features of every surface vertex against every triangle not holding it,  */
/* and edge-edge features of every two surface edges that share no node.     */
/* ------------------------------------------------------------------------ */

/* ContactFeatureKind (contact.h:26-30) */
#define SWB_FEATURE_VERTEX_TRIANGLE 0u
#define SWB_FEATURE_EDGE_EDGE 1u
#define SWB_FEATURE_SEGMENT_TRIANGLE 2u

/* GeometryQueryStatus (contact.h:32-37) */
#define SWB_GEOMETRY_CERTIFIED 0u
#define SWB_GEOMETRY_DEGENERATE 1u
#define SWB_GEOMETRY_NON_FINITE 2u
#define SWB_GEOMETRY_UNCERTIFIABLE 3u

/* CcdState (contact.h:153-158) */
#define SWB_CCD_NO_IMPACT 0u
#define SWB_CCD_IMPACT 1u
#define SWB_CCD_INITIALLY_PROXIMATE 2u
#define SWB_CCD_INDETERMINATE 3u

/* ContactFeatureKey (contact.h:95-101); keys order lexicographically by
 * (pair, kind, first[0..2], second[0..2]).  Vertex-triangle: first =
 * {vertex, 0, 0}, second = {triangle, 0, 0}; edge-edge: first and second
 * are the two edges {a, b, 0} (a < b), the lesser edge first. */
typedef struct swb_contact_key {
    uint64_t pair;
    uint32_t kind;
    uint32_t reserved;
    uint64_t first[3];
    uint64_t second[3];
} swb_contact_key;

/* ------------------------------------------------------------------------ */
/* Details of the last failure on this thread, for the callers that read    */
/* them off the reference's exceptions: SuspensionError::phase() and        */
/* entity() (src/softwing/include/softwing/suspension.h:27-53) and          */
/* ContactStepError::key() (src/softwing/include/softwing/contact.h:        */
/* 262-270).                                                                 */
/* ------------------------------------------------------------------------ */
/* softwing::SuspensionPhase, in declaration order. */
#define SWB_PHASE_PARSE 0u
#define SWB_PHASE_VALIDATION 1u
#define SWB_PHASE_ATTACHMENT_RESOLUTION 2u
#define SWB_PHASE_GRAPH_CONSTRUCTION 3u
#define SWB_PHASE_CONTROL 4u
#define SWB_PHASE_PREDICTION 5u
#define SWB_PHASE_LINE_SOLVE 6u
#define SWB_PHASE_GROUND_SOLVE 7u
#define SWB_PHASE_CERTIFICATION 8u
#define SWB_PHASE_DIAGNOSTICS 9u

typedef struct swb_error_detail {
    uint32_t status;              /* status of the failure described        */
    uint32_t suspension_phase;    /* SWB_SUSPENSION_ERROR: SWB_PHASE_*       */
    char suspension_entity[128];  /* SWB_SUSPENSION_ERROR: the entity, e.g.
                                     "segment:<stable id>", "line-residual",
                                     "payload", "payload-step"             */
    uint32_t has_contact_key;     /* SWB_CONTACT_ERROR: 1 when the failure
                                     belongs to a feature; 0 gives the
                                     reference's default-constructed key   */
    uint32_t reserved;
    swb_contact_key contact_key;  /* SWB_CONTACT_ERROR: the failing feature
                                     first in key order (the one the
                                     reference's key-ordered sweep throws
                                     at)                                    */
} swb_error_detail;

/* Copies the details of the last failing call on this thread (zeroed with
 * `status` SWB_OK when the last failure had none to give). */
swb_status swb_last_error_detail(swb_error_detail* out);

/* CcdSettings (contact.h:160-165) */
typedef struct swb_ccd_settings {
    int32_t conservative_iterations;   /* 32                                 */
    int32_t interval_subdivisions;     /* 256; at most SWB_CCD_MAX_SUBDIVISIONS */
    double time_tolerance;             /* 1e-8                               */
    double distance_tolerance;         /* 1e-10                              */
} swb_ccd_settings;

/* The interval fallback keeps its pending intervals in device scratch of
 * interval_subdivisions + 1 entries per query; larger budgets are refused. */
#define SWB_CCD_MAX_SUBDIVISIONS 4096

void swb_default_ccd_settings(swb_ccd_settings* out);

/* ClosestFeatureResult (contact.h:53-68); features are ClosestFeatureClass
 * values (contact.h:39-51: Point 0, SegmentStart 1, SegmentEnd 2,
 * SegmentInterior 3, TriangleVertex0..2 4-6, TriangleEdge01 7,
 * TriangleEdge12 8, TriangleEdge20 9, TriangleFace 10). */
typedef struct swb_closest_result {
    uint32_t status;
    uint32_t first_feature;
    uint32_t second_feature;
    uint32_t reserved;
    double first_point[3];
    double second_point[3];
    double first_weights[3];
    double second_weights[3];
    double normal[3];
    double distance;
    double gap;
} swb_closest_result;

/* CcdResult (contact.h:167-176) */
typedef struct swb_ccd_result {
    uint32_t state;
    int32_t conservative_iterations;
    int32_t interval_subdivisions;
    uint32_t used_interval_fallback;
    double time_of_impact;
    double bracket_lower;
    double bracket_upper;
    swb_closest_result geometry;
} swb_ccd_result;

/* Candidate features of the definition's fabric self-contact pair for the
 * motion previous -> current (node_count x 3 doubles each): the eligible
 * features whose swept, separation-expanded AABBs (sweptExpandedAabb,
 * contact.cpp:488-526, separation = 2 x half_thickness) overlap on all
 * three axes, in key order -- the candidate list of SoftBody's contact
 * iteration (contact.cpp:1057-1290 with sweepAndPruneContactPairs,
 * contact.cpp:528-668).  possible / excluded count the feature pairs before
 * and removed by the topology filter.  When the list exceeds `capacity`
 * only the count is written and the call returns SWB_OUT_OF_RANGE. */
swb_status swb_contact_candidates(const swb_structure_definition* definition,
                                  double half_thickness,
                                  const double* previous,
                                  const double* current,
                                  swb_contact_key* keys,
                                  uint64_t capacity,
                                  uint64_t* candidate_count,
                                  uint64_t* possible_count,
                                  uint64_t* excluded_count);

/* closestVertexTriangle / closestEdgeEdge (contact.cpp:141-305) for `count`
 * features of one kind.  Each feature reads 3 points (9 doubles) from
 * `first` and from `second` (unused points ignored: a vertex is first[0],
 * an edge first[0..1]). */
swb_status swb_contact_closest(uint32_t kind,
                               uint64_t count,
                               const double* first,
                               const double* second,
                               double separation,
                               swb_closest_result* results);

/* sweptContact (contact.cpp:669-945) for `count` features of one kind:
 * linear motion of each primitive from *_previous to *_current (9 doubles
 * per feature and side, as above). */
swb_status swb_contact_sweep(uint32_t kind,
                             uint64_t count,
                             const double* first_previous,
                             const double* first_current,
                             const double* second_previous,
                             const double* second_current,
                             double separation,
                             const swb_ccd_settings* settings,
                             swb_ccd_result* results);

/* ------------------------------------------------------------------------ */
/* Coupling callers with device-resident loads: the structural side of      */
/* simwing::fsi::ConservativeMacroStepCoupling::advanceStructure and        */
/* advanceStructureWithEndpointLoads (src/fsi/coupling.cpp:806-911).  A     */
/* coupling binds interface node i to structure node structure_nodes[i];    */
/* several interface nodes may load one structure node.                     */
/* ------------------------------------------------------------------------ */
typedef struct swb_coupling swb_coupling;

/* SWB_OUT_OF_RANGE when a binding names an unknown structure node. */
swb_status swb_coupling_create(swb_structure* structure,
                               const uint64_t* structure_nodes,
                               uint64_t bindings,
                               swb_coupling** out);
void swb_coupling_destroy(swb_coupling* coupling);

/* One structure step on the time-integrated interface impulses `impulses`
 * (DEVICE memory, bindings x 3 doubles, N s) over `duration` seconds, which
 * must equal settings->time_step: each binding adds impulse / duration to
 * its structure node, in binding order, on top of the loads already
 * pending.  Non-finite loads: SWB_INVALID_ARGUMENT before stepping; a failed
 * step leaves the pending loads as they were (the reference restores its
 * pre-call checkpoint). */
swb_status swb_coupling_advance_impulses(swb_coupling* coupling,
                                         const double* impulses,
                                         double duration,
                                         const swb_step_settings* settings,
                                         swb_diagnostics* out);

/* The same with endpoint tractions (DEVICE memory, bindings x 3 doubles
 * each, N): each binding adds the mean of its start and end load. */
swb_status swb_coupling_advance_endpoint_loads(swb_coupling* coupling,
                                               const double* start_loads,
                                               const double* end_loads,
                                               const swb_step_settings* settings,
                                               swb_diagnostics* out);

/* ------------------------------------------------------------------------ */
/* Closed cell (bay) volumes, the geometric input of the canopy's cell-air   */
/* pressure model: softwing::estimateClosedCellVolume (cell_volume.h:38-44, */
/* cell_volume.cpp:161-306) for many cells at once, on the device in FP64.  */
/* ------------------------------------------------------------------------ */

/* One cell: skin faces face_indices[face_begin, +face_count) and the two rib
 * loops (ordered closed polygons, first node not repeated)
 * loop_nodes[low_begin, +low_count) and loop_nodes[high_begin, +high_count). */
typedef struct swb_cell_def {
    uint64_t face_begin, face_count;
    uint64_t low_begin, low_count;
    uint64_t high_begin, high_count;
} swb_cell_def;

/* ClosedCellVolumeEstimate (cell_volume.h:14-32) */
typedef struct swb_cell_volume {
    double signed_volume;
    double volume;
    uint64_t skin_boundary_edges;
    uint64_t cap_boundary_edges_matched;
    uint64_t non_manifold_skin_edges;
    uint64_t degenerate_skin_faces;
    uint32_t valid;
    uint32_t watertight_after_capping;
    uint32_t used_geometric_orientation_fallback;
    uint32_t ambiguous_skin_orientation;
} swb_cell_volume;

/* Volumes of `cell_count` cells of the definition's triangles at `positions`
 * (node_count x 3 doubles, host); bit for bit the reference's estimates. */
swb_status swb_cell_volumes(const swb_structure_definition* definition,
                            const uint64_t* face_indices,
                            const uint64_t* loop_nodes,
                            const swb_cell_def* cells,
                            uint64_t cell_count,
                            const double* positions,
                            swb_cell_volume* out);

/* Device-resident form for a step loop: the cells' topology is computed and
 * uploaded once, at plan creation (the only allocations); each evaluation
 * then launches one kernel on the caller's stream, allocates nothing and
 * does not synchronise.  The plan lives on `device`. */
typedef struct swb_cell_volume_plan swb_cell_volume_plan;
swb_status swb_cell_volume_plan_create(const swb_structure_definition* definition,
                                       const uint64_t* face_indices,
                                       const uint64_t* loop_nodes,
                                       const swb_cell_def* cells,
                                       uint64_t cell_count,
                                       int device,
                                       swb_cell_volume_plan** out);
void swb_cell_volume_plan_destroy(swb_cell_volume_plan* plan);
/* `positions` (node_count x 3 doubles) and `out` (cell_count entries) in
 * DEVICE memory; `stream` a cudaStream_t (NULL: the legacy stream). */
swb_status swb_cell_volumes_device(const swb_cell_volume_plan* plan,
                                   const double* positions,
                                   swb_cell_volume* out,
                                   void* stream);

/* The same at a structure's committed state, read where it lives (its FP32
 * offsets from the FP64 frame origin, widened to FP64 world positions):
 * `out` in DEVICE memory, on the structure's stream, no host copy.  The
 * plan must come from the structure's definition and device; its first use
 * with a structure uploads that structure's node order once. */
swb_status swb_structure_cell_volumes(const swb_structure* structure,
                                      swb_cell_volume_plan* plan,
                                      swb_cell_volume* out);

/* ---- Pneumatic port mass flows --------------------------------------- */
/* evaluateOrificeMassFlow / evaluateConductanceMassFlow (pneumatics.cpp:   */
/* 132-232, pneumatics.h:46-92): the flow laws that move air between the    */
/* cells, inlets and reservoirs of the cell-air model, evaluated for many   */
/* ports in one launch.                                                     */
#define SWB_PORT_ORIFICE 0u     /* compressible orifice, choked or not     */
#define SWB_PORT_CONDUCTANCE 1u /* linear mass conductance                  */
#define SWB_FLOW_EQUILIBRIUM 0u
#define SWB_FLOW_FIRST_TO_SECOND 1u
#define SWB_FLOW_SECOND_TO_FIRST 2u

typedef struct swb_air_properties {      /* AirProperties                */
    double specific_gas_constant;        /* J/(kg K), 287.05 dry air     */
    double heat_capacity_ratio;          /* gamma, 1.4 dry air           */
} swb_air_properties;

typedef struct swb_flow_zone_state {     /* FlowZoneState                */
    double absolute_pressure;            /* Pa                           */
    double absolute_temperature;         /* K                            */
} swb_flow_zone_state;

typedef struct swb_port_def {
    uint32_t kind;                       /* SWB_PORT_*                   */
    uint32_t reserved;                   /* 0                            */
    uint64_t first, second;              /* zone indices                 */
    double discharge_coefficient;        /* orifice: 0 < Cd <= 1         */
    double effective_area;               /* orifice: m^2                 */
    double mass_conductance;             /* conductance: kg/(s Pa)       */
    double opening_fraction;             /* [0, 1]                       */
} swb_port_def;

typedef struct swb_mass_flow {           /* MassFlowEvaluation           */
    double signed_mass_rate;             /* kg/s, positive first->second */
    double magnitude;
    double pressure_ratio;
    double critical_pressure_ratio;
    uint32_t direction;                  /* SWB_FLOW_*                   */
    uint32_t choked;
} swb_mass_flow;

/* One evaluation per port, from the zones' states (host arrays).  A port
 * the reference would refuse (invalid air, zone state, opening or port
 * constants, a non-finite flow) makes the call return SWB_INVALID_ARGUMENT
 * with the first such port in *failed_port (nullable; port_count when none);
 * `out` is then unspecified.  A zone index past zone_count: SWB_OUT_OF_RANGE. */
swb_status swb_port_mass_flows(const swb_air_properties* air,
                               const swb_flow_zone_state* zones,
                               uint64_t zone_count,
                               const swb_port_def* ports,
                               uint64_t port_count,
                               swb_mass_flow* out,
                               uint64_t* failed_port);

/* The same on DEVICE arrays (zones, ports, out and the one-word
 * `failed_port`), for a network advanced on the device: two kernels on
 * `stream` (a cudaStream_t; NULL: the legacy stream), no allocation, no
 * synchronisation.  Every refusal -- a zone index past zone_count included
 * -- is reported through *failed_port (the first refused port, or
 * port_count when none), which the caller reads when it needs it. */
swb_status swb_port_mass_flows_device(const swb_air_properties* air,
                                      const swb_flow_zone_state* zones,
                                      uint64_t zone_count,
                                      const swb_port_def* ports,
                                      uint64_t port_count,
                                      swb_mass_flow* out,
                                      uint64_t* failed_port,
                                      void* stream);

/* The candidate features of the last step's contact certification
 * (contact.cpp:1583-1798: the final broadphase, in key order), for
 * inspection; valid until the next step.  SWB_OUT_OF_RANGE (count written)
 * when they exceed `capacity`; SWB_UNSUPPORTED without fabric self-contact. */
swb_status swb_structure_contact_candidates(const swb_structure* structure,
                                            swb_contact_key* keys,
                                            uint64_t capacity,
                                            uint64_t* count);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* SIMWING_B200_H */
