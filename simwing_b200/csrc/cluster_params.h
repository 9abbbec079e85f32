// Parameter blocks of the cluster step kernel (host and device).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "simwing_b200.h"
#include "step_params.h"

namespace swb {

namespace dev {
constexpr int kClusterMaxThreads = 768;  // threads per CTA of the cluster step kernels
constexpr int kClusterMaxCtasDev = 16;   // CTAs per cluster at most
}

struct ClusterKindDev {
    const uint32_t* offsets;   // [ctas * (stages + 1)]
    const uint4* rec;          // per record: ab, cd (dihedral), rest bits, compliance bits (sign = cable)
    int stages;
    uint32_t smem_lambda;      // byte offset of this kind's multipliers
    uint64_t sync_mask;        // bit g: a cluster barrier follows stage g (stages >= 64: always)
    int interior_stages;       // stages before this one touch only the CTA's own nodes
    int pad;
    const float4* aux;         // membranes: kMembraneAux float4 of element constants per record
};

// Membrane element constants, per record (float4 each):
//   0: inverse reference (chart) matrix m00 m01 m10 m11
//   1: sqrt(reference area), damping time, compression stiffness ratio, warp pre-tension
//   2: weft pre-tension, compliance xx yy zz
//   3: compliance xy xz yz, stiffness xx
//   4: stiffness yy zz xy, 0
constexpr int kMembraneAux = 5;

// ---- fabric self-contact (single-structure launches) -------------------
// A feature is coded row << 32 | col: row r < nv is surface vertex r
// (vertices in node order) against triangle col; row nv + i is edge i
// (edges in node-pair order) against the later edge col.  Codes order like
// the reference's ContactFeatureKey (contact.h:95-101).

// Per candidate of the current phase, written in parallel: the swept
// query's state and normal, and the closest features of the phase's
// snapshot (contact.cpp:1298-1351).
struct ContactQuery {
    double fw[3], sw[3];     // closest-feature weights, first / second primitive
    double normal[3];        // closest-feature normal (not yet oriented)
    double ccd_normal[3];    // normal of the swept query's geometry
    double eff;              // effective inverse mass sum w_i m_i^-1 w_i
    uint32_t addr[6];        // cluster shared-memory addresses of the nodes: first, then second primitive
    uint32_t slot[6];        // their slots
    float inv[6];            // their inverse masses
    uint32_t ccd_state;      // SWB_CCD_*
    uint32_t certified;      // the snapshot geometry is certified
    uint32_t fc, sc;         // nodes of the first / second primitive
};

// Warm start and record book of one feature over a substep
// (contactMultipliers_ and contactRecords_, contact.cpp:1320-1468).
struct ContactEntry {
    unsigned long long code;
    double lambda;
    double normal[3];        // normal of the record's last solver visit
    uint32_t flags;          // kEntry* bits
    uint32_t pad;
};
enum : uint32_t { kEntryApplied = 1, kEntryRecord = 2, kEntryVisited = 4 };

// A certified record the friction pass consumes (certifyContactState,
// contact.cpp:1583-2080).
struct ContactRecordDev {
    unsigned long long code;
    double fw[3], sw[3];
    double normal[3];
    double lambda;
    double eff;              // effective inverse mass
    uint32_t addr[6];        // node addresses and slots, as in ContactQuery
    uint32_t slot[6];
    float inv[6];
    uint32_t fc, sc;
    uint32_t active;         // normal multiplier > 0 and swept state not NoImpact
    uint32_t pad;
};

struct ContactDiagDev {
    unsigned long long candidates;     // candidates of the final certification
    unsigned long long active;         // active certified records
    unsigned long long records;        // certified + retained records
    double max_penetration;
};

struct ContactDev {
    uint32_t nv, ne, nt, pad;
    const uint32_t* vid;               // [nv] slot of surface vertex r
    const uint2* eid;                  // [ne] slots of edge i
    const uint3* tid;                  // [nt] slots of triangle t
    double separation;                 // 2 x half thickness
    double compliance, static_mu, dynamic_mu;
    swb_ccd_settings ccd;
    // scratch
    float4* snapshot;                  // [slots] positions at the phase start
    double* vbox;                      // [nv][6] swept boxes: lo xyz, hi xyz
    double* ebox;                      // [ne][6]
    double* tbox;                      // [nt][6]
    uint32_t* counts;                  // [nv + ne]
    unsigned long long* offsets;       // [nv + ne + 1]
    unsigned long long* cand;          // [cand_cap] codes of the phase's candidates
    unsigned long long cand_cap;
    ContactQuery* query;               // [cand_cap]
    double* queues;                    // [threads][queue_stride][4] swept-query intervals
    uint32_t queue_stride;
    uint32_t pad2;
    ContactEntry* table[2];            // ping-pong, sorted by code
    uint32_t* table_meta;              // [0] current buffer, [1] entries
    unsigned long long table_cap;
    ContactRecordDev* records;         // [record_cap]
    unsigned long long record_cap;
    // level schedule of a key-ordered pass: an item's level is one more than
    // the last level among the earlier items sharing one of its nodes, so
    // the items of a level share no node and run together
    uint32_t* hit;                     // [cand_cap] the candidates in contact, in key order
    // binned broadphase: the triangles (for vertex rows) and the edges (for
    // edge rows) bucketed by the low end of their boxes along `axis`
    int axis, axis2;                   // the grid's axes: the longest and second-longest extents
    uint32_t bins_cap;                 // grid cells per column set at most
    uint32_t* tbin;                    // [bins_cap + 1] counts, then starts
    uint32_t* tbin_fill;               // [bins_cap + 1]
    uint32_t* tbin_items;              // [nt]
    uint32_t* ebin;                    // [bins_cap + 1]
    uint32_t* ebin_fill;               // [bins_cap + 1]
    uint32_t* ebin_items;              // [ne]
    unsigned long long* range;         // [12] order keys per column set (triangles, then edges): on each
                                       // axis the low ends' minimum and maximum and the largest extent
    uint32_t* cand_tmp;                // [cand_cap] a row's hits before they are ordered
    uint32_t* mark_a;                  // [cand_cap + 1] per-candidate flags, then their exclusive scan
    uint32_t* mark_b;                  // [cand_cap + 1] per-table-entry flags, then their exclusive scan
    ContactEntry* cand_entry;          // [cand_cap] the candidate's table entry after the iteration
    ContactRecordDev* cand_rec;        // [cand_cap] the candidate's certified record
    unsigned long long* reduce;        // [2] active records, largest penetration (bits)
    unsigned long long* fail;          // [1] the failing feature first in key order, packed with its
                                       // detail code (contact_fail_at); all ones when none failed
    // order links of a key-ordered pass (cluster_order, run_order): node
    // buckets of the (node, item) pairs, each item's followers through its
    // nodes, the count of items each one still waits for, and the two
    // rounds' item lists
    uint32_t* lv_node_start;           // [slots + 1] counts, then bucket starts
    uint32_t* lv_node_fill;            // [slots]
    uint32_t* lv_pairs;                // [6 * cand_cap]
    uint32_t* lv_succ;                 // [6 * cand_cap]
    uint32_t* lv_nsucc;                // [cand_cap]
    uint32_t* lv_npred;                // [cand_cap]
    uint32_t* lv_front;                // [2 * cand_cap]
};

// Line-line contact of one structure: the cable segments (node references
// rank << 12 | index of both ends, in key order: by the smaller, then the
// larger node index of the definition) and each step's candidate pairs.
struct LineContactDev {
    uint32_t segments;
    uint32_t capacity;                 // candidate pairs a step may hold
    const uint32_t* seg;               // [segments] ref(a) | ref(b) << 16
    const uint2* seg_nodes;            // [segments] definition node indices (a, b), for the shared-node test
    float radius;                      // line radius: segments are kept 2 radius apart
    float reach;                       // box half-margin of the step's broadphase: radius + margin / 2
    float4* box;                       // [segments][2] the step's predicted boxes (lo, hi)
    uint32_t* pair;                    // [capacity] candidate pairs i << 16 | j, i < j, sorted after the broadphase
    uint32_t* sort;                    // [capacity] scratch of the sort, then each sorted pair's level
    uint32_t* order;                   // [capacity] the pairs by level, key order within a level
    uint32_t* pred;                    // [capacity][4] per node the latest earlier pair with it (~0u: none)
    uint32_t* level_off;               // [capacity + 1] each level's first place in `order`
    uint32_t* count;                   // [2] candidate pairs of the step, their level count
};

// Per-instance tables and state (one cluster each).
struct ClusterInstance {
    const float4* pos_in;
    const float4* vel_in;
    float4* pos_out;
    float4* vel_out;
    float4* prev_out;
    const float4* force;
    const uint32_t* tri_offsets;
    const uint32_t* tri_list;
    const uint4* tri;
    const uint32_t* patch_begin;   // [ctas + 1]
    ClusterKindDev kind[3];        // distance, dihedral, membrane (swept distance, membrane, dihedral)
    float* membrane_residual;      // per membrane record: normalized residual of the last substep
    const uint32_t* seam_offsets;
    const uint32_t* seam_ab;
    int seam_stages;
    int susp_cta;                  // -1 when absent
    const DevPayloadDef* payload_def;
    const DevPayloadState* payload_in;
    DevPayloadState* payload_out;
    const double* origin_in;
    double* origin_out;
    int* status;
    int recentre;
    // First of the two stages beside which the line iteration runs (on the
    // last warp of the suspension CTA, which has no record in either), or -1:
    // the line iteration then follows the iteration's stages behind a
    // cluster barrier.  Single-structure launches only.
    int line_stage;
    // 1: the momentum guard of free structures runs (no suspension, no
    // contact, bending or membranes present, every node free:
    // soft_body.cpp:1192-1202).  Single-structure launches only.
    int momentum_guard;
    // Load-path cable sweeps: levels of one pair (reverse pass, then forward
    // pass), per CTA and level offsets into pair_rec (distance records this
    // CTA runs).  Single-structure launches only.
    int pair_stages;
    const uint32_t* pair_offsets;  // [ctas * (pair_stages + 1)]
    const uint32_t* pair_rec;
    // Fabric self-contact, or nullptr.  Single-structure launches only.
    const ContactDev* contact;
    // Line-line contact (swb_structure_set_line_contact), or nullptr.
    // Single-structure launches only.
    const LineContactDev* lines;
    ContactDiagDev* contact_diag;  // the output state's contact diagnostics
};

// Rigid pilot as the adjoint sees it: the suspension endpoint nodes are
// numbered as attachment slots (distinct nodes, at most 16), each holding a
// local index into the owner CTA's patch.
struct AdjointPilot {
    int slots;
    int slot_node[16];     // local node index in the owner patch
    float slot_w[16];      // inverse mass of the slot's node
    int segments;
    int from_slot[8], to_slot[8], from_point[8], to_point[8];
    float rest[8], stiffness[8], damping[8];
    float3 hang_local[8];
    float3 com_local;
    float3 inertia;
    float mass;
    float min_length;
};

// Inputs of one line iteration, or of the payload finish, as recorded by the
// taping forward step.
struct PilotTape {
    float com[3];
    float q[4];            // w, x, y, z
    float lambda[8];
    float4 xs[16];         // slot positions (xyz)
    float4 vs[16];         // finish only: slot velocities before line damping
};

// Device pointers of one step's tape.  Per iteration, distance-type records
// store two float4 blocks of R0 entries (node a xyz + lambda, node b xyz) and
// dihedral records four blocks of R1 entries (a xyz + lambda, b, c, d); the
// seam pass stores two blocks of its record count.
struct TapeStep {
    float4* dist;
    float4* dih;
    float4* seam;
    PilotTape* line;       // [iterations]
    PilotTape* finish;     // [1]
    uint8_t* ground;       // [iterations][slots]: 1 where the ground projection moved the node
    // line-line contact (null without it): the step's candidates in level
    // order, the level offsets, [count, level count], and each candidate's
    // four end nodes before its projection, [iterations][line_cap][4]
    uint32_t* line_pairs;
    uint32_t* line_level_off;
    uint32_t* line_count;
    float4* line_in;
    uint32_t line_cap;
    uint32_t r0, r1, rs;   // records per kind and seam records
    const AdjointPilot* pilot;
};

// Packed launches (several structures per cluster): what one CTA runs.
// The loop bounds are those of the whole cluster, so that every CTA of the
// cluster takes the same cluster barriers.
struct ClusterSlot {
    int instance;      // index into the launch's structures; -1 = idle CTA
    int rank_base;     // first cluster rank of that structure
    int stages;        // colour stages per iteration: max over the cluster
    int seam_stages;   // seam stages: max over the cluster
    int suspension;    // 1 when a structure of the cluster has a pilot
    int guard;         // 1 when a structure of the cluster runs the momentum guard
    int ctas;          // ranks of this CTA's structure (0 when idle)
    int pad;
};

struct ClusterParams {
    const ClusterInstance* instances;  // one per cluster of the launch; packed: [structure][rotation][role]
    int ctas;                          // CTAs per cluster
    const ClusterSlot* slots;          // packed launches: one per CTA
    const int* rotation;               // packed launches: committed buffer per structure
    int role;                          // packed launches: 0 = S->T1, 1 = T1->T2, 2 = T2->T1
    float dt, inv_dt, inv_dt2, damping;
    float damping_loss;            // 1 - damping from FP64 (see StepParams)
    double dt64;                   // the substep in FP64 (contact phases)
    float3 gravity, ref_velocity;
    int iterations;
    int cable_pairs;               // load-path cable sweep pairs per substep (single-structure launches)
    long long copy_budget;
    uint32_t smem_x, smem_v;       // byte offsets of node and force/velocity arrays
    uint32_t smem_offsets;         // byte offset of the CTA's stage offsets
    TapeStep tape;                 // taping launches: where this step's tape goes
    // contact launches: clusters after the first that join only the contact
    // detection phases (broadphase and swept queries), synchronised with the
    // structure's cluster by the bounded grid barrier `grid` over all CTAs
    // of the (cooperative) launch; 0 = the structure's cluster alone
    int helper_clusters;
    dev::GridBarrier grid;
    // ground plane (swb_structure_set_ground), the same for every structure
    // of the launch: normal . x >= offset in world coordinates; 0 = none
    int ground;
    float ground_friction;
    float3 ground_normal;
    double ground_offset;
};

// Parameters of the reverse step kernel (one structure, one cluster).
struct AdjointParams {
    const ClusterInstance* inst;   // the step's instance record (in = step start, out = step end)
    TapeStep tape;
    const float4* xb_out;          // adjoint of the step's final positions (slot order)
    const float4* vb_out;          // adjoint of the step's final velocities
    float4* xb_in;                 // adjoint of the step-start positions
    float4* vb_in;                 // adjoint of the step-start velocities
    const float* pb_out;           // pilot adjoint: com 3, q 4 (w x y z), v 3, w 3
    float* pb_in;
    float4* fbar;                  // per-slot scratch: adjoint of the nodal force
    double* g_rest0;               // per distance-type record
    double* g_comp0;
    double* g_comp1;               // per dihedral record
    double* g_seg_rest;            // per device suspension segment
    double* g_mass;
    // scratch: Jacobian of each iteration's line iteration, [iterations]
    // blocks of nout x nin floats (output-major), written in the kernel's
    // prologue; nullptr without a pilot
    float* line_jac;
    int ctas;
    float dt, inv_dt, inv_dt2, damping;
    float3 gravity;
    int iterations;
    uint32_t smem_xb, smem_vb, smem_lam0, smem_lam1, smem_acc0r, smem_acc0c, smem_acc1c, smem_offsets;
    int ground;                    // the frictionless ground plane of the forward step (ClusterParams)
    float3 ground_normal;
};

}  // namespace swb
