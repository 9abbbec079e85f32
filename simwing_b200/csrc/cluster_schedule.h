// Cluster sweep schedule: one thread-block cluster solves one structure.
//
// The nodes are split into one patch per CTA of the cluster (recursive
// bisection, suspension endpoint nodes kept together) and live in that
// CTA's shared memory for the whole step.  Each constraint kind is
// coloured over the whole mesh (DSatur); a colour is one stage, and every
// constraint of a stage is executed by the CTA that owns most of its nodes,
// reaching nodes of other CTAs through distributed shared memory.  A
// cluster barrier separates stages.  Node references are 16-bit: the owner
// rank in the top 4 bits and the index in its patch in the low 12 bits.
//
// Split stages (optional, SWB_OPT_SPLIT_STAGES): a constraint whose
// nodes all lie in one CTA's patch is interior.  Per kind, the interior
// constraints run first, coloured per CTA, with only a CTA barrier between
// their stages (interior constraints of different CTAs share no node); one
// cluster barrier follows.  The constraints that span CTAs are coloured
// together; their large colours run one stage each with a cluster barrier
// after it, and the short tail of small colours runs on a single CTA with CTA
// barriers, closed by one cluster barrier.  Each stage carries the kind of
// barrier that follows it.  Classic stages (the default: one colouring of
// the whole mesh, a cluster barrier after every stage) are also what packed
// batches need, whose structures must take identical barriers.  On the
// B200 the classic form is faster: a stage's cost is mostly its records'
// issue and latency, not its barrier, and split stages double the stages.
//
// Sweep order per kind: stage-major, then CTA rank, then record order --
// the reference serial solver run on the definition permuted into this
// order performs exactly the device sweep: constraints of one stage share
// no node, and within a run of stages joined by CTA barriers every node is
// touched by one CTA only.
#pragma once

#include "common.h"

#include <array>
#include <cstdint>
#include <vector>

namespace swb {

constexpr int kClusterMaxCtas = 16;
constexpr uint32_t kClusterPatchNodes = 4096;

struct ClusterKind {
    int stages = 0;
    // [ctas * (stages + 1)]: record offsets of (cta, stage); records are
    // stored CTA-major, stage within.
    std::vector<uint32_t> offsets;
    std::vector<uint32_t> ab;    // ref(a) | ref(b) << 16
    std::vector<uint32_t> cd;    // dihedral: ref(c) | ref(d) << 16
    std::vector<float> rest;
    std::vector<float> comp;     // distance: sign bit = cable
    std::vector<uint32_t> def_index;
    uint32_t max_cta_records = 0;  // multipliers held in shared memory per CTA
    std::vector<uint8_t> cluster_sync;  // [stages]: 1 = cluster barrier after the stage, 0 = CTA barrier
    // split stages: the first interior_stages stages hold only records whose
    // nodes all lie in the executing CTA's patch; boundary_stages follow
    int interior_stages = 0, boundary_stages = 0;
};

struct ClusterSchedule {
    int ctas = 0;
    uint32_t node_count = 0;
    std::vector<uint32_t> node_of_slot, slot_of_node;  // slots: patch-major
    std::vector<uint32_t> patch_begin;                 // [ctas + 1]
    uint32_t max_patch = 0;
    // kinds[0] distance-type constraints, kinds[1] dihedrals, kinds[2]
    // membrane elements; an iteration runs distance, membrane, then dihedral
    // stages (soft_body.cpp:1318-1369)
    std::array<ClusterKind, 3> kinds;
    // seam closing pass: level-scheduled in sweep order, per (cta, stage)
    int seam_stages = 0;
    std::vector<uint32_t> seam_offsets;  // [ctas * (seam_stages + 1)]
    std::vector<uint32_t> seam_ab;
    int susp_cta = -1;
    // Line iteration window (classic stages only): when the last two stages
    // of an iteration touch no suspension endpoint node, the iteration's line
    // iteration runs beside them on a warp of the suspension CTA that has no
    // record in either, instead of after them behind a barrier of its own.
    // line_stage = the first of the two (global stage index: distance stages
    // then dihedral stages), -1 without a window; line_owner_records = the
    // suspension CTA's larger record count of the two.
    int line_stage = -1;
    uint32_t line_owner_records = 0;
    std::vector<uint64_t> distance_order, dihedral_order, membrane_order;
    // Load-path cable sweeps (soft_body.cpp:528-629, 1265-1317): one pair is
    // a reverse then a forward pass over the cables and ties in graph-depth
    // order; each pass is level-scheduled (a constraint one level after the
    // last earlier one sharing a node), so a level's constraints share no
    // node and the levels reproduce the serial pass.  pair_stages = levels of
    // both passes; pair_offsets [ctas * (pair_stages + 1)] index pair_rec,
    // the distance records (kind 0) each CTA runs per level (its own: their
    // multipliers are the general sweep's).
    int pair_stages = 0;
    std::vector<uint32_t> pair_offsets, pair_rec;
};

// Colour stages per iteration, all kinds.
inline int total_stages(const ClusterSchedule& s) {
    return s.kinds[0].stages + s.kinds[1].stages + s.kinds[2].stages;
}
// Kind and stage within the kind of global stage g of an iteration
// (distance stages, membrane stages, dihedral stages).
inline void global_stage(const ClusterSchedule& s, int g, int& kind, int& local) {
    const int S0 = s.kinds[0].stages, S2 = s.kinds[2].stages;
    if (g < S0) {
        kind = 0;
        local = g;
    } else if (g < S0 + S2) {
        kind = 2;
        local = g - S0;
    } else {
        kind = 1;
        local = g - S0 - S2;
    }
}

// Cluster barriers per constraint iteration (stages followed by one, plus
// the suspension stage unless the line iteration runs beside two stages).
inline int cluster_barriers_per_iteration(const ClusterSchedule& s) {
    int n = s.susp_cta >= 0 && s.line_stage < 0 ? 1 : 0;
    for (const ClusterKind& k : s.kinds)
        for (uint8_t b : k.cluster_sync) n += b;
    return n;
}

// Dynamic shared memory of the cluster step kernel for this schedule
// (nodes, forces/velocities, multipliers -- three per membrane element --,
// stage offsets; with slack for the 16-byte alignment of each array).
inline size_t cluster_shared_bytes(const ClusterSchedule& s) {
    return s.max_patch * 32ull + s.kinds[0].max_cta_records * 4ull + s.kinds[1].max_cta_records * 4ull +
           s.kinds[2].max_cta_records * 12ull + (total_stages(s) + 3) * 4ull + 80;
}

// Returns false (and leaves `out` empty) when the mesh does not fit one
// cluster of `ctas` CTAs (a patch over kClusterPatchNodes nodes).
bool build_cluster_schedule(const OwnedDefinition& d, const std::vector<uint32_t>& suspension_nodes, int ctas,
                            ClusterSchedule& out, bool split = false);

// Move budget of the search for a colouring with fewer colours (per colour
// count tried).
constexpr long kColourSearchMoves = 300000;

// Checks the invariants the cluster kernel relies on; raises on failure.
void verify_cluster_schedule(const OwnedDefinition& d, const std::vector<uint32_t>& suspension_nodes,
                             const ClusterSchedule& s);

// Colouring helper shared with the grid schedule: DSatur over constraints
// given as node lists (2 or 4 nodes), conflicts = shared nodes.
int dsatur_colour(const std::vector<std::array<uint32_t, 4>>& nodes, const std::vector<int>& counts,
                  std::vector<int>& colour);

// Recursive coordinate bisection of nodes into `parts` (see schedule.cpp).
std::vector<int> bisect_nodes(const OwnedDefinition& d, const std::vector<uint32_t>& grouped_nodes, int parts,
                              double tolerance);

}  // namespace swb
