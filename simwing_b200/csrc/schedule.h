// Device sweep schedule: node partitions, per-CTA constraint tables and
// colour stages.  Built once per mesh on the host.
//
// The XPBD sweep is Gauss-Seidel: a constraint sees every correction made
// before it.  Constraints that share no node commute exactly (their
// arithmetic touches disjoint memory), so any order that keeps the relative
// order of every pair of constraints sharing a node gives bit-identical
// results.  The schedule exploits that with a hierarchy of node partitions:
//
//   level 1   nodes are split into one patch per CTA; a constraint whose
//             nodes all lie in one patch is solved by that CTA out of shared
//             memory, one colour stage at a time (__syncthreads between
//             stages).  Patches are disjoint, so all CTAs run concurrently.
//   level 2.. the constraints cut by level 1 are partitioned again over the
//             nodes they touch with different cut planes; whatever becomes
//             interior is solved the same way from a gathered patch.
//   global    whatever is still cut after the last level is coloured
//             globally; each colour is one device-wide phase.
//
// The resulting sweep order per constraint kind is: level 1 (CTA-major,
// stage-major), level 2, ..., global colours.  `sweep_order` records it as
// definition indices so the reference serial solver can be run with its
// constraint lists permuted into exactly this order.
#pragma once

#include "common.h"

#include <array>
#include <cstdint>
#include <vector>

namespace swb {

constexpr int kMaxLevels = 4;
constexpr int kKinds = 2;  // 0 = distance-like, 1 = dihedral

// One per-level, per-kind table: constraints grouped by CTA, each CTA's
// group split into colour stages.  Node references are CTA-local indices
// into that level's patch.
struct Table {
    int stages = 0;                      // max stages over CTAs
    std::vector<uint32_t> block_begin;   // [G+1] element offsets (padded)
    std::vector<uint32_t> stage_offsets; // [G * (stages+1)] relative to block_begin
    // distance: ab = a | b << 16 (local), rest, comp (sign bit = cable)
    // dihedral: abcd = {a | b << 16, c | d << 16}, rest, comp
    std::vector<uint32_t> ab;
    std::vector<uint32_t> cd;            // dihedral only
    std::vector<float> rest;
    std::vector<float> comp;
    std::vector<uint32_t> def_index;     // definition index (for permutation)
    std::vector<uint8_t> valid;          // 0 for padding
    uint32_t max_block_count = 0;        // max padded elements in one CTA
};

// Global colour stages of one kind: node references are slots.
struct GlobalTable {
    std::vector<uint32_t> colour_offsets;  // [colours+1]
    std::vector<uint32_t> a, b, c, d;      // slots (c, d dihedral only)
    std::vector<float> rest, comp;
    std::vector<uint32_t> def_index;
};

struct Schedule {
    int blocks = 0;
    int levels = 0;  // number of local levels actually used (>= 1)
    uint32_t node_count = 0;
    // slot <-> node: slots are level-1 patch-major.
    std::vector<uint32_t> node_of_slot, slot_of_node;
    std::vector<uint32_t> l1_begin;        // [G+1] slot ranges (contiguous)
    // Level >= 2 patches: slot lists per CTA.
    std::array<std::vector<uint32_t>, kMaxLevels> patch_begin;  // [G+1]
    std::array<std::vector<uint32_t>, kMaxLevels> patch_slots;
    std::array<std::array<Table, kKinds>, kMaxLevels> tables;
    std::array<GlobalTable, kKinds> global;
    // Level-1 interface: local indices (within the CTA's patch) of nodes that
    // any non-level-1 phase touches.  Flushed to / reloaded from global
    // memory around those phases.
    std::vector<uint32_t> iface_begin;     // [G+1]
    std::vector<uint16_t> iface_local;
    // Seam-closing pass: stitches level-scheduled in sweep order, slots.
    std::vector<uint32_t> seam_stage_offsets;
    std::vector<uint32_t> seam_a, seam_b;
    // Suspension owner CTA (all suspension endpoint nodes are in its
    // level-1 patch), or -1.
    int suspension_block = -1;
    // Sweep orders (definition indices) for the oracle permutation.
    std::vector<uint64_t> distance_order, dihedral_order;
    // Stats.
    int max_patch_nodes = 0;         // level 1
    int max_gather_nodes = 0;        // levels >= 2
    uint64_t level_constraints[kMaxLevels] = {0, 0, 0, 0};
    uint64_t global_constraints = 0;
};

struct ScheduleOptions {
    int blocks = 148;
    int levels = 3;          // local levels (1..kMaxLevels)
    bool global_only = false;
    double balance_tolerance = 0.06;
};

// `suspension_nodes` lists node indices that must share one level-1 patch.
Schedule build_schedule(const OwnedDefinition& d,
                        const std::vector<uint32_t>& suspension_nodes,
                        const ScheduleOptions& options);

// Checks every invariant the device relies on (disjoint patches, node-
// disjoint stages, each constraint exactly once, interface completeness,
// sweep orders); raises SWB_INVALID_ARGUMENT describing the first failure.
void verify_schedule(const OwnedDefinition& d,
                     const std::vector<uint32_t>& suspension_nodes,
                     const Schedule& s);

// Nodes of the suspension segments' endpoints (attachments, junctions).
std::vector<uint32_t> suspension_endpoint_nodes(const OwnedDefinition& d);

}  // namespace swb
