// Host-side registration of the fabric self-contact surface and the
// candidate rows the device broadphase produces.
#pragma once

#include "common.h"

#include <array>
#include <cstdint>
#include <vector>

namespace swb {

// One contact surface over all triangles of a definition, paired with
// itself (structure.cpp:626-636 with SoftBody::addContactSurface,
// contact.cpp:2211-2286): the sorted set of its vertices, the sorted set of
// its edges (a < b) and the triangles in index order.
struct ContactSurface {
    double half_thickness = 0.0;
    std::vector<uint32_t> vertices;
    std::vector<std::array<uint32_t, 2>> edges;
    std::vector<std::array<uint32_t, 3>> triangles;
    uint64_t possible = 0;  // vertex-triangle plus edge-edge feature pairs
    uint64_t excluded = 0;  // of those, the pairs sharing a node
};

// Validates the surface as addContactSurface does (throws swb::Error).
ContactSurface build_contact_surface(const swb_structure_definition& definition, double half_thickness);

// Device broadphase output: row r < vertices.size() holds the triangles of
// vertex r's candidate features, row vertices.size() + i the later edges j
// of edge i's; cols[offsets[r] .. offsets[r + 1]) in ascending order.
struct CandidateRows {
    std::vector<uint64_t> offsets;
    std::vector<uint32_t> cols;
};

// The ContactFeatureKey (contact.h:95-101) of the candidate in `row`
// against column `col`: vertex-triangle {vertex} x {triangle}, edge-edge
// {a, b} x {c, d}.
swb_contact_key contact_key_of(const ContactSurface& surface, uint64_t row, uint64_t col);

CandidateRows contact_candidate_rows(const ContactSurface& surface, const double* prev, const double* cur,
                                     uint64_t node_count, double separation);

}  // namespace swb
