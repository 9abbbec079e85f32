// Fabric self-contact surface registration (SoftBody::addContactSurface,
// src/softwing/contact.cpp:2211-2286, for the surface group of all
// triangles that Structure registers, src/fsi/structure.cpp:626-636).
#include "contact_surface.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <map>

namespace swb {

namespace {

struct P3 {
    double x, y, z;
};
P3 sub(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
double norm2(P3 v) { return v.x * v.x + v.y * v.y + v.z * v.z; }
P3 cross(P3 a, P3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

}  // namespace

ContactSurface build_contact_surface(const swb_structure_definition& d, double half_thickness) {
    if (!std::isfinite(half_thickness) || !(half_thickness > 0.0))
        raise(SWB_INVALID_ARGUMENT, "Contact surface half-thickness must be finite and positive");
    if (d.node_count > std::numeric_limits<uint32_t>::max() || d.triangle_count > std::numeric_limits<uint32_t>::max())
        raise(SWB_INVALID_ARGUMENT, "contact surface too large for 32-bit indices");
    ContactSurface s;
    s.half_thickness = half_thickness;
    s.triangles.reserve(d.triangle_count);
    std::vector<uint8_t> used(d.node_count, 0);
    for (uint64_t t = 0; t < d.triangle_count; ++t) {
        const uint64_t* n = d.triangles[t].nodes;
        if (n[0] >= d.node_count || n[1] >= d.node_count || n[2] >= d.node_count)
            raise(SWB_OUT_OF_RANGE, "Contact surface triangle contains an invalid node");
        if (n[0] == n[1] || n[1] == n[2] || n[2] == n[0])
            raise(SWB_INVALID_ARGUMENT, "Contact surface contains a repeated-node triangle");
        const auto pos = [&](uint64_t i) {
            const swb_vec3& p = d.nodes[i].position;
            return P3{p.x, p.y, p.z};
        };
        const P3 a = pos(n[0]), b = pos(n[1]), c = pos(n[2]);
        for (const P3& p : {a, b, c})
            if (!std::isfinite(p.x) || !std::isfinite(p.y) || !std::isfinite(p.z))
                raise(SWB_INVALID_ARGUMENT, "Contact surface positions must be finite");
        const double ab2 = norm2(sub(b, a)), ac2 = norm2(sub(c, a)), bc2 = norm2(sub(c, b));
        const double scale2 = std::max({ab2, ac2, bc2});
        const double area2 = norm2(cross(sub(b, a), sub(c, a)));
        const double rel = 64.0 * std::numeric_limits<double>::epsilon();
        if (!(scale2 > 0.0) || !(area2 > rel * rel * scale2 * scale2))
            raise(SWB_INVALID_ARGUMENT, "Contact surface contains a degenerate triangle");
        const std::array<uint32_t, 3> tri{static_cast<uint32_t>(n[0]), static_cast<uint32_t>(n[1]),
                                          static_cast<uint32_t>(n[2])};
        s.triangles.push_back(tri);
        for (int k = 0; k < 3; ++k) {
            used[tri[k]] = 1;
            const uint32_t u = tri[k], v = tri[(k + 1) % 3];
            s.edges.push_back({std::min(u, v), std::max(u, v)});
        }
    }
    for (uint64_t i = 0; i < d.node_count; ++i)
        if (used[i]) s.vertices.push_back(static_cast<uint32_t>(i));
    std::sort(s.edges.begin(), s.edges.end());
    s.edges.erase(std::unique(s.edges.begin(), s.edges.end()), s.edges.end());
    // Feature pairs the reference enumerates (contact.cpp:1218-1257): every
    // vertex against every triangle, every two distinct edges.  Excluded:
    // a triangle holding the vertex (three per triangle), two edges sharing
    // a node (edge degree d contributes d (d - 1) / 2 at that node).
    const uint64_t nv = s.vertices.size(), ne = s.edges.size(), nt = s.triangles.size();
    std::vector<uint64_t> degree(d.node_count, 0);
    for (const auto& e : s.edges) {
        ++degree[e[0]];
        ++degree[e[1]];
    }
    uint64_t shared = 0;
    for (uint64_t g : degree) shared += g * (g ? g - 1 : 0) / 2;
    s.possible = nv * nt + (ne ? ne * (ne - 1) / 2 : 0);
    s.excluded = 3 * nt + shared;
    return s;
}

swb_contact_key contact_key_of(const ContactSurface& S, uint64_t row, uint64_t col) {
    swb_contact_key key{};
    const size_t nv = S.vertices.size();
    if (row < nv) {
        key.kind = SWB_FEATURE_VERTEX_TRIANGLE;
        key.first[0] = S.vertices[row];
        key.second[0] = col;
    } else {
        key.kind = SWB_FEATURE_EDGE_EDGE;
        key.first[0] = S.edges[row - nv][0];
        key.first[1] = S.edges[row - nv][1];
        key.second[0] = S.edges[col][0];
        key.second[1] = S.edges[col][1];
    }
    return key;
}

}  // namespace swb
