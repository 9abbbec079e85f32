// Scene -> structure definition: simwing::fsi::assembleSceneStructure
// (src/fsi/scene_structure.cpp:894-1284) with the scene-v2 checks it runs
// first (validateScene, src/fsi/scene.cpp:552-1040) for the fields a
// swb_scene carries (no regions, openings or metadata: they do not reach
// the structure).  The assembly is restated step for step where its result
// is compared bit for bit with the reference's: entities in stable-ID order,
// vertex nodes (those of triangles and surface attachments) then junction
// nodes, mass lumped in long double in triangle then seam order, hinges in
// (sheet, canonical edge) order with the series-strip compliance from the
// material charts and the signed rest angle from the geometry, seams as
// stitches then the two chains' rails, and the pilot's suspension tree
// oriented from the canopy leaves to the harness root by breadth-first
// search in endpoint order.
#include "common.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <queue>
#include <set>
#include <tuple>
#include <unordered_map>
#include <vector>

namespace swb {
namespace {

// EntityKind (scene.h:239-253) and the diagnostic codes
// (scene_structure.h:46-57, scene.h:255-276).
enum Entity : uint32_t {
    kScene = 1, kRegion, kVertex, kFabricMaterial, kTriangle, kOpening, kLineMaterial, kPilot, kAttachment,
    kSuspensionLine, kSeamMaterial, kSeam, kSuspensionJunction
};
enum Code : uint32_t {
    kInvalidScene = 1, kMappingOverflow, kMaterialIncompatible, kDegenerateChart, kZeroMassNode, kUnsupportedPilot,
    kUnsupportedHarness, kUnsupportedSuspension, kUnsupportedSeam, kUnsupportedBending
};
enum Validation : uint32_t {
    vDuplicateId = 4, vInvalidId, vNonFinite, vInvalidPhysical, vDegenerateTriangle, vDuplicateTriangle,
    vMissingVertex, vMissingRegion, vMissingMaterial, vInvalidSides, vInvalidOpening, vInvalidEnum, vMissingPilot,
    vInvalidAttachmentTarget, vDanglingLineAttachment, vInvalidLine, vInvalidSeam
};

struct Diag {
    uint32_t code, validation, kind;
    uint64_t id;
    std::string message;
};

struct V3 { double x, y, z; };
V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 cross3(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
double dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
double len3(V3 a) { return std::sqrt(dot3(a, a)); }
V3 scale3(V3 a, double s) { return {s * a.x, s * a.y, s * a.z}; }
V3 v3(const swb_vec3& v) { return {v.x, v.y, v.z}; }
bool finite3(const swb_vec3& v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); }
bool zero3(const swb_vec3& v) { return v.x == 0.0 && v.y == 0.0 && v.z == 0.0; }

template <class T>
std::vector<const T*> by_id(const T* items, uint64_t n) {
    std::vector<const T*> out;
    out.reserve(n);
    for (uint64_t i = 0; i < n; ++i) out.push_back(items + i);
    std::stable_sort(out.begin(), out.end(), [](const T* a, const T* b) { return a->id < b->id; });
    return out;
}

struct Assembler {
    const swb_scene& s;
    const swb_scene_settings& st;
    std::vector<Diag> diags;
    OwnedDefinition def;
    long double fabric_mass = 0.0L, seam_mass = 0.0L;

    void add(uint32_t code, uint32_t kind, uint64_t id, std::string message, uint32_t validation = 0) {
        diags.push_back({code, validation, kind, id, std::move(message)});
    }
    void invalid(uint32_t validation, uint32_t kind, uint64_t id, std::string message) {
        add(kInvalidScene, kind, id, std::move(message), validation);
    }

    template <class T>
    std::set<uint64_t> ids(const T* items, uint64_t n, uint32_t kind) {
        std::map<uint64_t, int> count;
        for (uint64_t i = 0; i < n; ++i) ++count[items[i].id];
        std::set<uint64_t> out;
        for (const auto& [id, c] : count) {
            if (id == 0) invalid(vInvalidId, kind, id, "stable ID must be non-zero");
            if (c > 1) invalid(vDuplicateId, kind, id, "duplicate stable ID");
            out.insert(id);
        }
        return out;
    }

    // validateScene for the fields a swb_scene carries.
    void validate() {
        const auto vertex_ids = ids(s.vertices, s.vertex_count, kVertex);
        const auto fabric_ids = ids(s.fabrics, s.fabric_count, kFabricMaterial);
        const auto seam_material_ids = ids(s.seam_materials, s.seam_material_count, kSeamMaterial);
        ids(s.triangles, s.triangle_count, kTriangle);
        ids(s.seams, s.seam_count, kSeam);
        const auto line_material_ids = ids(s.line_materials, s.line_material_count, kLineMaterial);
        const auto pilot_ids = ids(s.pilots, s.pilot_count, kPilot);
        const auto junction_ids = ids(s.junctions, s.junction_count, kSuspensionJunction);
        const auto attachment_ids = ids(s.attachments, s.attachment_count, kAttachment);
        ids(s.lines, s.line_count, kSuspensionLine);
        std::unordered_map<uint64_t, const swb_scene_vertex*> vertices;
        std::map<uint64_t, int> vcount;
        for (uint64_t i = 0; i < s.vertex_count; ++i) ++vcount[s.vertices[i].id];
        for (const auto* v : by_id(s.vertices, s.vertex_count)) {
            if (vcount[v->id] == 1) vertices.emplace(v->id, v);
            if (!finite3(v->position)) invalid(vNonFinite, kVertex, v->id, "vertex position is not finite");
        }
        for (const auto* m : by_id(s.fabrics, s.fabric_count)) {
            const double f[] = {m->warp_stiffness, m->weft_stiffness, m->shear_stiffness, m->bending_stiffness,
                                m->areal_density, m->damping_seconds, m->porosity, m->permeability};
            if (!std::all_of(std::begin(f), std::end(f), [](double x) { return std::isfinite(x); }))
                invalid(vNonFinite, kFabricMaterial, m->id, "fabric material contains a non-finite value");
            else if (!(m->warp_stiffness > 0.0) || !(m->weft_stiffness > 0.0) || !(m->shear_stiffness > 0.0) ||
                     m->bending_stiffness < 0.0 || !(m->areal_density > 0.0) || m->damping_seconds < 0.0 ||
                     m->porosity < 0.0 || m->porosity > 1.0 || m->permeability < 0.0)
                invalid(vInvalidPhysical, kFabricMaterial, m->id, "fabric material has an invalid physical value");
        }
        for (const auto* m : by_id(s.seam_materials, s.seam_material_count)) {
            if (!std::isfinite(m->linear_density) || !std::isfinite(m->axial_stiffness))
                invalid(vNonFinite, kSeamMaterial, m->id, "seam material contains a non-finite value");
            else if (!(m->linear_density > 0.0) || !(m->axial_stiffness > 0.0))
                invalid(vInvalidPhysical, kSeamMaterial, m->id,
                        "seam material density and axial stiffness must be positive");
        }
        std::set<std::array<uint64_t, 3>> faces;
        for (const auto* t : by_id(s.triangles, s.triangle_count)) {
            for (const auto& c : t->chart)
                if (!std::isfinite(c[0]) || !std::isfinite(c[1])) {
                    invalid(vNonFinite, kTriangle, t->id, "triangle material coordinate is not finite");
                    break;
                }
            std::set<uint64_t> local;
            for (uint64_t v : t->vertex_ids) {
                if (!vertex_ids.count(v)) invalid(vMissingVertex, kTriangle, t->id, "triangle references a missing vertex");
                local.insert(v);
            }
            if (local.size() != 3 || degenerate(t->vertex_ids, vertices))
                invalid(vDegenerateTriangle, kTriangle, t->id, "triangle has repeated or effectively collinear vertices");
            if (!fabric_ids.count(t->material_id))
                invalid(vMissingMaterial, kTriangle, t->id, "triangle references a missing fabric material");
            if (t->sheet_id == 0) invalid(vInvalidId, kTriangle, t->id, "triangle fabric sheet ID must be non-zero");
            std::array<uint64_t, 3> key{t->vertex_ids[0], t->vertex_ids[1], t->vertex_ids[2]};
            std::sort(key.begin(), key.end());
            if (!faces.insert(key).second)
                invalid(vDuplicateTriangle, kTriangle, t->id, "triangle duplicates an existing geometric face");
        }
        // seams (scene.cpp:825-893): equal chains of at least two vertices,
        // no vertex twice in a chain, a vertex in both chains only as their
        // shared first or last, every (sorted) pair once over all seams, at
        // least one distinct pair
        std::set<std::array<uint64_t, 2>> seam_pairs;
        for (const auto* m : by_id(s.seams, s.seam_count)) {
            const uint64_t n = m->count;
            if (m->first_begin + n > s.seam_vertex_id_count || m->second_begin + n > s.seam_vertex_id_count)
                raise(SWB_INVALID_ARGUMENT, "seam chain outside seam_vertex_ids");
            const uint64_t* chain[2] = {s.seam_vertex_ids + m->first_begin, s.seam_vertex_ids + m->second_begin};
            bool bad = n < 2;
            std::set<uint64_t> local[2];
            for (int c = 0; c < 2; ++c)
                for (uint64_t i = 0; i < n; ++i) {
                    if (!vertex_ids.count(chain[c][i]))
                        invalid(vMissingVertex, kSeam, m->id,
                                std::string("seam ") + (c ? "second" : "first") + " chain references a missing vertex");
                    if (!local[c].insert(chain[c][i]).second) bad = true;
                }
            for (uint64_t id : local[0]) {
                if (!local[1].count(id)) continue;
                const bool shared_first = n > 0 && chain[0][0] == id && chain[1][0] == id;
                const bool shared_last = n > 0 && chain[0][n - 1] == id && chain[1][n - 1] == id;
                if (!shared_first && !shared_last) bad = true;
            }
            size_t distinct = 0;
            for (uint64_t i = 0; i < n; ++i) {
                if (chain[0][i] != chain[1][i]) ++distinct;
                const std::array<uint64_t, 2> pair{std::min(chain[0][i], chain[1][i]),
                                                   std::max(chain[0][i], chain[1][i])};
                if (!seam_pairs.insert(pair).second) bad = true;
            }
            if (bad || distinct == 0)
                invalid(vInvalidSeam, kSeam, m->id,
                        "seam needs equal-length unique ordered chains with at least one distinct pair; only "
                        "matching endpoints may be shared");
            if (!seam_material_ids.count(m->material_id))
                invalid(vMissingMaterial, kSeam, m->id, "seam references a missing seam material");
        }
        for (const auto* m : by_id(s.line_materials, s.line_material_count)) {
            const double f[] = {m->diameter, m->linear_density, m->axial_stiffness, m->drag_coefficient};
            if (!std::all_of(std::begin(f), std::end(f), [](double x) { return std::isfinite(x); }))
                invalid(vNonFinite, kLineMaterial, m->id, "line material contains a non-finite value");
            else if (!(m->diameter > 0.0) || !(m->linear_density > 0.0) || !(m->axial_stiffness > 0.0) ||
                     m->drag_coefficient < 0.0)
                invalid(vInvalidPhysical, kLineMaterial, m->id, "line material has an invalid physical value");
        }
        for (const auto* p : by_id(s.pilots, s.pilot_count)) {
            const swb_quat& q = p->body_to_world;
            const double qq = q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z;
            if (!std::isfinite(p->mass) || !finite3(p->center_of_mass) || !finite3(p->linear_velocity) ||
                !std::isfinite(q.w) || !std::isfinite(q.x) || !std::isfinite(q.y) || !std::isfinite(q.z) ||
                !finite3(p->principal_inertia))
                invalid(vNonFinite, kPilot, p->id, "pilot contains a non-finite value");
            else if (!(p->mass > 0.0) || !(p->principal_inertia.x > 0.0) || !(p->principal_inertia.y > 0.0) ||
                     !(p->principal_inertia.z > 0.0) || std::abs(qq - 1.0) > 1.0e-6)
                invalid(vInvalidPhysical, kPilot, p->id,
                        "pilot mass/inertia must be positive and orientation normalized");
        }
        for (const auto* j : by_id(s.junctions, s.junction_count)) {
            if (!finite3(j->position) || !std::isfinite(j->mass))
                invalid(vNonFinite, kSuspensionJunction, j->id, "suspension junction contains a non-finite value");
            else if (j->mass < 0.0 || (!j->fixed && !(j->mass > 0.0)))
                invalid(vInvalidPhysical, kSuspensionJunction, j->id,
                        "dynamic suspension junction requires positive explicit mass");
            if (vertex_ids.count(j->id))
                invalid(vInvalidId, kSuspensionJunction, j->id,
                        "suspension junction ID must not collide with a surface vertex ID");
        }
        for (const auto* a : by_id(s.attachments, s.attachment_count)) {
            if (a->kind == SWB_ATTACH_SURFACE_VERTEX) {
                if (!vertex_ids.count(a->vertex_id) || a->pilot_id || a->junction_id || !zero3(a->pilot_local_position))
                    invalid(vInvalidAttachmentTarget, kAttachment, a->id,
                            "surface attachment must reference one existing vertex");
            } else if (a->kind == SWB_ATTACH_PILOT_HARNESS) {
                if (!pilot_ids.count(a->pilot_id))
                    invalid(vMissingPilot, kAttachment, a->id, "pilot attachment references a missing pilot");
                if (a->vertex_id || a->junction_id || !finite3(a->pilot_local_position))
                    invalid(vInvalidAttachmentTarget, kAttachment, a->id,
                            "pilot attachment target or local position is invalid");
            } else if (a->kind == SWB_ATTACH_JUNCTION) {
                if (!junction_ids.count(a->junction_id) || a->vertex_id || a->pilot_id ||
                    !zero3(a->pilot_local_position))
                    invalid(vInvalidAttachmentTarget, kAttachment, a->id,
                            "junction attachment must reference one existing suspension junction");
            } else {
                invalid(vInvalidEnum, kAttachment, a->id, "attachment kind is invalid");
            }
        }
        for (const auto* l : by_id(s.lines, s.line_count)) {
            if (l->role < 1 || l->role > 4) invalid(vInvalidEnum, kSuspensionLine, l->id, "suspension line role is invalid");
            if (!attachment_ids.count(l->start_attachment_id) || !attachment_ids.count(l->end_attachment_id))
                invalid(vDanglingLineAttachment, kSuspensionLine, l->id, "suspension line references a missing attachment");
            if (l->start_attachment_id == l->end_attachment_id || !std::isfinite(l->rest_length) ||
                !(l->rest_length > 0.0))
                invalid(vInvalidLine, kSuspensionLine, l->id, "suspension line endpoints and rest length are invalid");
            if (!line_material_ids.count(l->material_id))
                invalid(vMissingMaterial, kSuspensionLine, l->id, "suspension line references a missing line material");
        }
    }

    static bool degenerate(const uint64_t ids[3], const std::unordered_map<uint64_t, const swb_scene_vertex*>& vs) {
        const swb_scene_vertex* p[3];
        for (int k = 0; k < 3; ++k) {
            const auto it = vs.find(ids[k]);
            if (it == vs.end() || !finite3(it->second->position)) return false;
            p[k] = it->second;
        }
        const V3 ab = sub(v3(p[1]->position), v3(p[0]->position));
        const V3 ac = sub(v3(p[2]->position), v3(p[0]->position));
        const V3 bc = sub(v3(p[2]->position), v3(p[1]->position));
        const double longest = std::max({dot3(ab, ab), dot3(ac, ac), dot3(bc, bc)});
        if (!(longest > 0.0) || !std::isfinite(longest)) return true;
        const V3 c = cross3(ab, ac);
        return !(dot3(c, c) > 1.0e-24 * longest * longest);
    }

    // checkedMappingBytes bounds of checkBounds with the default limits
    // (10^7 nodes, triangles and constraints, 256 MiB of stable-ID maps).
    bool check_bounds() {
        const uint64_t nodes = s.vertex_count + s.junction_count;
        if (nodes > 10'000'000)
            add(kMappingOverflow, kScene, 0, "scene vertex and junction count exceeds the structure node bound");
        if (s.triangle_count > 10'000'000)
            add(kMappingOverflow, kScene, 0, "scene triangle count exceeds the structure triangle bound");
        uint64_t seam_constraints = 0;
        for (uint64_t i = 0; i < s.seam_count; ++i) seam_constraints += 3 * s.seams[i].count - 2;
        if (s.line_count + seam_constraints > 10'000'000)
            add(kMappingOverflow, kScene, 0, "scene seam and suspension-line constraints exceed the structure bound");
        const long double bytes = 8.0L * (s.vertex_count + s.junction_count + 2.0L * s.triangle_count +
                                          2.0L * s.line_count + s.attachment_count) +
                                  24.0L * s.seam_count + 32.0L * s.triangle_count;
        if (bytes > 256.0L * 1024.0L * 1024.0L)
            add(kMappingOverflow, kScene, 0, "stable-ID mappings exceed the configured byte bound");
        return diags.empty();
    }

    void run();
    void bending(const std::vector<const swb_scene_triangle*>& triangles,
                 const std::map<uint64_t, const swb_scene_vertex*>& vertices,
                 const std::map<uint64_t, const swb_scene_fabric*>& materials,
                 const std::map<uint64_t, uint64_t>& node);
    void seams(const std::map<uint64_t, const swb_scene_vertex*>& vertices, const std::map<uint64_t, uint64_t>& node,
               std::vector<long double>& lumped);
    void pilot_suspension(const swb_scene_pilot& pilot, const std::map<uint64_t, uint64_t>& node,
                          const std::map<uint64_t, const swb_scene_line_material*>& line_materials);
};

// compatibleMaterial (scene_structure.cpp:209-229): the diagonal case of
// the membrane stiffness inverse's conditioning test.
bool compatible_material(const swb_scene_fabric& m) {
    const double determinant = m.warp_stiffness * m.weft_stiffness * m.shear_stiffness;
    const double scale = std::max({m.warp_stiffness, m.weft_stiffness, m.shear_stiffness});
    const double tolerance = 128.0 * std::numeric_limits<double>::epsilon() * scale * scale * scale;
    return scale > 0.0 && std::isfinite(determinant) && std::isfinite(tolerance) && determinant > tolerance &&
           std::isfinite(1.0 / m.warp_stiffness) && std::isfinite(1.0 / m.weft_stiffness) &&
           std::isfinite(1.0 / m.shear_stiffness);
}

// compatibleMaterialCoordinates (:231-262): positive, well-conditioned chart.
bool compatible_chart(const swb_scene_triangle& t) {
    const double fx = t.chart[1][0] - t.chart[0][0], fy = t.chart[1][1] - t.chart[0][1];
    const double sx = t.chart[2][0] - t.chart[0][0], sy = t.chart[2][1] - t.chart[0][1];
    const double determinant = fx * sy - sx * fy;
    const double tx = t.chart[2][0] - t.chart[1][0], ty = t.chart[2][1] - t.chart[1][1];
    const double longest = std::max({fx * fx + fy * fy, sx * sx + sy * sy, tx * tx + ty * ty});
    const double tolerance = 64.0 * std::numeric_limits<double>::epsilon() * longest;
    return longest > 0.0 && std::isfinite(determinant) && std::isfinite(tolerance) && determinant > tolerance;
}

double chart_area(const swb_scene_triangle& t) {
    const double fx = t.chart[1][0] - t.chart[0][0], fy = t.chart[1][1] - t.chart[0][1];
    const double sx = t.chart[2][0] - t.chart[0][0], sy = t.chart[2][1] - t.chart[0][1];
    return 0.5 * (fx * sy - sx * fy);
}

// assembleBending (:278-420): per (sheet, canonical edge), two consistently
// oriented incidences make one hinge.
void Assembler::bending(const std::vector<const swb_scene_triangle*>& triangles,
                        const std::map<uint64_t, const swb_scene_vertex*>& vertices,
                        const std::map<uint64_t, const swb_scene_fabric*>& materials,
                        const std::map<uint64_t, uint64_t>& node) {
    struct Inc { const swb_scene_triangle* t; uint64_t from, to, opposite; };
    std::map<std::array<uint64_t, 3>, std::vector<Inc>> edges;
    for (const auto* t : triangles)
        for (int k = 0; k < 3; ++k) {
            const uint64_t from = t->vertex_ids[k], to = t->vertex_ids[(k + 1) % 3], opp = t->vertex_ids[(k + 2) % 3];
            edges[{t->sheet_id, std::min(from, to), std::max(from, to)}].push_back({t, from, to, opp});
        }
    for (const auto& [key, inc] : edges) {
        if (inc.size() == 1) continue;  // a boundary edge has no hinge
        if (inc.size() != 2) {
            add(kUnsupportedBending, kTriangle, inc.front().t->id,
                "non-manifold edge " + std::to_string(key[1]) + "-" + std::to_string(key[2]) + " in sheet " +
                    std::to_string(key[0]) + " cannot define one fabric bending hinge");
            continue;
        }
        const Inc& f = inc[0];
        const Inc& g = inc[1];
        if (f.from != g.to || f.to != g.from) {
            add(kUnsupportedBending, kTriangle, f.t->id,
                "inconsistently oriented edge " + std::to_string(key[1]) + "-" + std::to_string(key[2]) +
                    " in sheet " + std::to_string(key[0]) + " cannot define a signed fabric bending hinge");
            continue;
        }
        const double r0 = materials.at(f.t->material_id)->bending_stiffness;
        const double r1 = materials.at(g.t->material_id)->bending_stiffness;
        if (!(r0 > 0.0) || !(r1 > 0.0)) continue;  // a zero-rigidity side: a free hinge
        const V3 a = v3(vertices.at(f.from)->position), b = v3(vertices.at(f.to)->position);
        const V3 c = v3(vertices.at(f.opposite)->position), d = v3(vertices.at(g.opposite)->position);
        const V3 e = sub(b, a);
        const double el = len3(e);
        const V3 n1 = cross3(e, sub(c, a)), n2 = cross3(sub(d, a), e);
        const double l1 = len3(n1), l2 = len3(n2);
        auto chart_of = [](const swb_scene_triangle& t, uint64_t v) {
            for (int k = 0; k < 3; ++k)
                if (t.vertex_ids[k] == v) return std::array<double, 2>{t.chart[k][0], t.chart[k][1]};
            return std::array<double, 2>{0.0, 0.0};
        };
        auto strip = [&](const Inc& i) {
            const auto A = chart_of(*i.t, i.from), B = chart_of(*i.t, i.to), Cc = chart_of(*i.t, i.opposite);
            const double ex = B[0] - A[0], ey = B[1] - A[1], ox = Cc[0] - A[0], oy = Cc[1] - A[1];
            const double edge = std::hypot(ex, ey);
            return std::array<double, 2>{edge, std::abs(ex * oy - ey * ox) / edge};
        };
        const auto s0 = strip(f), s1 = strip(g);
        const double compliance = s0[1] / (2.0 * r0 * s0[0]) + s1[1] / (2.0 * r1 * s1[0]);
        const V3 eu = scale3(e, 1.0 / el), u1 = scale3(n1, 1.0 / l1), u2 = scale3(n2, 1.0 / l2);
        const double cosine = std::clamp(dot3(u1, u2), -1.0, 1.0);
        const double sine = dot3(eu, cross3(u1, u2));
        const double rest = std::atan2(sine, cosine);
        if (!std::isfinite(compliance) || compliance < 0.0 || !std::isfinite(rest)) {
            add(kMaterialIncompatible, kTriangle, f.t->id, "fabric bending hinge is outside the representable XPBD range");
            continue;
        }
        swb_dihedral_def h{};
        h.nodes[0] = node.at(f.from);
        h.nodes[1] = node.at(f.to);
        h.nodes[2] = node.at(f.opposite);
        h.nodes[3] = node.at(g.opposite);
        h.rest_angle = rest;
        h.compliance = compliance;
        def.dihedrals.push_back(h);
    }
}

// assembleSeams (:440-592): per seam, one rigid zero-rest stitch per distinct
// pair, then half-rigidity rails along each chain (compliance 2 L / EA), and
// each centreline segment's mass split over its four endpoint nodes.
void Assembler::seams(const std::map<uint64_t, const swb_scene_vertex*>& vertices,
                      const std::map<uint64_t, uint64_t>& node, std::vector<long double>& lumped) {
    std::map<uint64_t, const swb_scene_seam_material*> materials;
    for (uint64_t i = 0; i < s.seam_material_count; ++i) materials.emplace(s.seam_materials[i].id, &s.seam_materials[i]);
    for (const auto* m : by_id(s.seams, s.seam_count)) {
        const size_t before = diags.size();
        const auto* mat = materials.at(m->material_id);
        const uint64_t n = m->count;
        const uint64_t* chain[2] = {s.seam_vertex_ids + m->first_begin, s.seam_vertex_ids + m->second_begin};
        for (uint64_t i = 0; i < n; ++i) {
            const double sep = len3(sub(v3(vertices.at(chain[1][i])->position), v3(vertices.at(chain[0][i])->position)));
            if (!std::isfinite(sep) || sep > st.seam_coincidence_tolerance) {
                add(kUnsupportedSeam, kSeam, m->id,
                    "paired seam vertices are not coincident within the structural tolerance");
                break;
            }
        }
        std::array<std::vector<double>, 2> lengths;
        for (int c = 0; c < 2; ++c)
            for (uint64_t i = 0; i + 1 < n; ++i) {
                const double l = len3(sub(v3(vertices.at(chain[c][i + 1])->position),
                                          v3(vertices.at(chain[c][i])->position)));
                const double compliance = 2.0 * l / mat->axial_stiffness;
                if (!(l > 0.0) || !std::isfinite(l) || !std::isfinite(compliance)) {
                    add(kMaterialIncompatible, kSeam, m->id,
                        "seam segment stiffness cannot be represented as finite XPBD compliance");
                    break;
                }
                lengths[c].push_back(l);
            }
        if (diags.size() != before) continue;
        for (uint64_t i = 0; i < n; ++i) {
            if (chain[0][i] == chain[1][i]) continue;
            swb_constraint_def k{};
            k.kind = SWB_CONSTRAINT_SEAM_STITCH;
            k.first_node = node.at(chain[0][i]);
            k.second_node = node.at(chain[1][i]);
            def.constraints.push_back(k);
        }
        for (int c = 0; c < 2; ++c)
            for (uint64_t i = 0; i + 1 < n; ++i) {
                swb_constraint_def k{};
                k.kind = SWB_CONSTRAINT_DISTANCE;
                k.first_node = node.at(chain[c][i]);
                k.second_node = node.at(chain[c][i + 1]);
                k.rest_length = lengths[c][i];
                k.compliance = 2.0 * lengths[c][i] / mat->axial_stiffness;
                def.constraints.push_back(k);
            }
        for (uint64_t i = 0; i + 1 < n; ++i) {
            const double centreline = 0.5 * (lengths[0][i] + lengths[1][i]);
            const double mass = centreline * mat->linear_density;
            const long double share = static_cast<long double>(mass) / 4.0L;
            for (uint64_t id : {chain[0][i], chain[0][i + 1], chain[1][i], chain[1][i + 1]}) lumped[node.at(id)] += share;
            seam_mass += static_cast<long double>(mass);
        }
    }
}

// assemblePilotSuspension (:592-892): one rigid pilot owns the suspension
// tree; each component is an acyclic tree with one harness root and at
// least one surface leaf, oriented by breadth-first search from the root
// with neighbours in (endpoint kind, endpoint ID, line ID) order.
void Assembler::pilot_suspension(const swb_scene_pilot& pilot, const std::map<uint64_t, uint64_t>& node,
                                 const std::map<uint64_t, const swb_scene_line_material*>& line_materials) {
    const auto lines = by_id(s.lines, s.line_count);
    if (lines.empty()) {
        add(kUnsupportedPilot, kPilot, pilot.id, "rigid pilot requires a connected suspension tree");
        return;
    }
    std::map<uint64_t, const swb_scene_attachment*> attachments;
    for (uint64_t i = 0; i < s.attachment_count; ++i) attachments.emplace(s.attachments[i].id, &s.attachments[i]);
    std::map<uint64_t, const swb_scene_junction*> junctions;
    for (uint64_t i = 0; i < s.junction_count; ++i) junctions.emplace(s.junctions[i].id, &s.junctions[i]);
    using Key = std::pair<uint32_t, uint64_t>;  // (endpoint kind, stable ID)
    auto key_of = [](const swb_scene_attachment& a) -> Key {
        if (a.kind == SWB_ATTACH_SURFACE_VERTEX) return {SWB_ENDPOINT_SURFACE_ATTACHMENT, a.id};
        if (a.kind == SWB_ATTACH_JUNCTION) return {SWB_ENDPOINT_JUNCTION, a.junction_id};
        return {SWB_ENDPOINT_PILOT_HARNESS, a.id};
    };
    using Neighbor = std::pair<Key, const swb_scene_line*>;
    std::map<Key, std::vector<Neighbor>> adjacency;
    std::set<std::pair<Key, Key>> pairs;
    for (const auto* l : lines) {
        const Key a = key_of(*attachments.at(l->start_attachment_id));
        const Key b = key_of(*attachments.at(l->end_attachment_id));
        const auto canonical = a < b ? std::pair{a, b} : std::pair{b, a};
        if (a == b || !pairs.insert(canonical).second) {
            add(kUnsupportedSuspension, kSuspensionLine, l->id,
                "suspension tree contains a self-edge or duplicate endpoint pair");
            continue;
        }
        adjacency[a].push_back({b, l});
        adjacency[b].push_back({a, l});
    }
    for (auto& [endpoint, neighbors] : adjacency) {
        std::sort(neighbors.begin(), neighbors.end(), [](const Neighbor& x, const Neighbor& y) {
            return std::tuple{x.first.first, x.first.second, x.second->id} <
                   std::tuple{y.first.first, y.first.second, y.second->id};
        });
        if (endpoint.first == SWB_ENDPOINT_SURFACE_ATTACHMENT && neighbors.size() != 1)
            add(kUnsupportedSuspension, kAttachment, endpoint.second, "surface suspension attachment must be a tree leaf");
        if (endpoint.first == SWB_ENDPOINT_JUNCTION) {
            const auto* j = junctions.at(endpoint.second);
            if (j->fixed || neighbors.size() < 2)
                add(kUnsupportedSuspension, kSuspensionJunction, j->id,
                    j->fixed ? "pilot suspension junction must be dynamic"
                             : "pilot suspension junction cannot be a terminal leaf");
        }
    }
    if (!diags.empty()) return;
    std::set<Key> visited;
    std::map<uint64_t, std::pair<Key, Key>> oriented;  // line -> (from leaf side, to root side)
    for (const auto& [start, unused] : adjacency) {
        (void)unused;
        if (visited.count(start)) continue;
        std::vector<Key> component;
        std::queue<Key> pending;
        pending.push(start);
        visited.insert(start);
        size_t degree = 0;
        while (!pending.empty()) {
            const Key cur = pending.front();
            pending.pop();
            component.push_back(cur);
            degree += adjacency.at(cur).size();
            for (const auto& nb : adjacency.at(cur))
                if (visited.insert(nb.first).second) pending.push(nb.first);
        }
        std::vector<Key> roots;
        size_t leaves = 0;
        for (const Key& e : component) {
            if (e.first == SWB_ENDPOINT_PILOT_HARNESS) roots.push_back(e);
            else if (e.first == SWB_ENDPOINT_SURFACE_ATTACHMENT) ++leaves;
        }
        if (roots.size() != 1 || leaves == 0 || degree / 2 != component.size() - 1) {
            add(kUnsupportedSuspension, kSuspensionLine, lines.front()->id,
                "each suspension component must be an acyclic tree with one harness root and at least one surface "
                "leaf");
            continue;
        }
        std::set<Key> rooted{roots.front()};
        std::queue<Key> outward;
        outward.push(roots.front());
        while (!outward.empty()) {
            const Key parent = outward.front();
            outward.pop();
            for (const auto& nb : adjacency.at(parent)) {
                if (!rooted.insert(nb.first).second) continue;
                oriented.emplace(nb.second->id, std::pair{nb.first, parent});
                outward.push(nb.first);
            }
        }
    }
    if (!diags.empty() || oriented.size() != lines.size()) {
        if (diags.empty())
            add(kUnsupportedSuspension, kSuspensionLine, lines.front()->id,
                "suspension tree could not be oriented toward the pilot");
        return;
    }
    swb_suspension_def& sp = def.suspension;
    std::memset(&sp, 0, sizeof sp);
    sp.pilot_stable_id = pilot.id;
    sp.pilot_mass = pilot.mass;
    sp.pilot_initial_com_world = pilot.center_of_mass;
    sp.pilot_initial_linear_velocity = pilot.linear_velocity;
    sp.pilot_initial_body_to_world = pilot.body_to_world;
    sp.pilot_principal_inertia = pilot.principal_inertia;
    sp.solver_iterations = st.suspension_solver_iterations;
    sp.attachment_tolerance = st.suspension_attachment_tolerance;
    sp.minimum_line_length = st.suspension_minimum_line_length;
    sp.maximum_line_residual = st.suspension_maximum_line_residual;
    sp.maximum_control_work = st.suspension_maximum_control_work;
    for (const auto& [endpoint, unused] : adjacency) {
        (void)unused;
        if (endpoint.first == SWB_ENDPOINT_SURFACE_ATTACHMENT) {
            def.attachments.push_back({endpoint.second, node.at(attachments.at(endpoint.second)->vertex_id)});
        } else if (endpoint.first == SWB_ENDPOINT_JUNCTION) {
            def.junctions.push_back({endpoint.second, node.at(endpoint.second)});
        } else {
            const auto* a = attachments.at(endpoint.second);
            if (a->pilot_id != pilot.id) {
                add(kUnsupportedHarness, kAttachment, a->id, "harness root belongs to a different pilot");
                continue;
            }
            def.harness.push_back({endpoint.second, a->pilot_local_position});
        }
    }
    for (const auto* l : lines) {
        const auto& o = oriented.at(l->id);
        swb_suspension_segment g{};
        g.stable_id = l->id;
        g.from = {o.first.first, 0, o.first.second};
        g.to = {o.second.first, 0, o.second.second};
        g.rest_length = l->rest_length;
        g.axial_stiffness = line_materials.at(l->material_id)->axial_stiffness;
        g.axial_damping = 0.0;
        g.role = l->role;
        def.segments.push_back(g);
    }
    if (diags.empty()) def.has_suspension = true;
}

void Assembler::run() {
    validate();
    if (!diags.empty()) return;
    if (!check_bounds()) return;
    if (!(st.seam_coincidence_tolerance >= 0.0) || !std::isfinite(st.seam_coincidence_tolerance))
        add(kUnsupportedSeam, kScene, 0, "invalid seam coincidence tolerance");
    if (st.suspension_solver_iterations <= 0 || !(st.suspension_attachment_tolerance > 0.0) ||
        !std::isfinite(st.suspension_attachment_tolerance) || !(st.suspension_minimum_line_length > 0.0) ||
        !std::isfinite(st.suspension_minimum_line_length) || st.suspension_maximum_line_residual < 0.0 ||
        !std::isfinite(st.suspension_maximum_line_residual) || st.suspension_maximum_control_work < 0.0 ||
        !std::isfinite(st.suspension_maximum_control_work))
        add(kUnsupportedSuspension, kScene, 0, "invalid suspension solver settings");
    if (st.has_fabric_self_contact) {
        const swb_fabric_contact_def& c = st.fabric_self_contact;
        if (!(c.half_thickness > 0.0) || !std::isfinite(c.half_thickness) || c.normal_compliance < 0.0 ||
            !std::isfinite(c.normal_compliance) || c.static_friction < 0.0 || !std::isfinite(c.static_friction) ||
            c.dynamic_friction < 0.0 || !std::isfinite(c.dynamic_friction) || c.dynamic_friction > c.static_friction)
            add(kMaterialIncompatible, kScene, 0, "invalid explicit fabric contact settings");
    }
    const auto pilots = by_id(s.pilots, s.pilot_count);
    if (pilots.size() > 1)
        for (const auto* p : pilots)
            add(kUnsupportedPilot, kPilot, p->id, "one Structure instance supports exactly one rigid pilot");
    std::set<uint64_t> fabric_vertices;
    for (uint64_t i = 0; i < s.triangle_count; ++i)
        fabric_vertices.insert(s.triangles[i].vertex_ids, s.triangles[i].vertex_ids + 3);
    for (const auto* m : by_id(s.seams, s.seam_count)) {
        bool reported = false;
        for (uint64_t begin : {m->first_begin, m->second_begin})
            for (uint64_t i = 0; i < m->count && !reported; ++i)
                if (!fabric_vertices.count(s.seam_vertex_ids[begin + i])) {
                    add(kUnsupportedSeam, kSeam, m->id, "seam vertices must belong to fabric triangles");
                    reported = true;
                }
    }
    std::map<uint64_t, const swb_scene_attachment*> attachments;
    for (uint64_t i = 0; i < s.attachment_count; ++i) attachments.emplace(s.attachments[i].id, &s.attachments[i]);
    const auto lines = by_id(s.lines, s.line_count);
    auto node_id_of = [](const swb_scene_attachment& a) {
        return a.kind == SWB_ATTACH_SURFACE_VERTEX ? a.vertex_id : a.junction_id;
    };
    for (const auto* l : lines) {
        const auto* a = attachments.at(l->start_attachment_id);
        const auto* b = attachments.at(l->end_attachment_id);
        if (pilots.empty() && (a->kind == SWB_ATTACH_PILOT_HARNESS || b->kind == SWB_ATTACH_PILOT_HARNESS))
            add(kUnsupportedSuspension, kSuspensionLine, l->id, "a pilot harness line requires exactly one rigid pilot");
        else if (a->kind != SWB_ATTACH_PILOT_HARNESS && b->kind != SWB_ATTACH_PILOT_HARNESS && a->kind == b->kind &&
                 node_id_of(*a) == node_id_of(*b))
            add(kUnsupportedSuspension, kSuspensionLine, l->id,
                "suspension line endpoints must be distinct structural nodes");
    }
    if (!diags.empty()) return;

    // nodes: vertices of triangles and surface attachments, then junctions
    std::set<uint64_t> structural = fabric_vertices;
    for (uint64_t i = 0; i < s.attachment_count; ++i)
        if (s.attachments[i].kind == SWB_ATTACH_SURFACE_VERTEX) structural.insert(s.attachments[i].vertex_id);
    std::map<uint64_t, uint64_t> node;
    std::map<uint64_t, const swb_scene_vertex*> vertices;
    for (const auto* v : by_id(s.vertices, s.vertex_count)) {
        if (!structural.count(v->id)) continue;
        node.emplace(v->id, def.nodes.size());
        vertices.emplace(v->id, v);
        swb_node_def n{};
        n.position = v->position;
        def.nodes.push_back(n);
    }
    const size_t vertex_nodes = def.nodes.size();
    for (const auto* j : by_id(s.junctions, s.junction_count)) {
        node.emplace(j->id, def.nodes.size());
        swb_node_def n{};
        n.position = j->position;
        n.mass = j->mass;
        n.fixed = j->fixed ? 1u : 0u;
        def.nodes.push_back(n);
    }
    std::map<uint64_t, const swb_scene_fabric*> materials;
    for (const auto* m : by_id(s.fabrics, s.fabric_count)) {
        materials.emplace(m->id, m);
        if (!compatible_material(*m))
            add(kMaterialIncompatible, kFabricMaterial, m->id,
                "fabric stiffness is too ill-conditioned for the XPBD membrane inverse");
    }
    std::vector<long double> lumped(vertex_nodes, 0.0L);
    const auto triangles = by_id(s.triangles, s.triangle_count);
    for (const auto* t : triangles) {
        if (!compatible_chart(*t)) {
            add(kDegenerateChart, kTriangle, t->id, "triangle material coordinates are singular or ill-conditioned");
            continue;
        }
        swb_triangle_def tri{};
        for (int k = 0; k < 3; ++k) tri.nodes[k] = node.at(t->vertex_ids[k]);
        const uint64_t index = def.triangles.size();
        def.triangles.push_back(tri);
        const swb_scene_fabric& mat = *materials.at(t->material_id);
        swb_membrane_def m{};
        m.triangle = index;
        for (int k = 0; k < 3; ++k) {
            m.chart[k][0] = t->chart[k][0];
            m.chart[k][1] = t->chart[k][1];
        }
        m.material.warp_stiffness = mat.warp_stiffness;
        m.material.weft_stiffness = mat.weft_stiffness;
        m.material.coupling_stiffness = 0.0;
        m.material.shear_stiffness = mat.shear_stiffness;
        m.material.warp_pretension = 0.0;
        m.material.weft_pretension = 0.0;
        m.material.damping_seconds = mat.damping_seconds;
        m.material.compression_stiffness_ratio = 1.0;
        m.role = SWB_ROLE_BULK;
        def.membranes.push_back(m);
        const double mass = chart_area(*t) * mat.areal_density;
        if (!(mass > 0.0) || !std::isfinite(mass)) {
            add(kMappingOverflow, kTriangle, t->id, "triangle fabric mass is non-finite or underflows to zero");
            continue;
        }
        const long double share = static_cast<long double>(mass) / 3.0L;
        for (int k = 0; k < 3; ++k) lumped[tri.nodes[k]] += share;
        fabric_mass += static_cast<long double>(mass);
    }
    if (diags.empty()) bending(triangles, vertices, materials, node);
    std::map<uint64_t, const swb_scene_line_material*> line_materials;
    for (uint64_t i = 0; i < s.line_material_count; ++i)
        line_materials.emplace(s.line_materials[i].id, &s.line_materials[i]);
    if (pilots.empty()) {
        for (const auto* l : lines) {
            const auto* a = attachments.at(l->start_attachment_id);
            const auto* b = attachments.at(l->end_attachment_id);
            const auto* mat = line_materials.at(l->material_id);
            const double compliance = l->rest_length / mat->axial_stiffness;
            if (!std::isfinite(compliance) || compliance < 0.0) {
                add(kMaterialIncompatible, kLineMaterial, mat->id,
                    "line stiffness cannot be represented as finite XPBD compliance");
                continue;
            }
            swb_constraint_def k{};
            k.kind = SWB_CONSTRAINT_CABLE;
            k.first_node = node.at(node_id_of(*a));
            k.second_node = node.at(node_id_of(*b));
            k.rest_length = l->rest_length;
            k.compliance = compliance;
            def.constraints.push_back(k);
        }
    } else if (pilots.size() == 1) {
        pilot_suspension(*pilots.front(), node, line_materials);
    }
    if (diags.empty()) seams(vertices, node, lumped);
    for (size_t i = 0; i < lumped.size(); ++i) {
        const double mass = static_cast<double>(lumped[i]);
        if (!(mass > 0.0) || !std::isfinite(mass)) {
            uint64_t id = 0;
            for (const auto& [vid, n] : node)
                if (n == i) id = vid;
            add(kZeroMassNode, kVertex, id, "scene vertex has no finite positive lumped fabric or seam mass");
        } else {
            def.nodes[i].mass = mass;
        }
    }
    if (st.has_fabric_self_contact) {
        def.has_contact = true;
        def.contact = st.fabric_self_contact;
    }
    if (!std::isfinite(static_cast<double>(fabric_mass)))
        add(kMappingOverflow, kScene, 0, "total fabric mass exceeds the representable structure range");
    if (!std::isfinite(static_cast<double>(seam_mass)))
        add(kMappingOverflow, kScene, 0, "total seam mass exceeds the representable structure range");
}

}  // namespace
}  // namespace swb

using namespace swb;

extern "C" {

void swb_default_scene_settings(swb_scene_settings* out) {
    if (!out) return;
    std::memset(out, 0, sizeof(*out));
    out->seam_coincidence_tolerance = 1.0e-9;
    out->suspension_solver_iterations = 12;
    out->suspension_attachment_tolerance = 1.0e-10;
    out->suspension_minimum_line_length = 1.0e-10;
    out->suspension_maximum_line_residual = 2.0e-4;
    out->suspension_maximum_control_work = 1.0e6;
}

swb_status swb_assemble_scene(const swb_scene* scene, const swb_scene_settings* settings, swb_definition** out,
                              swb_scene_report* report) {
    return guarded([&] {
        if (!scene || !out) raise(SWB_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        auto ptr_ok = [](uint64_t n, const void* p) { return n == 0 || p != nullptr; };
        if (!ptr_ok(scene->vertex_count, scene->vertices) || !ptr_ok(scene->fabric_count, scene->fabrics) ||
            !ptr_ok(scene->triangle_count, scene->triangles) ||
            !ptr_ok(scene->seam_material_count, scene->seam_materials) || !ptr_ok(scene->seam_count, scene->seams) ||
            !ptr_ok(scene->seam_vertex_id_count, scene->seam_vertex_ids) ||
            !ptr_ok(scene->line_material_count, scene->line_materials) ||
            !ptr_ok(scene->pilot_count, scene->pilots) || !ptr_ok(scene->junction_count, scene->junctions) ||
            !ptr_ok(scene->attachment_count, scene->attachments) || !ptr_ok(scene->line_count, scene->lines))
            raise(SWB_INVALID_ARGUMENT, "null scene array");
        swb_scene_settings defaults;
        swb_default_scene_settings(&defaults);
        Assembler a{*scene, settings ? *settings : defaults, {}, {}};
        a.run();
        std::stable_sort(a.diags.begin(), a.diags.end(), [](const Diag& x, const Diag& y) {
            return std::tie(x.kind, x.id, x.code, x.validation, x.message) <
                   std::tie(y.kind, y.id, y.code, y.validation, y.message);
        });
        if (report) {
            std::memset(report, 0, sizeof(*report));
            report->diagnostic_count = static_cast<uint32_t>(a.diags.size());
            if (!a.diags.empty()) {
                const Diag& d = a.diags.front();
                report->first_code = d.code;
                report->first_validation_code = d.validation;
                report->first_entity_kind = d.kind;
                report->first_entity_id = d.id;
                std::snprintf(report->first_message, sizeof report->first_message, "%s", d.message.c_str());
            } else {
                report->assembled = 1;
                report->total_fabric_mass = static_cast<double>(a.fabric_mass);
                report->total_seam_mass = static_cast<double>(a.seam_mass);
            }
        }
        if (!a.diags.empty()) raise(SWB_INVALID_ARGUMENT, "scene assembly refused: " + a.diags.front().message);
        auto* def = new swb_definition;
        def->def = std::move(a.def);
        def->def.sync_view();
        *out = def;
    });
}

}  // extern "C"
