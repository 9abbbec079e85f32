// Definition layer: owned copies, validation and fingerprint of the
// StructureDefinition-shaped input, and the reference colouring.
#include "common.h"

#include <algorithm>
#include <bit>
#include <cmath>
#include <cstring>
#include <string>

namespace swb {

thread_local std::string g_last_error;

thread_local swb_error_detail g_last_detail{};

void set_last_error(const std::string& message) {
    g_last_error = message;
    g_last_detail = swb_error_detail{};
}

void set_last_error_detail(const swb_error_detail* detail) {
    g_last_detail = detail ? *detail : swb_error_detail{};
}

void OwnedDefinition::assign(const swb_structure_definition& s) {
    if ((s.node_count && !s.nodes) || (s.triangle_count && !s.triangles) ||
        (s.constraint_count && !s.constraints) ||
        (s.membrane_count && !s.membranes) ||
        (s.dihedral_count && !s.dihedrals))
        raise(SWB_INVALID_ARGUMENT, "definition array pointer is null");
    nodes.assign(s.nodes, s.nodes + s.node_count);
    triangles.assign(s.triangles, s.triangles + s.triangle_count);
    constraints.assign(s.constraints, s.constraints + s.constraint_count);
    membranes.assign(s.membranes, s.membranes + s.membrane_count);
    dihedrals.assign(s.dihedrals, s.dihedrals + s.dihedral_count);
    has_contact = s.fabric_self_contact != nullptr;
    if (has_contact) contact = *s.fabric_self_contact;
    has_suspension = s.suspension != nullptr;
    if (has_suspension) {
        const swb_suspension_def& p = *s.suspension;
        suspension = p;
        if ((p.attachment_count && !p.attachments) ||
            (p.junction_count && !p.junctions) ||
            (p.harness_count && !p.harness_points) ||
            (p.segment_count && !p.segments))
            raise(SWB_INVALID_ARGUMENT, "suspension array pointer is null");
        attachments.assign(p.attachments, p.attachments + p.attachment_count);
        junctions.assign(p.junctions, p.junctions + p.junction_count);
        harness.assign(p.harness_points, p.harness_points + p.harness_count);
        segments.assign(p.segments, p.segments + p.segment_count);
    }
    sync_view();
}

void OwnedDefinition::sync_view() {
    view.node_count = nodes.size();
    view.nodes = nodes.data();
    view.triangle_count = triangles.size();
    view.triangles = triangles.data();
    view.constraint_count = constraints.size();
    view.constraints = constraints.data();
    view.membrane_count = membranes.size();
    view.membranes = membranes.data();
    view.dihedral_count = dihedrals.size();
    view.dihedrals = dihedrals.data();
    view.fabric_self_contact = has_contact ? &contact : nullptr;
    if (has_suspension) {
        suspension.attachment_count = attachments.size();
        suspension.attachments = attachments.data();
        suspension.junction_count = junctions.size();
        suspension.junctions = junctions.data();
        suspension.harness_count = harness.size();
        suspension.harness_points = harness.data();
        suspension.segment_count = segments.size();
        suspension.segments = segments.data();
        view.suspension = &suspension;
    } else {
        view.suspension = nullptr;
    }
}

namespace {

bool finite3(const swb_vec3& v) {
    return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z);
}

void require_node(uint64_t index, uint64_t count, const char* entity) {
    if (index >= count)
        raise(SWB_INVALID_ARGUMENT,
              std::string(entity) + " references an unknown node");
}

// validateOrthotropicMembraneMaterial (membrane.cpp:298-326): finite
// entries, positive warp/weft/shear, non-negative coupling below the
// geometric mean, pre-tension in [0, 0.25), non-negative damping time,
// compression ratio in (0, 1].  The stiffness matrix diag(warp, weft, shear)
// with one off-diagonal coupling term is then SPD by construction of the
// previous inequalities.
void validate_material(const swb_membrane_material& m) {
    const double values[] = {m.warp_stiffness,   m.weft_stiffness,
                             m.coupling_stiffness, m.shear_stiffness,
                             m.warp_pretension,  m.weft_pretension,
                             m.damping_seconds,  m.compression_stiffness_ratio};
    for (double v : values)
        if (!std::isfinite(v))
            raise(SWB_INVALID_ARGUMENT, "Membrane material values must be finite");
    if (!(m.warp_stiffness > 0.0) || !(m.weft_stiffness > 0.0) ||
        !(m.shear_stiffness > 0.0) || m.coupling_stiffness < 0.0 ||
        !(m.coupling_stiffness * m.coupling_stiffness <
          m.warp_stiffness * m.weft_stiffness) ||
        m.warp_pretension < 0.0 || m.warp_pretension >= 0.25 ||
        m.weft_pretension < 0.0 || m.weft_pretension >= 0.25 ||
        m.damping_seconds < 0.0 || !(m.compression_stiffness_ratio > 0.0) ||
        m.compression_stiffness_ratio > 1.0)
        raise(SWB_INVALID_ARGUMENT, "Invalid orthotropic membrane material");
}

}  // namespace

// Structure's validateDefinition (src/fsi/structure.cpp:102-291).
void validate_definition(const swb_structure_definition& d) {
    for (uint64_t i = 0; i < d.node_count; ++i) {
        const swb_node_def& n = d.nodes[i];
        if (!finite3(n.position) || !std::isfinite(n.mass) || n.mass < 0.0 ||
            (!n.fixed && !(n.mass > 0.0)))
            raise(SWB_INVALID_ARGUMENT, "Invalid structure node definition");
    }
    for (uint64_t i = 0; i < d.triangle_count; ++i) {
        const swb_triangle_def& t = d.triangles[i];
        for (uint64_t n : t.nodes) require_node(n, d.node_count, "Triangle");
        if (t.nodes[0] == t.nodes[1] || t.nodes[1] == t.nodes[2] ||
            t.nodes[2] == t.nodes[0])
            raise(SWB_INVALID_ARGUMENT, "Triangle repeats a node");
        if (!std::isfinite(t.pressure_difference))
            raise(SWB_INVALID_ARGUMENT, "Triangle pressure must be finite");
    }
    for (uint64_t i = 0; i < d.constraint_count; ++i) {
        const swb_constraint_def& c = d.constraints[i];
        require_node(c.first_node, d.node_count, "Constraint");
        require_node(c.second_node, d.node_count, "Constraint");
        if (c.first_node == c.second_node || !std::isfinite(c.rest_length) ||
            c.rest_length < 0.0 || !std::isfinite(c.compliance) ||
            c.compliance < 0.0)
            raise(SWB_INVALID_ARGUMENT, "Invalid structure constraint");
        switch (c.kind) {
        case SWB_CONSTRAINT_DISTANCE:
        case SWB_CONSTRAINT_CABLE:
        case SWB_CONSTRAINT_SUSPENSION_TIE:
            break;
        case SWB_CONSTRAINT_SEAM_STITCH:
            if (c.rest_length != 0.0 || c.compliance != 0.0)
                raise(SWB_INVALID_ARGUMENT,
                      "Seam stitch must be rigid and zero-rest");
            break;
        default:
            raise(SWB_INVALID_ARGUMENT, "Unknown structure constraint kind");
        }
    }
    for (uint64_t i = 0; i < d.membrane_count; ++i) {
        const swb_membrane_def& m = d.membranes[i];
        if (m.triangle >= d.triangle_count)
            raise(SWB_INVALID_ARGUMENT, "Membrane references an unknown triangle");
        for (int k = 0; k < 3; ++k)
            if (!std::isfinite(m.chart[k][0]) || !std::isfinite(m.chart[k][1]))
                raise(SWB_INVALID_ARGUMENT,
                      "Membrane material coordinates must be finite");
        validate_material(m.material);
        if (m.role < SWB_ROLE_BULK || m.role > SWB_ROLE_REINFORCEMENT)
            raise(SWB_INVALID_ARGUMENT, "Unknown structure material role");
    }
    for (uint64_t i = 0; i < d.dihedral_count; ++i) {
        const swb_dihedral_def& h = d.dihedrals[i];
        for (uint64_t n : h.nodes) require_node(n, d.node_count, "Dihedral");
        uint64_t u[4] = {h.nodes[0], h.nodes[1], h.nodes[2], h.nodes[3]};
        std::sort(u, u + 4);
        if (u[0] == u[1] || u[1] == u[2] || u[2] == u[3] ||
            !std::isfinite(h.rest_angle) || !std::isfinite(h.compliance) ||
            h.compliance < 0.0)
            raise(SWB_INVALID_ARGUMENT, "Invalid dihedral definition");
    }
    if (d.fabric_self_contact) {
        const swb_fabric_contact_def& c = *d.fabric_self_contact;
        if (d.triangle_count == 0 || !std::isfinite(c.half_thickness) ||
            !(c.half_thickness > 0.0) || !std::isfinite(c.normal_compliance) ||
            c.normal_compliance < 0.0 || !std::isfinite(c.static_friction) ||
            c.static_friction < 0.0 || !std::isfinite(c.dynamic_friction) ||
            c.dynamic_friction < 0.0 || c.dynamic_friction > c.static_friction)
            raise(SWB_INVALID_ARGUMENT,
                  "Invalid structure fabric self-contact definition");
    }
    if (d.suspension) {
        const swb_suspension_def& s = *d.suspension;
        auto unique_ids = [](auto begin, auto end, const char* label) {
            std::vector<uint64_t> ids;
            for (auto it = begin; it != end; ++it) {
                if (it->stable_id == 0)
                    raise(SWB_INVALID_ARGUMENT,
                          std::string(label) + " stable ID must be nonzero");
                ids.push_back(it->stable_id);
            }
            std::sort(ids.begin(), ids.end());
            if (std::adjacent_find(ids.begin(), ids.end()) != ids.end())
                raise(SWB_INVALID_ARGUMENT,
                      std::string(label) + " stable IDs must be unique");
        };
        const double qw = s.pilot_initial_body_to_world.w,
                     qx = s.pilot_initial_body_to_world.x,
                     qy = s.pilot_initial_body_to_world.y,
                     qz = s.pilot_initial_body_to_world.z;
        if (s.pilot_stable_id == 0 || !(s.pilot_mass > 0.0) ||
            !std::isfinite(s.pilot_mass) || !finite3(s.pilot_com_local) ||
            !finite3(s.pilot_initial_com_world) ||
            !finite3(s.pilot_initial_linear_velocity) ||
            !finite3(s.pilot_initial_angular_velocity) || !std::isfinite(qw) ||
            !std::isfinite(qx) || !std::isfinite(qy) || !std::isfinite(qz) ||
            !(s.pilot_principal_inertia.x > 0.0) ||
            !(s.pilot_principal_inertia.y > 0.0) ||
            !(s.pilot_principal_inertia.z > 0.0) ||
            !finite3(s.pilot_principal_inertia) || s.attachment_count == 0 ||
            s.harness_count == 0 || s.segment_count == 0 ||
            s.solver_iterations <= 0 || !(s.attachment_tolerance > 0.0) ||
            !std::isfinite(s.attachment_tolerance) ||
            !(s.minimum_line_length > 0.0) ||
            !std::isfinite(s.minimum_line_length) ||
            s.maximum_line_residual < 0.0 ||
            !std::isfinite(s.maximum_line_residual) ||
            s.maximum_control_work < 0.0 || !std::isfinite(s.maximum_control_work))
            raise(SWB_INVALID_ARGUMENT, "Invalid structure suspension definition");
        unique_ids(s.attachments, s.attachments + s.attachment_count,
                   "Suspension attachment");
        unique_ids(s.junctions, s.junctions + s.junction_count,
                   "Suspension junction");
        unique_ids(s.harness_points, s.harness_points + s.harness_count,
                   "Pilot harness");
        unique_ids(s.segments, s.segments + s.segment_count,
                   "Suspension segment");
        for (uint64_t i = 0; i < s.attachment_count; ++i)
            require_node(s.attachments[i].node, d.node_count,
                         "Suspension attachment");
        for (uint64_t i = 0; i < s.junction_count; ++i) {
            require_node(s.junctions[i].node, d.node_count, "Suspension junction");
            if (d.nodes[s.junctions[i].node].fixed)
                raise(SWB_INVALID_ARGUMENT,
                      "Suspension junction must be a dynamic node");
        }
        for (uint64_t i = 0; i < s.harness_count; ++i)
            if (!finite3(s.harness_points[i].local_position))
                raise(SWB_INVALID_ARGUMENT, "Pilot harness position must be finite");
        for (uint64_t i = 0; i < s.segment_count; ++i) {
            const swb_suspension_segment& g = s.segments[i];
            if (g.from.stable_id == 0 || g.to.stable_id == 0 ||
                (g.from.kind == g.to.kind && g.from.stable_id == g.to.stable_id) ||
                !(g.rest_length > 0.0) || !std::isfinite(g.rest_length) ||
                !(g.axial_stiffness > 0.0) || !std::isfinite(g.axial_stiffness) ||
                g.axial_damping < 0.0 || !std::isfinite(g.axial_damping))
                raise(SWB_INVALID_ARGUMENT, "Invalid structure suspension segment");
        }
    }
}

namespace {

// FNV-1a over little-endian bytes (structure.cpp:293-324).
struct Fnv {
    uint64_t value = 14695981039346656037ULL;
    void add(uint64_t v) {
        for (int byte = 0; byte < 8; ++byte) {
            value ^= static_cast<uint8_t>(v & 0xffU);
            value *= 1099511628211ULL;
            v >>= 8U;
        }
    }
    void add(double v) { add(std::bit_cast<uint64_t>(v)); }
    void add(const swb_vec3& v) { add(v.x); add(v.y); add(v.z); }
};

}  // namespace

// computeDefinitionFingerprint (structure.cpp:326-420).  The per-face
// pressure, which the reference definition does not carry, is hashed after
// the triangles only when some face has one, so pressure-free definitions
// keep the reference value.
uint64_t definition_fingerprint(const swb_structure_definition& d) {
    Fnv h;
    h.add(uint64_t{2});
    h.add(d.node_count);
    for (uint64_t i = 0; i < d.node_count; ++i) {
        const swb_node_def& n = d.nodes[i];
        h.add(n.position.x); h.add(n.position.y); h.add(n.position.z);
        h.add(n.mass);
        h.add(n.fixed ? uint64_t{1} : uint64_t{0});
    }
    h.add(d.triangle_count);
    bool pressure = false;
    for (uint64_t i = 0; i < d.triangle_count; ++i) {
        for (uint64_t n : d.triangles[i].nodes) h.add(n);
        pressure = pressure || d.triangles[i].pressure_difference != 0.0;
    }
    if (pressure)
        for (uint64_t i = 0; i < d.triangle_count; ++i)
            h.add(d.triangles[i].pressure_difference);
    h.add(d.constraint_count);
    for (uint64_t i = 0; i < d.constraint_count; ++i) {
        const swb_constraint_def& c = d.constraints[i];
        h.add(uint64_t{c.kind});
        h.add(c.first_node);
        h.add(c.second_node);
        h.add(c.rest_length);
        h.add(c.compliance);
    }
    h.add(d.membrane_count);
    for (uint64_t i = 0; i < d.membrane_count; ++i) {
        const swb_membrane_def& m = d.membranes[i];
        h.add(m.triangle);
        for (int k = 0; k < 3; ++k) { h.add(m.chart[k][0]); h.add(m.chart[k][1]); }
        h.add(m.material.warp_stiffness);
        h.add(m.material.weft_stiffness);
        h.add(m.material.coupling_stiffness);
        h.add(m.material.shear_stiffness);
        h.add(m.material.warp_pretension);
        h.add(m.material.weft_pretension);
        h.add(m.material.damping_seconds);
        h.add(m.material.compression_stiffness_ratio);
        h.add(uint64_t{m.role});
    }
    h.add(d.dihedral_count);
    for (uint64_t i = 0; i < d.dihedral_count; ++i) {
        const swb_dihedral_def& g = d.dihedrals[i];
        for (uint64_t n : g.nodes) h.add(n);
        h.add(g.rest_angle);
        h.add(g.compliance);
    }
    h.add(d.fabric_self_contact ? uint64_t{1} : uint64_t{0});
    if (d.fabric_self_contact) {
        h.add(d.fabric_self_contact->half_thickness);
        h.add(d.fabric_self_contact->normal_compliance);
        h.add(d.fabric_self_contact->static_friction);
        h.add(d.fabric_self_contact->dynamic_friction);
    }
    h.add(d.suspension ? uint64_t{1} : uint64_t{0});
    if (d.suspension) {
        const swb_suspension_def& s = *d.suspension;
        h.add(s.pilot_stable_id);
        h.add(s.pilot_mass);
        h.add(s.pilot_com_local);
        h.add(s.pilot_initial_com_world);
        h.add(s.pilot_initial_linear_velocity);
        h.add(s.pilot_initial_angular_velocity);
        h.add(s.pilot_initial_body_to_world.w);
        h.add(s.pilot_initial_body_to_world.x);
        h.add(s.pilot_initial_body_to_world.y);
        h.add(s.pilot_initial_body_to_world.z);
        h.add(s.pilot_principal_inertia);
        h.add(s.attachment_count);
        for (uint64_t i = 0; i < s.attachment_count; ++i) {
            h.add(s.attachments[i].stable_id);
            h.add(s.attachments[i].node);
        }
        h.add(s.junction_count);
        for (uint64_t i = 0; i < s.junction_count; ++i) {
            h.add(s.junctions[i].stable_id);
            h.add(s.junctions[i].node);
        }
        h.add(s.harness_count);
        for (uint64_t i = 0; i < s.harness_count; ++i) {
            h.add(s.harness_points[i].stable_id);
            h.add(s.harness_points[i].local_position);
        }
        h.add(s.segment_count);
        for (uint64_t i = 0; i < s.segment_count; ++i) {
            const swb_suspension_segment& g = s.segments[i];
            h.add(g.stable_id);
            h.add(uint64_t{g.from.kind});
            h.add(g.from.stable_id);
            h.add(uint64_t{g.to.kind});
            h.add(g.to.stable_id);
            h.add(g.rest_length);
            h.add(g.axial_stiffness);
            h.add(g.axial_damping);
            h.add(uint64_t{g.role});
        }
        h.add(static_cast<uint64_t>(static_cast<int64_t>(s.solver_iterations)));
        h.add(s.attachment_tolerance);
        h.add(s.minimum_line_length);
        h.add(s.maximum_line_residual);
        h.add(s.maximum_control_work);
    }
    return h.value;
}

// SoftBody::constraintColouring (soft_body.cpp:1978-2075): greedy first fit
// over the line graph in insertion order with a per-node colour mask of
// ceil((2*maxDegree+1)/64) words, then colours ranked by descending size
// (ties by colour id); colours smaller than 1024 constraints at the tail are
// the serial remainder (kConstraintsPerBarrier, soft_body.cpp:1938).
ReferenceColouring reference_colouring(uint64_t node_count,
                                       const std::vector<uint32_t>& a,
                                       const std::vector<uint32_t>& b) {
    ReferenceColouring out;
    const size_t m = a.size();
    if (m == 0) return out;
    std::vector<uint64_t> degree(node_count, 0);
    for (size_t i = 0; i < m; ++i) { ++degree[a[i]]; ++degree[b[i]]; }
    const uint64_t max_degree = *std::max_element(degree.begin(), degree.end());
    const uint64_t bound = 2 * max_degree + 1;
    const uint64_t words = std::max<uint64_t>(1, (bound + 63) / 64);
    std::vector<uint64_t> mask(node_count * words, 0);
    std::vector<uint64_t> colour_of(m, 0);
    uint64_t colours = 0;
    for (size_t i = 0; i < m; ++i) {
        const uint64_t* ma = &mask[a[i] * words];
        const uint64_t* mb = &mask[b[i] * words];
        uint64_t colour = 0;
        for (uint64_t w = 0; w < words; ++w) {
            const uint64_t used = ma[w] | mb[w];
            if (used != ~uint64_t{0}) {
                colour = 64 * w + static_cast<uint64_t>(std::countr_one(used));
                break;
            }
            colour = 64 * (w + 1);
        }
        if (colour >= bound)
            raise(SWB_INVALID_ARGUMENT,
                  "Constraint colouring exceeded its degree bound");
        const uint64_t bit = uint64_t{1} << (colour % 64);
        mask[a[i] * words + colour / 64] |= bit;
        mask[b[i] * words + colour / 64] |= bit;
        colour_of[i] = colour;
        colours = std::max(colours, colour + 1);
    }
    std::vector<uint64_t> sizes(colours, 0);
    for (uint64_t c : colour_of) ++sizes[c];
    std::vector<uint64_t> by_size(colours);
    for (uint64_t c = 0; c < colours; ++c) by_size[c] = c;
    std::sort(by_size.begin(), by_size.end(), [&](uint64_t l, uint64_t r) {
        if (sizes[l] != sizes[r]) return sizes[l] > sizes[r];
        return l < r;
    });
    std::vector<uint64_t> rank(colours, 0);
    for (uint64_t r = 0; r < colours; ++r) rank[by_size[r]] = r;
    out.offsets.assign(colours + 1, 0);
    for (uint64_t r = 0; r < colours; ++r)
        out.offsets[r + 1] = out.offsets[r] + sizes[by_size[r]];
    out.order.assign(m, 0);
    std::vector<uint64_t> cursor(out.offsets.begin(), out.offsets.end() - 1);
    for (size_t i = 0; i < m; ++i) out.order[cursor[rank[colour_of[i]]]++] = i;
    uint64_t parallel = colours;
    while (parallel > 0 &&
           out.offsets[parallel] - out.offsets[parallel - 1] < 1024)
        --parallel;
    out.parallel_colours = parallel;
    return out;
}

}  // namespace swb

using namespace swb;

extern "C" {

const char* swb_last_error(void) { return swb::g_last_error.c_str(); }

swb_status swb_last_error_detail(swb_error_detail* out) {
    if (!out) return SWB_INVALID_ARGUMENT;
    *out = swb::g_last_detail;
    return SWB_OK;
}

uint32_t swb_abi_version(void) { return SWB_ABI_VERSION; }

void swb_default_step_settings(swb_step_settings* out) {
    std::memset(out, 0, sizeof(*out));
    out->time_step = 1.0 / 120.0;
    out->substeps = 2;
    out->constraint_iterations = 12;
    out->cable_sweep_pairs = 0;
    out->worker_threads = 0;
    out->gravity = {0.0, 0.0, -9.80665};
    out->velocity_damping = 0.25;
    out->damping_reference_velocity = {0.0, 0.0, 0.0};
}

swb_status swb_validate_definition(const swb_structure_definition* definition) {
    return guarded([&] {
        if (!definition) raise(SWB_INVALID_ARGUMENT, "definition is null");
        OwnedDefinition copy;
        copy.assign(*definition);
        validate_definition(copy.view);
    });
}

uint64_t swb_definition_fingerprint(const swb_structure_definition* definition) {
    return definition ? definition_fingerprint(*definition) : 0;
}

swb_status swb_definition_copy(const swb_structure_definition* source,
                               swb_definition** out) {
    return guarded([&] {
        if (!source || !out) raise(SWB_INVALID_ARGUMENT, "null argument");
        auto* d = new swb_definition;
        try {
            d->def.assign(*source);
        } catch (...) {
            delete d;
            throw;
        }
        *out = d;
    });
}

swb_status swb_definition_permute(swb_definition* definition,
                                  const uint64_t* constraint_order,
                                  const uint64_t* dihedral_order) {
    return guarded([&] {
        if (!definition) raise(SWB_INVALID_ARGUMENT, "definition is null");
        OwnedDefinition& d = definition->def;
        auto apply = [](auto& vec, const uint64_t* order) {
            if (!order) return;
            std::vector<uint8_t> seen(vec.size(), 0);
            auto copy = vec;
            for (size_t k = 0; k < vec.size(); ++k) {
                if (order[k] >= vec.size() || seen[order[k]])
                    raise(SWB_INVALID_ARGUMENT, "order is not a permutation");
                seen[order[k]] = 1;
                vec[k] = copy[order[k]];
            }
        };
        apply(d.constraints, constraint_order);
        apply(d.dihedrals, dihedral_order);
        d.sync_view();
    });
}

swb_status swb_definition_permute_membranes(swb_definition* definition, const uint64_t* membrane_order) {
    return guarded([&] {
        if (!definition) raise(SWB_INVALID_ARGUMENT, "definition is null");
        OwnedDefinition& d = definition->def;
        if (!membrane_order) return;
        std::vector<uint8_t> seen(d.membranes.size(), 0);
        const auto copy = d.membranes;
        for (size_t k = 0; k < d.membranes.size(); ++k) {
            if (membrane_order[k] >= copy.size() || seen[membrane_order[k]])
                raise(SWB_INVALID_ARGUMENT, "order is not a permutation");
            seen[membrane_order[k]] = 1;
            d.membranes[k] = copy[membrane_order[k]];
        }
        d.sync_view();
    });
}

swb_status swb_definition_set_contact(swb_definition* definition, const swb_fabric_contact_def* contact) {
    return guarded([&] {
        if (!definition) raise(SWB_INVALID_ARGUMENT, "definition is null");
        OwnedDefinition& d = definition->def;
        d.has_contact = contact != nullptr;
        d.contact = contact ? *contact : swb_fabric_contact_def{};
        d.sync_view();
    });
}

swb_status swb_definition_scale_rest(swb_definition* definition,
                                     uint64_t index, double factor) {
    return guarded([&] {
        if (!definition) raise(SWB_INVALID_ARGUMENT, "definition is null");
        OwnedDefinition& d = definition->def;
        if (index < d.constraints.size()) {
            if (d.constraints[index].kind == SWB_CONSTRAINT_SEAM_STITCH)
                raise(SWB_INVALID_ARGUMENT, "seam stitches are zero-rest");
            d.constraints[index].rest_length *= factor;
        } else if (d.has_suspension &&
                   index - d.constraints.size() < d.segments.size()) {
            d.segments[index - d.constraints.size()].rest_length *= factor;
        } else {
            raise(SWB_OUT_OF_RANGE, "rest-length index out of range");
        }
        d.sync_view();
    });
}

const swb_structure_definition* swb_definition_view(const swb_definition* d) {
    return d ? &d->def.view : nullptr;
}

void swb_definition_destroy(swb_definition* d) { delete d; }

swb_status swb_reference_colouring(const swb_structure_definition* definition,
                                   uint64_t* order, uint64_t* offsets,
                                   uint64_t offsets_capacity,
                                   uint64_t* colour_count,
                                   uint64_t* parallel_colours) {
    return guarded([&] {
        if (!definition || !order || !offsets || !colour_count ||
            !parallel_colours)
            raise(SWB_INVALID_ARGUMENT, "null argument");
        std::vector<uint32_t> a(definition->constraint_count),
            b(definition->constraint_count);
        for (uint64_t i = 0; i < definition->constraint_count; ++i) {
            if (definition->constraints[i].first_node >= definition->node_count ||
                definition->constraints[i].second_node >= definition->node_count)
                raise(SWB_INVALID_ARGUMENT, "constraint references an unknown node");
            a[i] = static_cast<uint32_t>(definition->constraints[i].first_node);
            b[i] = static_cast<uint32_t>(definition->constraints[i].second_node);
        }
        ReferenceColouring c =
            reference_colouring(definition->node_count, a, b);
        if (c.offsets.size() > offsets_capacity)
            raise(SWB_INVALID_ARGUMENT, "offsets capacity too small");
        std::copy(c.order.begin(), c.order.end(), order);
        std::copy(c.offsets.begin(), c.offsets.end(), offsets);
        *colour_count = c.offsets.empty() ? 0 : c.offsets.size() - 1;
        *parallel_colours = c.parallel_colours;
    });
}

}  // extern "C"
