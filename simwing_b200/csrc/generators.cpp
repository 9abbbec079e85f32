// Deterministic synthetic definitions: the hanging cloth patch and the
// ram-air wing with cascaded lines and a rigid pilot.  They are emitted the
// way the reference's scene assembly would (src/fsi/scene_structure.cpp):
//   * fabric mass lumped from each triangle's area equally to its three
//     vertices (scene_structure.h:134-137);
//   * one dihedral per consistently oriented two-triangle edge of one sheet,
//     canonical-edge order, signed rest angle from the authored geometry,
//     compliance h0/(2 D0 L0) + h1/(2 D1 L1) (assembleBending,
//     scene_structure.cpp:278-420);
//   * seams as rigid zero-rest SeamStitch pairs plus distance rails of
//     compliance 2L/EA on both chains (assembleSeams,
//     scene_structure.cpp:440-590);
//   * cable lines with compliance L/EA; a rigid pilot owning two riser
//     segments (assemblePilotSuspension, scene_structure.cpp:592-892).
// The edge distance constraints (one per unique triangle edge) follow the
// cloth construction of SoftBody::addRectangularPatch
// (soft_body.cpp:2589-2640).
#include "common.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

namespace swb {
namespace {

// splitmix64 stream with Box-Muller normals: a fixed, documented generator
// so the same seed yields the same definition on every platform.
struct Rng {
    uint64_t state;
    explicit Rng(uint64_t seed) : state(seed) {}
    uint64_t next() {
        uint64_t z = (state += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    double uniform() {  // (0, 1)
        return (static_cast<double>(next() >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    }
    double normal() {
        const double u1 = uniform(), u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

struct V { double x, y, z; };
V operator-(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V operator+(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V operator*(V a, double s) { return {a.x * s, a.y * s, a.z * s}; }
double dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V cross(V a, V b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
double length(V a) { return std::sqrt(dot(a, a)); }

struct Builder {
    OwnedDefinition& d;
    std::vector<V> design;      // authored (unjittered) positions
    std::vector<double> mass;

    explicit Builder(OwnedDefinition& def) : d(def) {}

    uint64_t node(V p, bool fixed = false) {
        design.push_back(p);
        mass.push_back(0.0);
        swb_node_def n{};
        n.position = {p.x, p.y, p.z};
        n.fixed = fixed ? 1u : 0u;
        d.nodes.push_back(n);
        return d.nodes.size() - 1;
    }
    void triangle(uint64_t a, uint64_t b, uint64_t c, double pressure,
                  double density) {
        swb_triangle_def t{};
        t.nodes[0] = a; t.nodes[1] = b; t.nodes[2] = c;
        t.pressure_difference = pressure;
        d.triangles.push_back(t);
        const double area =
            0.5 * length(cross(design[b] - design[a], design[c] - design[a]));
        const double share = density * area / 3.0;
        mass[a] += share; mass[b] += share; mass[c] += share;
    }
    void distance(uint32_t kind, uint64_t a, uint64_t b, double rest,
                  double compliance) {
        swb_constraint_def c{};
        c.kind = kind;
        c.first_node = a;
        c.second_node = b;
        c.rest_length = rest;
        c.compliance = compliance;
        d.constraints.push_back(c);
    }

    // One distance constraint per unique edge of triangles [first, last) in
    // triangle-major, corner order.
    void edge_constraints(size_t first, size_t last, double compliance) {
        std::map<std::pair<uint64_t, uint64_t>, bool> seen;
        for (size_t t = first; t < last; ++t)
            for (int k = 0; k < 3; ++k) {
                uint64_t a = d.triangles[t].nodes[k];
                uint64_t b = d.triangles[t].nodes[(k + 1) % 3];
                auto key = std::minmax(a, b);
                if (seen.emplace(key, true).second)
                    distance(SWB_CONSTRAINT_DISTANCE, a, b,
                             length(design[b] - design[a]), compliance);
            }
    }

    // One membrane element per triangle of [first, last): the chart is the
    // triangle's own rest shape in its plane, warp along `warp` projected
    // into the plane (so the element starts unstrained and its chart is
    // positively oriented).
    void membranes(size_t first, size_t last, V warp, const swb_membrane_material& material) {
        for (size_t t = first; t < last; ++t) {
            const V a = design[d.triangles[t].nodes[0]], b = design[d.triangles[t].nodes[1]],
                    c = design[d.triangles[t].nodes[2]];
            V n = cross(b - a, c - a);
            n = n * (1.0 / length(n));
            V u = warp - n * dot(warp, n);
            if (!(length(u) > 1e-9)) u = b - a;
            u = u * (1.0 / length(u));
            const V v = cross(n, u);
            swb_membrane_def m{};
            m.triangle = t;
            m.chart[0][0] = 0.0;
            m.chart[0][1] = 0.0;
            m.chart[1][0] = dot(b - a, u);
            m.chart[1][1] = dot(b - a, v);
            m.chart[2][0] = dot(c - a, u);
            m.chart[2][1] = dot(c - a, v);
            m.material = material;
            m.role = SWB_ROLE_BULK;
            d.membranes.push_back(m);
        }
    }

    // assembleBending for one sheet: triangles [first, last).  When
    // `fixed_compliance` >= 0 it replaces the series-strip formula.
    void dihedrals(size_t first, size_t last, double rigidity,
                   double fixed_compliance) {
        struct Inc { uint64_t from, to, opposite; };
        std::map<std::pair<uint64_t, uint64_t>, std::vector<Inc>> edges;
        for (size_t t = first; t < last; ++t)
            for (int k = 0; k < 3; ++k) {
                const uint64_t from = d.triangles[t].nodes[k];
                const uint64_t to = d.triangles[t].nodes[(k + 1) % 3];
                const uint64_t opp = d.triangles[t].nodes[(k + 2) % 3];
                edges[std::minmax(from, to)].push_back({from, to, opp});
            }
        for (const auto& [edge, inc] : edges) {
            if (inc.size() != 2) continue;
            const Inc& f = inc[0];
            const Inc& s = inc[1];
            if (f.from != s.to || f.to != s.from) continue;
            const V a = design[f.from], b = design[f.to];
            const V c = design[f.opposite], dd = design[s.opposite];
            const V e = b - a;
            const double el = length(e);
            const V A1 = cross(e, c - a), A2 = cross(dd - a, e);
            const double l1 = length(A1), l2 = length(A2);
            double compliance = fixed_compliance;
            if (compliance < 0.0) {
                const double h0 = l1 / el, h1 = l2 / el;
                compliance = h0 / (2.0 * rigidity * el) + h1 / (2.0 * rigidity * el);
            }
            const V eu = e * (1.0 / el), n1 = A1 * (1.0 / l1), n2 = A2 * (1.0 / l2);
            const double cosine = std::clamp(dot(n1, n2), -1.0, 1.0);
            const double sine = dot(eu, cross(n1, n2));
            swb_dihedral_def h{};
            h.nodes[0] = f.from; h.nodes[1] = f.to;
            h.nodes[2] = f.opposite; h.nodes[3] = s.opposite;
            h.rest_angle = std::atan2(sine, cosine);
            h.compliance = compliance;
            d.dihedrals.push_back(h);
        }
    }

    void finish_masses(double minimum) {
        for (size_t i = 0; i < d.nodes.size(); ++i)
            d.nodes[i].mass = std::max(mass[i], minimum);
    }
};

}  // namespace
}  // namespace swb

using namespace swb;

extern "C" {

void swb_default_patch_params(swb_patch_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->nx = 33;
    p->ny = 33;
    p->width = 1.0;
    p->height = 1.0;
    p->areal_density = 0.040;
    p->distance_compliance = 1.0e-7;
    p->bend_compliance = 1.0e-3;
    p->jitter = 1.0e-3;
    p->seed = 1;
    p->pin_top_corners = 1;
}

void swb_default_wing_params(swb_wing_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->cells = 40;
    p->chordwise = 60;
    p->spanwise_per_cell = 4;
    p->rib_layers = 10;
    p->span = 11.0;
    p->root_chord = 2.6;
    p->thickness = 0.15;
    p->areal_density = 0.045;
    p->skin_compliance = 1.0e-7;
    p->bend_rigidity = 1.0e-3;
    p->line_compliance_scale = 1.0;
    p->pressure = 30.0;
    p->line_levels = 4;
    p->line_particles = 8;
    p->line_rows = 4;
    p->pilot = 1;
    p->pilot_mass = 90.0;
    p->aspect_ratio = 0.0;
    p->compliance_jitter = 0.0;
    p->seed = 1;
}

// Hanging cloth patch: nx x ny particles on a width x height sheet in the
// x-z plane, triangulated like SoftBody::addRectangularPatch
// (soft_body.cpp:2622-2632), one distance constraint per unique triangle
// edge, one dihedral per interior edge (flat rest angle), area/3 lumped
// mass, the two top corners fixed, every coordinate jittered by N(0, jitter);
// optionally one membrane element per triangle.
swb_status swb_generate_patch(const swb_patch_params* p, swb_definition** out) {
    return guarded([&] {
        if (!p || !out) raise(SWB_INVALID_ARGUMENT, "null argument");
        if (p->nx < 2 || p->ny < 2 || !(p->width > 0) || !(p->height > 0) ||
            !(p->areal_density > 0) || p->distance_compliance < 0 ||
            p->bend_compliance < 0 || p->jitter < 0)
            raise(SWB_INVALID_ARGUMENT, "invalid patch parameters");
        auto* def = new swb_definition;
        try {
            Builder b(def->def);
            const double dx = p->width / (p->nx - 1);
            const double dz = p->height / (p->ny - 1);
            for (uint32_t j = 0; j < p->ny; ++j)
                for (uint32_t i = 0; i < p->nx; ++i) {
                    const bool top = j == p->ny - 1;
                    const bool corner = top && (i == 0 || i == p->nx - 1);
                    b.node({i * dx, 0.0, j * dz}, p->pin_top_corners && corner);
                }
            auto id = [&](uint32_t i, uint32_t j) { return uint64_t{j} * p->nx + i; };
            for (uint32_t j = 0; j + 1 < p->ny; ++j)
                for (uint32_t i = 0; i + 1 < p->nx; ++i) {
                    const uint64_t n00 = id(i, j), n01 = id(i + 1, j);
                    const uint64_t n10 = id(i, j + 1), n11 = id(i + 1, j + 1);
                    b.triangle(n00, n01, n11, 0.0, p->areal_density);
                    b.triangle(n00, n11, n10, 0.0, p->areal_density);
                }
            b.edge_constraints(0, def->def.triangles.size(), p->distance_compliance);
            b.dihedrals(0, def->def.triangles.size(), 0.0, p->bend_compliance);
            if (p->membranes > 2) raise(SWB_INVALID_ARGUMENT, "invalid patch membrane option");
            if (p->membranes) {
                // orthotropic fabric: warp along x, weft along z (N/m)
                swb_membrane_material m{};
                m.warp_stiffness = 2.0e4;
                m.weft_stiffness = 1.5e4;
                m.coupling_stiffness = 3.0e3;
                m.shear_stiffness = 2.0e3;
                m.compression_stiffness_ratio = 1.0;
                if (p->membranes == 2) {
                    m.warp_pretension = 1.0e-3;
                    m.weft_pretension = 5.0e-4;
                    m.damping_seconds = 2.0e-3;
                    m.compression_stiffness_ratio = 0.1;
                }
                for (uint64_t t = 0; t < def->def.triangles.size(); ++t) {
                    swb_membrane_def md{};
                    md.triangle = t;
                    for (int k = 0; k < 3; ++k) {
                        const uint64_t n = def->def.triangles[t].nodes[k];
                        md.chart[k][0] = static_cast<double>(n % p->nx) * dx;
                        md.chart[k][1] = static_cast<double>(n / p->nx) * dz;
                    }
                    md.material = m;
                    md.role = SWB_ROLE_BULK;
                    def->def.membranes.push_back(md);
                }
            }
            b.finish_masses(0.0);
            Rng rng(p->seed);
            for (auto& n : def->def.nodes) {
                n.position.x += p->jitter * rng.normal();
                n.position.y += p->jitter * rng.normal();
                n.position.z += p->jitter * rng.normal();
            }
            def->def.sync_view();
        } catch (...) {
            delete def;
            throw;
        }
        *out = def;
    });
}

// Ram-air wing.  Geometry: elliptical planform chord c0*sqrt(1-0.9*eta^2)
// along a circular arc (anhedral), quarter-chord line straight, closed
// symmetric 4-digit-style section of the given thickness, uniform chordwise
// stations (x = j / C; clustering them at the leading edge makes sliver
// triangles whose constraint solve is ill-conditioned).  The skin is one closed sheet (top and bottom share the leading
// and trailing edge), 2*chordwise quads around and cells*spanwise_per_cell
// quads across, oriented with outward right-hand normals and carrying the
// outward pressure jump.  Each of the cells+1 ribs is its own sheet meshed
// (chordwise-2) x rib_layers quads plus leading/trailing fans, with its own
// boundary nodes sewn to the skin by seam stitches and rails.  Lines: rows
// at chord fractions 0.10, 0.35, 0.60 and the trailing edge (brake, every
// other rib), cascaded pairwise over `line_levels` levels to two riser tops,
// each line a chain of line_particles internal particles joined by cables.
// Two suspension segments join the riser tops to harness points of a rigid
// pilot.
swb_status swb_generate_wing(const swb_wing_params* p, swb_definition** out) {
    return guarded([&] {
        if (!p || !out) raise(SWB_INVALID_ARGUMENT, "null argument");
        if (p->cells < 1 || p->chordwise < 4 || p->spanwise_per_cell < 1 ||
            p->rib_layers < 1 || p->fabric > 1 || !(p->root_chord > 0) || !(p->thickness > 0) ||
            !(p->areal_density > 0) || p->skin_compliance < 0 ||
            !(p->bend_rigidity > 0) || p->line_rows > 4 || p->line_levels < 1 ||
            p->line_levels > 6 || p->line_particles > 64 ||
            (p->attachments_per_cell > 1 && p->spanwise_per_cell % p->attachments_per_cell != 0))
            raise(SWB_INVALID_ARGUMENT, "invalid wing parameters");
        auto* def = new swb_definition;
        try {
            Builder b(def->def);
            Rng rng(p->seed);
            const double c0 = p->root_chord;
            double span = p->span;
            if (p->aspect_ratio > 0.0) span = p->aspect_ratio * 3.141592653589793 * c0 / 4.0;
            const double jitter_scale =
                p->compliance_jitter > 0 ? std::exp(p->compliance_jitter * rng.normal()) : 1.0;
            const double skin_compliance = p->skin_compliance * jitter_scale;
            const uint32_t C = p->chordwise;
            const uint32_t S = p->cells * p->spanwise_per_cell;
            const uint32_t loop = 2 * C;
            const double phi_max = 0.5;
            const double radius = 0.5 * span / phi_max;
            std::vector<double> xi(C + 1);
            for (uint32_t j = 0; j <= C; ++j)
                xi[j] = static_cast<double>(j) / C;
            auto half_thickness = [&](double x) {
                return 5.0 * p->thickness *
                       (0.2969 * std::sqrt(x) - 0.1260 * x - 0.3516 * x * x +
                        0.2843 * x * x * x - 0.1036 * x * x * x * x);
            };
            struct Station { V centre, up; double chord; };
            auto station = [&](uint32_t s) {
                const double eta = -1.0 + 2.0 * s / S;
                const double phi = eta * phi_max;
                Station st;
                st.centre = {0.0, radius * std::sin(phi), radius * (std::cos(phi) - 1.0)};
                st.up = {0.0, -std::sin(phi), std::cos(phi)};
                st.chord = c0 * std::sqrt(1.0 - 0.9 * eta * eta);
                return st;
            };
            auto surface_point = [&](const Station& st, double x, double side) {
                const double yt = half_thickness(x) * st.chord;
                V q = st.centre;
                q.x += -0.25 * st.chord + x * st.chord;
                return q + st.up * (side * yt);
            };
            // Skin nodes: loop index k -- 0..C bottom from TE to LE, C..2C-1
            // top from LE towards TE.
            std::vector<uint64_t> skin((S + 1) * loop);
            for (uint32_t s = 0; s <= S; ++s) {
                const Station st = station(s);
                for (uint32_t k = 0; k < loop; ++k) {
                    const bool bottom = k <= C;
                    const double x = bottom ? xi[C - k] : xi[k - C];
                    skin[s * loop + k] = b.node(surface_point(st, x, bottom ? -1.0 : 1.0));
                }
            }
            const size_t skin_first = def->def.triangles.size();
            for (uint32_t s = 0; s < S; ++s)
                for (uint32_t k = 0; k < loop; ++k) {
                    const uint64_t A = skin[s * loop + k];
                    const uint64_t B = skin[s * loop + (k + 1) % loop];
                    const uint64_t Cn = skin[(s + 1) * loop + (k + 1) % loop];
                    const uint64_t D = skin[(s + 1) * loop + k];
                    b.triangle(A, B, Cn, p->pressure, p->areal_density);
                    b.triangle(A, Cn, D, p->pressure, p->areal_density);
                }
            const size_t skin_last = def->def.triangles.size();
            // fabric: edge constraints, or membrane elements (ripstop nylon:
            // warp along the chord, N/m)
            swb_membrane_material fabric{};
            fabric.warp_stiffness = 4.0e4;
            fabric.weft_stiffness = 3.0e4;
            fabric.coupling_stiffness = 6.0e3;
            fabric.shear_stiffness = 1.5e3;
            fabric.compression_stiffness_ratio = 1.0;
            const V chordwise{1.0, 0.0, 0.0};
            if (p->fabric == 1)
                b.membranes(skin_first, skin_last, chordwise, fabric);
            else
                b.edge_constraints(skin_first, skin_last, skin_compliance);
            b.dihedrals(skin_first, skin_last, p->bend_rigidity, -1.0);

            // Ribs with their own nodes, sewn to the skin.  The last rib
            // column is one station before the trailing edge (the section is
            // thinnest there); the rib fans from it to the trailing-edge node,
            // and the skin station between them is not sewn.  Each column is
            // split through the thickness into as many layers as keep its
            // elements about as tall as the chordwise station spacing (at
            // most rib_layers, at least one), so no rib element is a sliver
            // where the section thins towards the trailing edge.  The two end ribs close the end cells and carry
            // the outward pressure jump; the inner ribs separate pressurised
            // cells and carry none.
            const uint32_t L = p->rib_layers;
            const uint32_t J = C - 1;  // rib columns 1 .. J-1, fan from J-1 to the trailing edge
            const double seam_ea = 1.0e5;
            for (uint32_t r = 0; r <= p->cells; ++r) {
                const uint32_t s = r * p->spanwise_per_cell;
                const Station st = station(s);
                std::vector<std::vector<uint64_t>> col(C + 1);
                const uint64_t le = b.node(surface_point(st, 0.0, 1.0));
                const uint64_t te = b.node(surface_point(st, 1.0, 1.0));
                // layers per column: about the section height over the
                // station spacing, graded so that neighbouring columns differ
                // by at most one layer (a strip then adds at most one
                // triangle)
                std::vector<uint32_t> layers(C + 1, 1);
                for (uint32_t j = 1; j < J; ++j) {
                    const double height = length(surface_point(st, xi[j], 1.0) - surface_point(st, xi[j], -1.0));
                    const double spacing = 0.5 * (xi[j + 1] - xi[j - 1]) * st.chord;
                    layers[j] = static_cast<uint32_t>(
                        std::clamp(std::round(height / spacing), 1.0, static_cast<double>(L)));
                }
                for (uint32_t j = 2; j < J; ++j) layers[j] = std::min(layers[j], layers[j - 1] + 1);
                for (uint32_t j = J - 2; j >= 1; --j) layers[j] = std::min(layers[j], layers[j + 1] + 1);
                for (uint32_t j = 1; j < J; ++j) {
                    const V lo = surface_point(st, xi[j], -1.0);
                    const V hi = surface_point(st, xi[j], 1.0);
                    for (uint32_t l = 0; l <= layers[j]; ++l)
                        col[j].push_back(b.node(lo + (hi - lo) * (double(l) / layers[j])));
                }
                // End ribs: the normal of the fans and strips below points
                // to -y (the r = 0 side); the far end rib takes the jump with
                // the opposite sign so that both push outwards.
                const double rib_pressure =
                    r == 0 ? p->pressure : (r == p->cells ? -p->pressure : 0.0);
                const size_t first = def->def.triangles.size();
                for (size_t l = 0; l + 1 < col[1].size(); ++l)
                    b.triangle(le, col[1][l], col[1][l + 1], rib_pressure, p->areal_density);
                for (uint32_t j = 1; j + 1 < J; ++j) {
                    const std::vector<uint64_t>& u = col[j];
                    const std::vector<uint64_t>& w = col[j + 1];
                    // advance the column with more layers left: the extra
                    // triangle of a graded strip sits at the bottom boundary,
                    // whose nodes have the fewest triangles, so no rib node
                    // gathers more than six; quads split along one diagonal
                    size_t a = 0, c = 0;
                    while (a + 1 < u.size() || c + 1 < w.size()) {
                        const bool advance_u = u.size() - a > w.size() - c;
                        if (advance_u) {
                            b.triangle(u[a], w[c], u[a + 1], rib_pressure, p->areal_density);
                            ++a;
                        } else {
                            b.triangle(u[a], w[c], w[c + 1], rib_pressure, p->areal_density);
                            ++c;
                        }
                    }
                }
                for (size_t l = 0; l + 1 < col[J - 1].size(); ++l)
                    b.triangle(col[J - 1][l], te, col[J - 1][l + 1], rib_pressure, p->areal_density);
                const size_t last = def->def.triangles.size();
                if (p->fabric == 1)
                    b.membranes(first, last, chordwise, fabric);
                else
                    b.edge_constraints(first, last, skin_compliance);
                b.dihedrals(first, last, p->bend_rigidity, -1.0);
                // Seam: the rib boundary loop (skin loop order, skipping the
                // skin station next to the trailing edge on both surfaces)
                // sewn to the matching skin nodes.
                std::vector<uint64_t> rib_loop, skin_loop;
                for (uint32_t k = 0; k < loop; ++k) {
                    if (k == 1 || k == loop - 1) continue;
                    skin_loop.push_back(skin[s * loop + k]);
                    if (k == 0) rib_loop.push_back(te);
                    else if (k == C) rib_loop.push_back(le);
                    else if (k < C) rib_loop.push_back(col[C - k].front());
                    else rib_loop.push_back(col[k - C].back());
                }
                const size_t seam = rib_loop.size();
                for (size_t k = 0; k < seam; ++k)
                    b.distance(SWB_CONSTRAINT_SEAM_STITCH, rib_loop[k], skin_loop[k], 0.0, 0.0);
                for (const auto* chain : {&rib_loop, &skin_loop})
                    for (size_t k = 0; k < seam; ++k) {
                        const uint64_t a = (*chain)[k], bb = (*chain)[(k + 1) % seam];
                        const double len = length(b.design[bb] - b.design[a]);
                        b.distance(SWB_CONSTRAINT_DISTANCE, a, bb, len, 2.0 * len / seam_ea);
                    }
            }
            const size_t fabric_nodes = def->def.nodes.size();

            // Lines.
            const V pilot_com = {0.25 * c0, 0.0, -7.0};
            const V harness_local[2] = {{0.0, -0.22, 0.35}, {0.0, 0.22, 0.35}};
            const double riser_length = 0.45;
            uint64_t riser_top[2] = {0, 0};
            const double line_density = 0.006;  // kg/m
            if (p->line_rows > 0) {
                for (int side = 0; side < 2; ++side) {
                    const V top = pilot_com + harness_local[side] + V{0.0, 0.0, riser_length};
                    riser_top[side] = b.node(top);
                    b.mass[riser_top[side]] = 0.08;
                }
                auto add_line = [&](uint64_t from, uint64_t to, double ea) {
                    const V a = b.design[from], c = b.design[to];
                    const uint32_t pieces = p->line_particles + 1;
                    const double piece = length(c - a) / pieces;
                    uint64_t prev = from;
                    for (uint32_t q = 1; q <= pieces; ++q) {
                        uint64_t next = to;
                        if (q < pieces) {
                            next = b.node(a + (c - a) * (double(q) / pieces));
                            b.mass[next] = line_density * piece;
                        }
                        b.distance(SWB_CONSTRAINT_CABLE, prev, next, piece,
                                   p->line_compliance_scale * jitter_scale * piece / ea);
                        prev = next;
                    }
                    b.mass[from] += 0.5 * line_density * piece;
                    b.mass[to] += 0.5 * line_density * piece;
                };
                const double row_x[4] = {0.10, 0.35, 0.60, 1.0};
                // Attachment stations: every rib, or `attachments_per_cell`
                // evenly spaced stations per cell.
                const uint32_t per_cell = p->attachments_per_cell ? p->attachments_per_cell : 1u;
                const uint32_t stride = p->spanwise_per_cell / per_cell;
                const uint32_t stations = p->cells * per_cell;
                for (uint32_t row = 0; row < p->line_rows; ++row) {
                    for (int side = 0; side < 2; ++side) {
                        // Attachments of this row and side, ordered from the
                        // centre outwards.
                        std::vector<uint64_t> level;
                        const bool brake = row == 3;
                        for (uint32_t r = 0; r <= stations; ++r) {
                            const double eta = -1.0 + 2.0 * r / stations;
                            if ((side == 0) != (eta <= 0.0)) continue;
                            if (brake && (r % 2) != 0) continue;
                            const uint32_t s = r * stride;
                            uint32_t best = 0;
                            for (uint32_t k = 0; k <= C; ++k)
                                if (std::fabs(xi[C - k] - row_x[row]) <
                                    std::fabs(xi[C - best] - row_x[row]))
                                    best = k;
                            level.push_back(skin[s * loop + best]);
                        }
                        if (side == 0) std::reverse(level.begin(), level.end());
                        const V riser = b.design[riser_top[side]];
                        for (uint32_t lv = p->line_levels; lv >= 1 && !level.empty(); --lv) {
                            std::vector<uint64_t> parents;
                            const double ea = 2.0e4 * (1.0 + (p->line_levels - lv));
                            if (lv == 1) {
                                for (uint64_t n : level) add_line(n, riser_top[side], ea);
                                break;
                            }
                            const double pull = 1.0 - double(lv - 1) / p->line_levels;
                            for (size_t g = 0; g < level.size(); g += 2) {
                                const size_t e = std::min(level.size(), g + 2);
                                V centre{0, 0, 0};
                                for (size_t q = g; q < e; ++q) centre = centre + b.design[level[q]];
                                centre = centre * (1.0 / double(e - g));
                                const uint64_t knot = b.node(centre + (riser - centre) * pull);
                                b.mass[knot] = 0.01;
                                for (size_t q = g; q < e; ++q) add_line(level[q], knot, ea);
                                parents.push_back(knot);
                            }
                            level.swap(parents);
                        }
                    }
                }
            }
            b.finish_masses(0.0);
            // Fabric nodes carry area/3 mass plus their line share.
            for (size_t i = fabric_nodes; i < def->def.nodes.size(); ++i)
                if (!(def->def.nodes[i].mass > 0.0)) def->def.nodes[i].mass = 1.0e-3;

            if (p->pilot && p->line_rows > 0) {
                OwnedDefinition& d = def->def;
                d.has_suspension = true;
                swb_suspension_def& sp = d.suspension;
                std::memset(&sp, 0, sizeof(sp));
                sp.pilot_stable_id = 1;
                sp.pilot_mass = p->pilot_mass;
                sp.pilot_com_local = {0.0, 0.0, 0.0};
                sp.pilot_initial_com_world = {pilot_com.x, pilot_com.y, pilot_com.z};
                sp.pilot_initial_body_to_world = {1.0, 0.0, 0.0, 0.0};
                sp.pilot_principal_inertia = {12.0, 10.0, 6.0};
                sp.solver_iterations = 48;
                sp.attachment_tolerance = 1.0e-10;
                sp.minimum_line_length = 1.0e-10;
                sp.maximum_line_residual = 2.0e-4;
                sp.maximum_control_work = 1.0e6;
                for (int side = 0; side < 2; ++side) {
                    d.attachments.push_back({uint64_t(side + 1), riser_top[side]});
                    d.harness.push_back({uint64_t(side + 1),
                                         {harness_local[side].x, harness_local[side].y,
                                          harness_local[side].z}});
                    swb_suspension_segment g{};
                    g.stable_id = uint64_t(side + 1);
                    g.from = {SWB_ENDPOINT_SURFACE_ATTACHMENT, 0, uint64_t(side + 1)};
                    g.to = {SWB_ENDPOINT_PILOT_HARNESS, 0, uint64_t(side + 1)};
                    g.rest_length = riser_length;
                    g.axial_stiffness = 4.0e5;
                    g.axial_damping = 40.0;
                    g.role = 1;
                    d.segments.push_back(g);
                }
            }
            def->def.sync_view();
        } catch (...) {
            delete def;
            throw;
        }
        *out = def;
    });
}

}  // extern "C"
