// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into the product.
//
// FP64 reference gradient of a rollout loss through the XPBD structure step,
// for checking the device adjoint.  The reference has no adjoint; this is the
// discrete adjoint of the oracle's own forward step (xpbd_oracle.c, which is
// pinned bit for bit to the reference's Structure::step), computed
// independently of the device code: every local operation is re-evaluated in
// forward mode with dual numbers to obtain its Jacobian, and the Jacobians
// are chained in reverse order over the recorded inputs of each operation.
//
// Forward step restated here (double instantiation; the same operations and
// order as xpbd_oracle.c, and a test checks the two agree bit for bit):
//   pressure_scatter   soft_body.cpp:1492-1509
//   integrate_payload  suspension.cpp:1075-1102
//   predict            soft_body.cpp:1536-1566
//   project_distance   soft_body.cpp:1598-1640
//   dihedral           soft_body.cpp:1648-1711, 1754-1792
//   line_iteration     suspension.cpp:2197-2274
//   seam closing pass  soft_body.cpp:1389-1405
//   finalize           soft_body.cpp:1568-1585
//   payload finish     suspension.cpp:2386-2479 (velocity reconstruction and
//                      line damping; certification changes no state)
//
// Loss: L = sum_i m_i |x_i(T) - target_i|^2 / sum_i m_i over the final
// positions.  Gradients: every constraint's rest length and compliance,
// every dihedral's compliance, every suspension segment's rest length and
// the pilot mass.  One substep per step; momentum restoration (free
// membranes only) is not restated.
#include "simwing_b200.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

// ---- dual numbers ------------------------------------------------------------
template <int N>
struct Dual {
    double v = 0.0;
    std::array<double, N> d{};
    Dual() = default;
    Dual(double x) : v(x) {}  // NOLINT: constants promote implicitly
};

double val(double x) { return x; }
template <int N> double val(const Dual<N>& x) { return x.v; }

template <int N> Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r(a.v + b.v);
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N> Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r(a.v - b.v);
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N> Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r(-a.v);
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int N> Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r(a.v * b.v);
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N> Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r(a.v / b.v);
    const double ib = 1.0 / b.v;
    for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}
template <int N> Dual<N> operator+(const Dual<N>& a, double b) { return a + Dual<N>(b); }
template <int N> Dual<N> operator+(double a, const Dual<N>& b) { return Dual<N>(a) + b; }
template <int N> Dual<N> operator-(const Dual<N>& a, double b) { return a - Dual<N>(b); }
template <int N> Dual<N> operator-(double a, const Dual<N>& b) { return Dual<N>(a) - b; }
template <int N> Dual<N> operator*(const Dual<N>& a, double b) { return a * Dual<N>(b); }
template <int N> Dual<N> operator*(double a, const Dual<N>& b) { return Dual<N>(a) * b; }
template <int N> Dual<N> operator/(const Dual<N>& a, double b) { return a / Dual<N>(b); }
template <int N> Dual<N> operator/(double a, const Dual<N>& b) { return Dual<N>(a) / b; }

template <int N> Dual<N> chain(const Dual<N>& a, double f, double df) {
    Dual<N> r(f);
    for (int i = 0; i < N; ++i) r.d[i] = df * a.d[i];
    return r;
}
template <int N> Dual<N> sqrt(const Dual<N>& a) {
    const double s = std::sqrt(a.v);
    return chain(a, s, 0.5 / s);
}
template <int N> Dual<N> sin(const Dual<N>& a) { return chain(a, std::sin(a.v), std::cos(a.v)); }
template <int N> Dual<N> cos(const Dual<N>& a) { return chain(a, std::cos(a.v), -std::sin(a.v)); }
template <int N> Dual<N> acos(const Dual<N>& a) {
    return chain(a, std::acos(a.v), -1.0 / std::sqrt(1.0 - a.v * a.v));
}
template <int N> Dual<N> fabs(const Dual<N>& a) { return a.v < 0.0 ? -a : a; }
template <int N> Dual<N> atan2(const Dual<N>& y, const Dual<N>& x) {
    Dual<N> r(std::atan2(y.v, x.v));
    const double den = x.v * x.v + y.v * y.v;
    for (int i = 0; i < N; ++i) r.d[i] = (x.v * y.d[i] - y.v * x.d[i]) / den;
    return r;
}
template <int N> Dual<N> copysign(const Dual<N>& mag, const Dual<N>& sgn) {
    const bool flip = std::signbit(mag.v) != std::signbit(sgn.v);
    return flip ? -mag : mag;
}
// remainder(x, 2 pi): the integer multiple is piecewise constant
template <int N> Dual<N> remainder2pi(const Dual<N>& x, double two_pi) {
    const double r = std::remainder(x.v, two_pi);
    Dual<N> out = x;
    out.v = r;
    return out;
}
inline double remainder2pi(double x, double two_pi) { return std::remainder(x, two_pi); }

using std::acos;
using std::atan2;
using std::copysign;
using std::cos;
using std::fabs;
using std::sin;
using std::sqrt;

// ---- vectors, matrices, quaternions -----------------------------------------
template <class T> struct V3 { T x, y, z; };
template <class T> V3<T> v3(T x, T y, T z) { return {x, y, z}; }
template <class T> V3<T> add(const V3<T>& a, const V3<T>& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> V3<T> sub(const V3<T>& a, const V3<T>& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T, class S> V3<T> mul(const V3<T>& a, const S& s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T, class S> V3<T> smul(const S& s, const V3<T>& a) { return {a.x * s, a.y * s, a.z * s}; }
template <class T, class S> V3<T> vdiv(const V3<T>& a, const S& s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> V3<T> neg(const V3<T>& a) { return {-a.x, -a.y, -a.z}; }
template <class T> T dot(const V3<T>& a, const V3<T>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> V3<T> cross(const V3<T>& a, const V3<T>& b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> T len(const V3<T>& a) { return sqrt(dot(a, a)); }
template <class T> V3<T> normalized(const V3<T>& a) {
    const T l = len(a);
    if (!(val(l) > 0.0)) return {T(0.0), T(0.0), T(0.0)};
    return vdiv(a, l);
}
template <class T> struct M3 { T v[9]; };
template <class T> M3<T> m3mul(const M3<T>& a, const M3<T>& b) {
    M3<T> r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            r.v[i * 3 + j] = a.v[i * 3 + 0] * b.v[0 * 3 + j] + a.v[i * 3 + 1] * b.v[1 * 3 + j] +
                             a.v[i * 3 + 2] * b.v[2 * 3 + j];
    return r;
}
template <class T> M3<T> m3t(const M3<T>& a) {
    M3<T> r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.v[i * 3 + j] = a.v[j * 3 + i];
    return r;
}
template <class T> V3<T> m3v(const M3<T>& m, const V3<T>& v) {
    return {m.v[0] * v.x + m.v[1] * v.y + m.v[2] * v.z, m.v[3] * v.x + m.v[4] * v.y + m.v[5] * v.z,
            m.v[6] * v.x + m.v[7] * v.y + m.v[8] * v.z};
}
template <class T> T det3(const M3<T>& m) {
    return m.v[0] * (m.v[4] * m.v[8] - m.v[5] * m.v[7]) - m.v[1] * (m.v[3] * m.v[8] - m.v[5] * m.v[6]) +
           m.v[2] * (m.v[3] * m.v[7] - m.v[4] * m.v[6]);
}
template <class T> bool m3inv(const M3<T>& m, M3<T>& out) {
    int best = 0;
    for (int i = 0; i < 9; ++i)
        if (std::fabs(val(m.v[i])) > std::fabs(val(m.v[best]))) best = i;
    const T scale = fabs(m.v[best]);
    if (!(val(scale) > 0.0)) return false;
    M3<T> n = m;
    for (int i = 0; i < 9; ++i) n.v[i] = n.v[i] / scale;
    const T det = det3(n);
    if (!(std::fabs(val(det)) > 1.0e-14)) return false;
    M3<T> r = {{n.v[4] * n.v[8] - n.v[5] * n.v[7], n.v[2] * n.v[7] - n.v[1] * n.v[8],
                n.v[1] * n.v[5] - n.v[2] * n.v[4], n.v[5] * n.v[6] - n.v[3] * n.v[8],
                n.v[0] * n.v[8] - n.v[2] * n.v[6], n.v[2] * n.v[3] - n.v[0] * n.v[5],
                n.v[3] * n.v[7] - n.v[4] * n.v[6], n.v[1] * n.v[6] - n.v[0] * n.v[7],
                n.v[0] * n.v[4] - n.v[1] * n.v[3]}};
    const T f = det * scale;
    for (int i = 0; i < 9; ++i) r.v[i] = r.v[i] / f;
    out = r;
    return true;
}
template <class T> struct Q { T w, x, y, z; };
template <class T> bool qcanon(const Q<T>& q, Q<T>& out) {
    const T n2 = q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z;
    if (!(val(n2) > 1.0e-28)) return false;
    const T inv = 1.0 / sqrt(n2);
    Q<T> r = {q.w * inv, q.x * inv, q.y * inv, q.z * inv};
    const bool flip = val(r.w) < 0.0 ||
                      (val(r.w) == 0.0 && (val(r.x) < 0.0 || (val(r.x) == 0.0 && (val(r.y) < 0.0 ||
                                                                                 (val(r.y) == 0.0 && val(r.z) < 0.0)))));
    if (flip) r = {-r.w, -r.x, -r.y, -r.z};
    out = r;
    return true;
}
template <class T> Q<T> qmul(const Q<T>& a, const Q<T>& b) {
    return {a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z, a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
            a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x, a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w};
}
template <class T> bool qrot(const Q<T>& o, M3<T>& out) {
    Q<T> q;
    if (!qcanon(o, q)) return false;
    const T xx = q.x * q.x, yy = q.y * q.y, zz = q.z * q.z;
    const T xy = q.x * q.y, xz = q.x * q.z, yz = q.y * q.z;
    const T wx = q.w * q.x, wy = q.w * q.y, wz = q.w * q.z;
    out = {{1.0 - 2.0 * (yy + zz), 2.0 * (xy - wz), 2.0 * (xz + wy), 2.0 * (xy + wz), 1.0 - 2.0 * (xx + zz),
            2.0 * (yz - wx), 2.0 * (xz - wy), 2.0 * (yz + wx), 1.0 - 2.0 * (xx + yy)}};
    return true;
}
template <class T> bool qincrement(const V3<T>& r, Q<T>& out) {
    const T angle = len(r);
    if (val(angle) < 1.0e-12) return qcanon(Q<T>{T(1.0), 0.5 * r.x, 0.5 * r.y, 0.5 * r.z}, out);
    const T half = 0.5 * angle;
    const T scale = sin(half) / angle;
    out = {cos(half), r.x * scale, r.y * scale, r.z * scale};
    return true;
}

// ---- model --------------------------------------------------------------------
constexpr double kMinimumLength = 1.0e-12;
constexpr double kTwoPi = 6.283185307179586476925286766559;

struct Seg {
    int from_node = -1, to_node = -1, from_point = -1, to_point = -1;
    double rest = 0, stiffness = 0, damping = 0;
    uint64_t definition_index = 0;
};

struct Model {
    uint64_t n = 0, t = 0, m = 0, h = 0;
    std::vector<V3<double>> x0, v0;
    std::vector<double> w;
    std::vector<std::array<uint64_t, 3>> tri;
    std::vector<double> pressure;
    std::vector<uint64_t> ca, cb;
    std::vector<uint32_t> kind;
    std::vector<double> rest, comp;
    std::vector<std::array<uint64_t, 4>> hn;
    std::vector<double> hrest, hcomp;
    bool susp = false;
    double mass = 0;
    V3<double> com_local{0, 0, 0};
    M3<double> inertia{};
    std::vector<V3<double>> hang_local;
    std::vector<Seg> seg;
    std::vector<int> att_nodes;  // distinct nodes referenced by segments
    double min_line_length = 0;
    // initial payload
    V3<double> p_com{0, 0, 0}, p_v{0, 0, 0}, p_w{0, 0, 0};
    Q<double> p_q{1, 0, 0, 0};
    std::vector<V3<double>> pending;
};

int cmp_u64str(uint64_t a, uint64_t b) {
    char sa[32], sb[32];
    std::snprintf(sa, sizeof sa, "%llu", static_cast<unsigned long long>(a));
    std::snprintf(sb, sizeof sb, "%llu", static_cast<unsigned long long>(b));
    return std::strcmp(sa, sb);
}

V3<double> fromabi(const swb_vec3& a) { return {a.x, a.y, a.z}; }

bool build_model(const swb_structure_definition& d, Model& M, std::string& err) {
    if (d.membrane_count || d.fabric_self_contact) {
        err = "membranes/contact not restated";
        return false;
    }
    M.n = d.node_count;
    M.t = d.triangle_count;
    M.m = d.constraint_count;
    M.h = d.dihedral_count;
    for (uint64_t i = 0; i < M.n; ++i) {
        M.x0.push_back(fromabi(d.nodes[i].position));
        M.v0.push_back({0, 0, 0});
        M.w.push_back(d.nodes[i].fixed ? 0.0 : 1.0 / d.nodes[i].mass);
    }
    for (uint64_t i = 0; i < M.t; ++i) {
        M.tri.push_back({d.triangles[i].nodes[0], d.triangles[i].nodes[1], d.triangles[i].nodes[2]});
        M.pressure.push_back(d.triangles[i].pressure_difference);
    }
    for (uint64_t i = 0; i < M.m; ++i) {
        const swb_constraint_def& c = d.constraints[i];
        M.ca.push_back(c.first_node);
        M.cb.push_back(c.second_node);
        M.kind.push_back(c.kind);
        M.rest.push_back(c.kind == SWB_CONSTRAINT_SEAM_STITCH ? 0.0 : c.rest_length);
        M.comp.push_back(c.kind == SWB_CONSTRAINT_SEAM_STITCH ? 0.0 : c.compliance);
    }
    for (uint64_t i = 0; i < M.h; ++i) {
        const swb_dihedral_def& h = d.dihedrals[i];
        M.hn.push_back({h.nodes[0], h.nodes[1], h.nodes[2], h.nodes[3]});
        M.hrest.push_back(h.rest_angle);
        M.hcomp.push_back(h.compliance);
    }
    M.pending.assign(M.n, {0, 0, 0});
    if (d.suspension) {
        const swb_suspension_def& sp = *d.suspension;
        M.susp = true;
        M.mass = sp.pilot_mass;
        M.com_local = fromabi(sp.pilot_com_local);
        M.inertia = {{sp.pilot_principal_inertia.x, 0, 0, 0, sp.pilot_principal_inertia.y, 0, 0, 0,
                      sp.pilot_principal_inertia.z}};
        M.p_com = fromabi(sp.pilot_initial_com_world);
        Q<double> q0 = {sp.pilot_initial_body_to_world.w, sp.pilot_initial_body_to_world.x,
                        sp.pilot_initial_body_to_world.y, sp.pilot_initial_body_to_world.z};
        if (!qcanon(q0, M.p_q)) {
            err = "invalid pilot orientation";
            return false;
        }
        M.p_v = fromabi(sp.pilot_initial_linear_velocity);
        M.p_w = fromabi(sp.pilot_initial_angular_velocity);
        M.min_line_length = sp.minimum_line_length;
        std::vector<uint64_t> ho(sp.harness_count), so(sp.segment_count);
        for (uint64_t i = 0; i < ho.size(); ++i) ho[i] = i;
        for (uint64_t i = 0; i < so.size(); ++i) so[i] = i;
        std::stable_sort(ho.begin(), ho.end(), [&](uint64_t a, uint64_t b) {
            return cmp_u64str(sp.harness_points[a].stable_id, sp.harness_points[b].stable_id) < 0;
        });
        std::stable_sort(so.begin(), so.end(), [&](uint64_t a, uint64_t b) {
            return cmp_u64str(sp.segments[a].stable_id, sp.segments[b].stable_id) < 0;
        });
        for (uint64_t i : ho) M.hang_local.push_back(fromabi(sp.harness_points[i].local_position));
        for (uint64_t k : so) {
            const swb_suspension_segment& g = sp.segments[k];
            Seg s;
            s.definition_index = k;
            s.rest = g.rest_length;
            s.stiffness = g.axial_stiffness;
            s.damping = g.axial_damping;
            const swb_suspension_endpoint* ends[2] = {&g.from, &g.to};
            for (int e = 0; e < 2; ++e) {
                int node = -1, point = -1;
                if (ends[e]->kind == SWB_ENDPOINT_SURFACE_ATTACHMENT) {
                    for (uint64_t a = 0; a < sp.attachment_count; ++a)
                        if (sp.attachments[a].stable_id == ends[e]->stable_id) node = static_cast<int>(sp.attachments[a].node);
                } else if (ends[e]->kind == SWB_ENDPOINT_JUNCTION) {
                    for (uint64_t a = 0; a < sp.junction_count; ++a)
                        if (sp.junctions[a].stable_id == ends[e]->stable_id) node = static_cast<int>(sp.junctions[a].node);
                } else {
                    for (uint64_t a = 0; a < ho.size(); ++a)
                        if (sp.harness_points[ho[a]].stable_id == ends[e]->stable_id) point = static_cast<int>(a);
                }
                (e == 0 ? s.from_node : s.to_node) = node;
                (e == 0 ? s.from_point : s.to_point) = point;
            }
            if (s.from_node < 0 && s.from_point < 0) {
                err = "unresolved endpoint";
                return false;
            }
            if (s.to_node < 0 && s.to_point < 0) {
                err = "unresolved endpoint";
                return false;
            }
            M.seg.push_back(s);
            for (int node : {s.from_node, s.to_node})
                if (node >= 0 && std::find(M.att_nodes.begin(), M.att_nodes.end(), node) == M.att_nodes.end())
                    M.att_nodes.push_back(node);
        }
    }
    return true;
}

// ---- templated local operations --------------------------------------------
template <class T>
struct Payload {
    V3<T> com, v, w;
    Q<T> q;
};

template <class T>
bool world_inertia(const M3<double>& Ib, const Q<T>& q, M3<T>& out) {
    M3<T> r;
    if (!qrot(q, r)) return false;
    M3<T> I;
    for (int i = 0; i < 9; ++i) I.v[i] = T(Ib.v[i]);
    const M3<T> a = m3mul(r, I);
    out = m3mul(a, m3t(r));
    return true;
}

template <class T>
void project_distance(V3<T>& a, V3<T>& b, double wa, double wb, T& lambda, const T& rest, const T& comp,
                      uint32_t kind, double inv_dt2) {
    const V3<T> diff = sub(b, a);
    const T l = len(diff);
    if (val(l) <= kMinimumLength) return;
    const T value = l - rest;
    if (kind == SWB_CONSTRAINT_CABLE && val(value) <= 0.0 && val(lambda) == 0.0) return;
    const double wsum = wa + wb;
    const T alpha = comp * inv_dt2;
    if (val(wsum + alpha) <= 0.0) return;
    const T dl = (-value - alpha * lambda) / (wsum + alpha);
    T applied = dl;
    if (kind == SWB_CONSTRAINT_CABLE) {
        const T s = lambda + dl;
        const T newl = val(s) < 0.0 ? s : T(0.0);
        applied = newl - lambda;
        lambda = newl;
    } else {
        lambda = lambda + dl;
    }
    const T scale = applied / l;
    a = sub(a, mul(diff, wa * scale));
    b = add(b, mul(diff, wb * scale));
}

template <class T>
void project_dihedral(V3<T> p[4], const double w[4], T& lambda, const T& rest, const T& comp, double inv_dt2) {
    const V3<T> edge = sub(p[1], p[0]);
    const V3<T> toC = sub(p[2], p[0]);
    const V3<T> toD = sub(p[3], p[0]);
    const V3<T> A1 = cross(edge, toC);
    const V3<T> A2 = cross(toD, edge);
    const T el = len(edge), l1 = len(A1), l2 = len(A2);
    if (!(val(el) > kMinimumLength) || !(val(l1) > kMinimumLength * val(el)) ||
        !(val(l2) > kMinimumLength * val(el)))
        return;
    const V3<T> e = vdiv(edge, el);
    const V3<T> n1 = vdiv(A1, l1);
    const V3<T> n2 = vdiv(A2, l2);
    T cosine = dot(n1, n2);
    if (val(cosine) < -1.0) cosine = T(-1.0);
    if (1.0 < val(cosine)) cosine = T(1.0);
    const T sine = dot(e, cross(n1, n2));
    const V3<T> n1adj = sub(smul(cosine, cross(n2, e)), smul(sine, n2));
    const V3<T> n2adj = sub(smul(cosine, cross(e, n1)), smul(sine, n1));
    const V3<T> eadj = smul(cosine, cross(n1, n2));
    const V3<T> a1adj = vdiv(sub(n1adj, smul(dot(n1adj, n1), n1)), l1);
    const V3<T> a2adj = vdiv(sub(n2adj, smul(dot(n2adj, n2), n2)), l2);
    V3<T> edgeadj = vdiv(sub(eadj, smul(dot(eadj, e), e)), el);
    edgeadj = add(edgeadj, cross(toC, a1adj));
    const V3<T> cadj = cross(a1adj, edge);
    edgeadj = add(edgeadj, cross(a2adj, toD));
    const V3<T> dadj = cross(edge, a2adj);
    const T angle = atan2(sine, cosine);
    V3<T> g[4];
    g[1] = edgeadj;
    g[2] = cadj;
    g[3] = dadj;
    g[0] = smul(T(-1.0), add(add(edgeadj, cadj), dadj));
    if (!std::isfinite(val(angle))) return;
    T wg = T(0.0);
    for (int k = 0; k < 4; ++k) wg = wg + w[k] * dot(g[k], g[k]);
    const T alpha = comp * inv_dt2;
    const T den = wg + alpha;
    if (!(val(den) > 0.0) || !std::isfinite(val(den))) return;
    const T value = remainder2pi(angle - rest, kTwoPi);
    const T dl = (-value - alpha * lambda) / den;
    if (!std::isfinite(val(dl))) return;
    for (int k = 0; k < 4; ++k) p[k] = add(p[k], smul(w[k] * dl, g[k]));
    lambda = lambda + dl;
}

template <class T>
bool integrate_payload(const Model& M, Payload<T>& s, const T& mass, double dt, const V3<double>& g) {
    if (!qcanon(s.q, s.q)) return false;
    M3<T> I, inv;
    if (!world_inertia(M.inertia, s.q, I)) return false;
    const V3<T> angular = m3v(I, s.w);
    const V3<T> force = {mass * g.x, mass * g.y, mass * g.z};
    s.v = add(s.v, mul(force, dt / mass));
    if (!m3inv(I, inv)) return false;
    s.w = m3v(inv, angular);
    s.com = add(s.com, mul(s.v, T(dt)));
    Q<T> inc;
    if (!qincrement(mul(s.w, T(dt)), inc)) return false;
    if (!qcanon(qmul(inc, s.q), s.q)) return false;
    if (!world_inertia(M.inertia, s.q, I) || !m3inv(I, inv)) return false;
    s.w = m3v(inv, angular);
    return true;
}

template <class T>
bool point_position(const Model& M, const Payload<T>& s, const V3<double>& local, V3<T>& out) {
    M3<T> r;
    if (!qrot(s.q, r)) return false;
    const V3<double> d = sub(local, M.com_local);
    out = add(s.com, m3v(r, V3<T>{T(d.x), T(d.y), T(d.z)}));
    return true;
}

// One line iteration over all segments.  xs[k] are the positions of
// M.att_nodes[k]; lam the segment multipliers; rest the segment rest lengths.
template <class T>
bool line_iteration(const Model& M, Payload<T>& s, std::vector<V3<T>>& xs, std::vector<T>& lam,
                    const std::vector<T>& rest, const T& mass, double dt) {
    M3<T> I, invI;
    if (!world_inertia(M.inertia, s.q, I) || !m3inv(I, invI)) return false;
    auto slot = [&](int node) {
        return static_cast<size_t>(std::find(M.att_nodes.begin(), M.att_nodes.end(), node) - M.att_nodes.begin());
    };
    for (size_t k = 0; k < M.seg.size(); ++k) {
        const Seg& g = M.seg[k];
        V3<T> p[2], off[2];
        T w[2];
        bool rigid[2], fixed[2];
        const int node[2] = {g.from_node, g.to_node};
        const int point[2] = {g.from_point, g.to_point};
        for (int e = 0; e < 2; ++e) {
            off[e] = {T(0.0), T(0.0), T(0.0)};
            if (node[e] >= 0) {
                p[e] = xs[slot(node[e])];
                w[e] = T(M.w[node[e]]);
                fixed[e] = M.w[node[e]] == 0.0;
                rigid[e] = false;
            } else {
                if (!point_position(M, s, M.hang_local[point[e]], p[e])) return false;
                off[e] = sub(p[e], s.com);
                rigid[e] = true;
                fixed[e] = false;
                w[e] = 1.0 / mass;
            }
        }
        const V3<T> diff = sub(p[1], p[0]);
        const T l = len(diff);
        if (!(val(l) > M.min_line_length)) return false;
        const V3<T> dir = vdiv(diff, l);
        const V3<T> grad[2] = {dir, neg(dir)};
        T eff = T(0.0);
        for (int e = 0; e < 2; ++e) {
            T r = w[e];
            if (rigid[e] && !fixed[e] && val(w[e]) > 0.0) {
                const V3<T> rot = cross(off[e], grad[e]);
                r = r + dot(rot, m3v(invI, rot));
            }
            eff = eff + r;
        }
        const double at = 1.0 / (g.stiffness * dt * dt);
        const T gap = rest[k] - l;
        const T cand = lam[k] + (-gap - at * lam[k]) / (eff + at);
        const T acc = 0.0 < val(cand) ? cand : T(0.0);
        const T inc = acc - lam[k];
        lam[k] = acc;
        for (int e = 0; e < 2; ++e) {
            if (fixed[e]) continue;
            if (node[e] >= 0) {
                V3<T>& X = xs[slot(node[e])];
                X = add(X, mul(grad[e], w[e] * inc));
            } else {
                s.com = add(s.com, mul(grad[e], w[e] * inc));
                const V3<T> rot = mul(m3v(invI, cross(off[e], grad[e])), inc);
                Q<T> qi;
                if (!qincrement(rot, qi) || !qcanon(qmul(qi, s.q), s.q)) return false;
            }
        }
    }
    return true;
}

// Velocity reconstruction and line damping; xs/vs: attachment node
// positions and velocities (M.att_nodes order); lam: segment multipliers
// (only their sign matters here).
template <class T>
bool payload_finish(const Model& M, Payload<T>& s, const Payload<T>& start, const std::vector<V3<T>>& xs,
                    std::vector<V3<T>>& vs, const std::vector<double>& lam, const T& mass, double dt) {
    s.v = vdiv(sub(s.com, start.com), T(dt));
    const Q<T> conj = {start.q.w, -start.q.x, -start.q.y, -start.q.z};
    Q<T> delta;
    if (!qcanon(qmul(s.q, conj), delta)) return false;
    T cw = delta.w;
    if (val(cw) < -1.0) cw = T(-1.0);
    if (1.0 < val(cw)) cw = T(1.0);
    const T half = acos(cw);
    const T sn = sin(half);
    if (std::fabs(val(sn)) < 1.0e-12) {
        s.w = mul(V3<T>{delta.x, delta.y, delta.z}, T(2.0 / dt));
    } else {
        const V3<T> axis = {delta.x / sn, delta.y / sn, delta.z / sn};
        s.w = mul(axis, 2.0 * half / dt);
    }
    M3<T> I, invI;
    if (!world_inertia(M.inertia, s.q, I) || !m3inv(I, invI)) return false;
    auto slot = [&](int node) {
        return static_cast<size_t>(std::find(M.att_nodes.begin(), M.att_nodes.end(), node) - M.att_nodes.begin());
    };
    auto position = [&](int node, int point, V3<T>& out) {
        if (node >= 0) {
            out = xs[slot(node)];
            return true;
        }
        return point_position(M, s, M.hang_local[point], out);
    };
    auto velocity = [&](int node, int point, V3<T>& out) {
        if (node >= 0) {
            out = vs[slot(node)];
            return true;
        }
        M3<T> r;
        if (!qrot(s.q, r)) return false;
        const V3<double> d = sub(M.hang_local[point], M.com_local);
        const V3<T> offset = m3v(r, V3<T>{T(d.x), T(d.y), T(d.z)});
        out = add(s.v, cross(s.w, offset));
        return true;
    };
    for (size_t k = 0; k < M.seg.size(); ++k) {
        const Seg& g = M.seg[k];
        if (!(lam[k] > 0.0) || !(g.damping > 0.0)) continue;
        V3<T> from, to, vf, vt;
        if (!position(g.from_node, g.from_point, from) || !position(g.to_node, g.to_point, to)) return false;
        const V3<T> dir = normalized(sub(to, from));
        if (!velocity(g.to_node, g.to_point, vt) || !velocity(g.from_node, g.from_point, vf)) return false;
        const T rel = dot(sub(vt, vf), dir);
        T eff = T(0.0);
        if (g.from_node >= 0) eff = eff + M.w[g.from_node];
        else {
            const V3<T> rxn = cross(sub(from, s.com), dir);
            eff = eff + (1.0 / mass + dot(rxn, m3v(invI, rxn)));
        }
        if (g.to_node >= 0) eff = eff + M.w[g.to_node];
        else {
            const V3<T> rxn = cross(sub(to, s.com), dir);
            eff = eff + (1.0 / mass + dot(rxn, m3v(invI, rxn)));
        }
        if (!(val(eff) > 0.0) || val(rel) == 0.0) continue;
        T mag = T(0.0);
        {
            const T req = g.damping * fabs(rel) * dt;
            const T stop = fabs(rel) / eff;
            mag = copysign(val(stop) < val(req) ? stop : req, rel);
        }
        const V3<T> fi = mul(dir, mag);
        const V3<T> ti = neg(fi);
        for (int e = 0; e < 2; ++e) {
            const int node = e == 0 ? g.from_node : g.to_node;
            const V3<T> point = e == 0 ? from : to;
            const V3<T> imp = e == 0 ? fi : ti;
            if (node >= 0) {
                if (M.w[node] > 0.0) vs[slot(node)] = add(vs[slot(node)], mul(imp, M.w[node]));
            } else {
                s.v = add(s.v, vdiv(imp, mass));
                s.w = add(s.w, m3v(invI, cross(sub(point, s.com), imp)));
            }
        }
    }
    return true;
}

// ---- Jacobian-transpose products by forward mode ------------------------------
template <int N> Dual<N> seed(double v, int i) {
    Dual<N> r(v);
    if (i >= 0) r.d[i] = 1.0;
    return r;
}
template <int N> V3<Dual<N>> seed3(const V3<double>& v, int i) {
    return {seed<N>(v.x, i), seed<N>(v.y, i + 1), seed<N>(v.z, i + 2)};
}
template <int N> void acc3(double* ubar, const V3<Dual<N>>& y, const V3<double>& ybar) {
    for (int i = 0; i < N; ++i) ubar[i] += y.x.d[i] * ybar.x + y.y.d[i] * ybar.y + y.z.d[i] * ybar.z;
}
template <int N> void acc1(double* ubar, const Dual<N>& y, double ybar) {
    for (int i = 0; i < N; ++i) ubar[i] += y.d[i] * ybar;
}

// ---- rollout --------------------------------------------------------------------
struct StepTape {
    std::vector<V3<double>> X, V;            // state at step start
    Payload<double> P;                       // payload at step start
    std::vector<V3<double>> force;           // external + pressure
    // iteration inputs
    std::vector<std::array<V3<double>, 2>> dist_in;   // [it * m + i]
    std::vector<double> dist_lambda;
    std::vector<std::array<V3<double>, 4>> dih_in;    // [it * h + i]
    std::vector<double> dih_lambda;
    std::vector<Payload<double>> line_P;              // [it]
    std::vector<std::vector<V3<double>>> line_x;      // [it]
    std::vector<std::vector<double>> line_lambda;     // [it]
    std::vector<std::array<V3<double>, 2>> seam_in;   // [i] (seam stitches in order)
    std::vector<double> seam_lambda;
    Payload<double> P_end;                            // after the iterations
    std::vector<V3<double>> fin_x, fin_v;             // attachment nodes at finish
    std::vector<double> fin_lambda;
    std::vector<uint8_t> ground_moved;                // [it * n + i]: the ground plane moved the node
    std::vector<std::array<size_t, 2>> line_pairs;    // the step's line-line candidates (segment indices), key order
    std::vector<std::array<V3<double>, 4>> line_in;   // [it * pairs + k]: the candidate's end nodes before it
};

struct Rollout {
    Model M;
    double dt = 1.0 / 120.0, damping = 1.0, inv_dt2 = 0;
    V3<double> g{0, 0, 0}, ref{0, 0, 0};
    int iterations = 0;
    std::vector<V3<double>> X, V;
    Payload<double> P;
    std::vector<StepTape> tape;
    std::vector<uint64_t> seams;  // seam stitch indices in sweep order
    // frictionless ground plane normal . x >= offset after each iteration
    // (the device's swb_structure_set_ground; no reference counterpart)
    bool ground = false;
    V3<double> ground_normal{0, 0, 1};
    double ground_offset = 0.0;
    // line-line contact of the cable segments (the device's
    // swb_structure_set_line_contact; no reference counterpart): segments by
    // (smaller, larger) node, the radius and the box reach
    bool lines = false;
    double line_radius = 0.0, line_reach = 0.0;
    std::vector<std::array<uint64_t, 2>> line_seg;
};

// Closest points of two segments (Ericson, Real-Time Collision Detection
// 5.1.9) as the device computes them, the clamps as constants.
template <class T> T clamp01(const T& x) { return val(x) < 0.0 ? T(0.0) : (val(x) > 1.0 ? T(1.0) : x); }

// One line-line projection: the segments' closest points pushed apart to
// `gap`, rigidly, the correction shared by the end nodes by inverse mass and
// barycentric weight.
template <class T>
void project_line_pair(V3<T>& A, V3<T>& B, V3<T>& C, V3<T>& D, const double w[4], double gap) {
    const V3<T> d1 = sub(B, A), d2 = sub(D, C), r = sub(A, C);
    constexpr double eps = 1.0e-12;
    const T a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    T s(0.0), t(0.0);
    if (val(a) <= eps && val(e) <= eps) {
    } else if (val(a) <= eps) {
        t = clamp01(f / e);
    } else {
        const T c = dot(d1, r);
        if (val(e) <= eps) {
            s = clamp01(-c / a);
        } else {
            const T b = dot(d1, d2), denom = a * e - b * b;
            s = val(denom) != 0.0 ? clamp01((b * f - c * e) / denom) : T(0.0);
            t = (b * s + f) / e;
            if (val(t) < 0.0) {
                t = T(0.0);
                s = clamp01(-c / a);
            } else if (val(t) > 1.0) {
                t = T(1.0);
                s = clamp01((b - c) / a);
            }
        }
    }
    const V3<T> diff = sub(add(A, mul(d1, s)), add(C, mul(d2, t)));
    const T dist = sqrt(dot(diff, diff));
    if (!(val(dist) < gap) || !(val(dist) > 0.0)) return;
    const V3<T> n = mul(diff, T(1.0) / dist);
    const T wa = w[0] * (1.0 - s), wb = w[1] * s, wc = w[2] * (1.0 - t), wd = w[3] * t;
    const T W = wa * (1.0 - s) + wb * s + wc * (1.0 - t) + wd * t;
    if (!(val(W) > 0.0)) return;
    const T dl = (gap - dist) / W;
    A = add(A, mul(n, wa * dl));
    B = add(B, mul(n, wb * dl));
    C = sub(C, mul(n, wc * dl));
    D = sub(D, mul(n, wd * dl));
}

// The step's line-line candidates at the predicted positions: segments that
// share no node and whose boxes, widened by the reach, overlap, in key order.
std::vector<std::array<size_t, 2>> line_candidates(const Rollout& R, const std::vector<V3<double>>& x) {
    std::vector<std::array<size_t, 2>> out;
    const double r = R.line_reach;
    const auto& S = R.line_seg;
    for (size_t i = 0; i < S.size(); ++i) {
        const V3<double> a = x[S[i][0]], b = x[S[i][1]];
        for (size_t j = i + 1; j < S.size(); ++j) {
            if (S[j][0] == S[i][0] || S[j][0] == S[i][1] || S[j][1] == S[i][0] || S[j][1] == S[i][1]) continue;
            const V3<double> c = x[S[j][0]], d = x[S[j][1]];
            if (std::fmin(a.x, b.x) - r > std::fmax(c.x, d.x) + r || std::fmin(c.x, d.x) - r > std::fmax(a.x, b.x) + r ||
                std::fmin(a.y, b.y) - r > std::fmax(c.y, d.y) + r || std::fmin(c.y, d.y) - r > std::fmax(a.y, b.y) + r ||
                std::fmin(a.z, b.z) - r > std::fmax(c.z, d.z) + r || std::fmin(c.z, d.z) - r > std::fmax(a.z, b.z) + r)
                continue;
            out.push_back({i, j});
        }
    }
    return out;
}

bool forward_step(Rollout& R, bool record) {
    const Model& M = R.M;
    StepTape T;
    if (record) {
        T.X = R.X;
        T.V = R.V;
        T.P = R.P;
    }
    // pressure_scatter
    std::vector<V3<double>> force = M.pending;
    for (uint64_t t = 0; t < M.t; ++t) {
        const V3<double> a = R.X[M.tri[t][0]], b = R.X[M.tri[t][1]], c = R.X[M.tri[t][2]];
        const V3<double> area = smul(0.5, cross(sub(b, a), sub(c, a)));
        const V3<double> f = vdiv(smul(M.pressure[t], area), 3.0);
        for (int k = 0; k < 3; ++k) force[M.tri[t][k]] = add(force[M.tri[t][k]], f);
    }
    if (record) T.force = force;
    Payload<double> P = R.P;
    const Payload<double> P_start = R.P;
    std::vector<double> seg_lambda(M.seg.size(), 0.0);
    if (M.susp && !integrate_payload(M, P, M.mass, R.dt, R.g)) return false;
    // predict
    std::vector<V3<double>> x = R.X, v = R.V;
    for (uint64_t i = 0; i < M.n; ++i) {
        if (M.w[i] == 0.0) {
            v[i] = {0, 0, 0};
            continue;
        }
        const V3<double> acc = add(R.g, mul(force[i], M.w[i]));
        v[i] = add(R.ref, mul(sub(add(v[i], mul(acc, R.dt)), R.ref), R.damping));
        x[i] = add(x[i], mul(v[i], R.dt));
    }
    std::vector<std::array<size_t, 2>> line_pairs;
    if (R.lines) line_pairs = line_candidates(R, x);
    if (record) {
        T.line_pairs = line_pairs;
        T.line_in.resize(static_cast<size_t>(R.iterations) * line_pairs.size());
    }
    std::vector<double> lam(M.m, 0.0), hlam(M.h, 0.0);
    if (record) {
        T.dist_in.resize(static_cast<size_t>(R.iterations) * M.m);
        T.dist_lambda.resize(static_cast<size_t>(R.iterations) * M.m);
        T.dih_in.resize(static_cast<size_t>(R.iterations) * M.h);
        T.dih_lambda.resize(static_cast<size_t>(R.iterations) * M.h);
    }
    for (int it = 0; it < R.iterations; ++it) {
        for (uint64_t i = 0; i < M.m; ++i) {
            if (record) {
                T.dist_in[it * M.m + i] = {x[M.ca[i]], x[M.cb[i]]};
                T.dist_lambda[it * M.m + i] = lam[i];
            }
            project_distance(x[M.ca[i]], x[M.cb[i]], M.w[M.ca[i]], M.w[M.cb[i]], lam[i], M.rest[i], M.comp[i],
                             M.kind[i], R.inv_dt2);
        }
        for (uint64_t i = 0; i < M.h; ++i) {
            V3<double> p[4] = {x[M.hn[i][0]], x[M.hn[i][1]], x[M.hn[i][2]], x[M.hn[i][3]]};
            const double w[4] = {M.w[M.hn[i][0]], M.w[M.hn[i][1]], M.w[M.hn[i][2]], M.w[M.hn[i][3]]};
            if (record) {
                T.dih_in[it * M.h + i] = {p[0], p[1], p[2], p[3]};
                T.dih_lambda[it * M.h + i] = hlam[i];
            }
            project_dihedral(p, w, hlam[i], M.hrest[i], M.hcomp[i], R.inv_dt2);
            for (int k = 0; k < 4; ++k) x[M.hn[i][k]] = p[k];
        }
        if (M.susp) {
            std::vector<V3<double>> xs;
            for (int node : M.att_nodes) xs.push_back(x[node]);
            if (record) {
                T.line_P.push_back(P);
                T.line_x.push_back(xs);
                T.line_lambda.push_back(seg_lambda);
            }
            std::vector<double> rest;
            for (const Seg& s : M.seg) rest.push_back(s.rest);
            if (!line_iteration(M, P, xs, seg_lambda, rest, M.mass, R.dt)) return false;
            for (size_t k = 0; k < M.att_nodes.size(); ++k) x[M.att_nodes[k]] = xs[k];
        }
        for (size_t k = 0; k < line_pairs.size(); ++k) {
            const auto& s1 = R.line_seg[line_pairs[k][0]];
            const auto& s2 = R.line_seg[line_pairs[k][1]];
            const uint64_t nd[4] = {s1[0], s1[1], s2[0], s2[1]};
            if (record) T.line_in[it * line_pairs.size() + k] = {x[nd[0]], x[nd[1]], x[nd[2]], x[nd[3]]};
            const double w[4] = {M.w[nd[0]], M.w[nd[1]], M.w[nd[2]], M.w[nd[3]]};
            project_line_pair(x[nd[0]], x[nd[1]], x[nd[2]], x[nd[3]], w, 2.0 * R.line_radius);
        }
        if (R.ground) {
            if (record) T.ground_moved.resize(static_cast<size_t>(R.iterations) * M.n, 0);
            for (uint64_t i = 0; i < M.n; ++i) {
                if (M.w[i] == 0.0) continue;
                const double c = dot(R.ground_normal, x[i]) - R.ground_offset;
                if (!(c < 0.0)) continue;
                x[i] = sub(x[i], mul(R.ground_normal, c));
                if (record) T.ground_moved[static_cast<size_t>(it) * M.n + i] = 1;
            }
        }
    }
    if (R.iterations > 0)
        for (uint64_t i : R.seams) {
            if (record) {
                T.seam_in.push_back({x[M.ca[i]], x[M.cb[i]]});
                T.seam_lambda.push_back(lam[i]);
            }
            project_distance(x[M.ca[i]], x[M.cb[i]], M.w[M.ca[i]], M.w[M.cb[i]], lam[i], M.rest[i], M.comp[i],
                             M.kind[i], R.inv_dt2);
        }
    // finalize
    const double inv = 1.0 / R.dt;
    for (uint64_t i = 0; i < M.n; ++i) v[i] = M.w[i] == 0.0 ? V3<double>{0, 0, 0} : mul(sub(x[i], R.X[i]), inv);
    if (M.susp) {
        std::vector<V3<double>> xs, vs;
        for (int node : M.att_nodes) {
            xs.push_back(x[node]);
            vs.push_back(v[node]);
        }
        if (record) {
            T.P_end = P;
            T.fin_x = xs;
            T.fin_v = vs;
            T.fin_lambda = seg_lambda;
        }
        if (!payload_finish(M, P, P_start, xs, vs, seg_lambda, M.mass, R.dt)) return false;
        for (size_t k = 0; k < M.att_nodes.size(); ++k) v[M.att_nodes[k]] = vs[k];
    }
    R.X = x;
    R.V = v;
    R.P = P;
    if (record) R.tape.push_back(std::move(T));
    return true;
}

struct Grad {
    std::vector<double> rest, comp, hcomp, seg_rest;
    double mass = 0;
};

// Reverse of one recorded step: (Xb, Vb, Pb) adjoint of the step's output
// -> adjoint of its input; parameter adjoints accumulate into G.
void reverse_step(const Rollout& R, const StepTape& T, std::vector<V3<double>>& Xb, std::vector<V3<double>>& Vb,
                  Payload<double>& Pb, Grad& G) {
    const Model& M = R.M;
    const double dt = R.dt, inv = 1.0 / dt;
    std::vector<V3<double>> xb = Xb;  // adjoint of the final positions
    std::vector<V3<double>> vb = Vb;  // adjoint of the final velocities
    std::vector<V3<double>> Xb_in(M.n, {0, 0, 0});
    Payload<double> Pb_start{{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0, 0}};
    Payload<double> Pb_it = Pb;  // adjoint of the payload after the iterations (com, q)
    const size_t na = M.att_nodes.size(), ns = M.seg.size();
    // ---- payload finish ------------------------------------------------------
    if (M.susp) {
        constexpr int N = 3 + 4 + 3 + 4 + 6 + 6 + 1;  // P_end com,q | start com,q | xs | vs | mass
        static_assert(N == 27, "layout");
        if (na > 2) {
            std::fprintf(stderr, "adjoint oracle: more than 2 attachment nodes\n");
            std::abort();
        }
        using D = Dual<N>;
        Payload<D> s, st;
        s.com = seed3<N>(T.P_end.com, 0);
        s.q = {seed<N>(T.P_end.q.w, 3), seed<N>(T.P_end.q.x, 4), seed<N>(T.P_end.q.y, 5), seed<N>(T.P_end.q.z, 6)};
        s.v = {D(0.0), D(0.0), D(0.0)};
        s.w = {D(0.0), D(0.0), D(0.0)};
        st.com = seed3<N>(T.P.com, 7);
        st.q = {seed<N>(T.P.q.w, 10), seed<N>(T.P.q.x, 11), seed<N>(T.P.q.y, 12), seed<N>(T.P.q.z, 13)};
        st.v = {D(0.0), D(0.0), D(0.0)};
        st.w = {D(0.0), D(0.0), D(0.0)};
        std::vector<V3<D>> xs, vs;
        for (size_t k = 0; k < na; ++k) {
            xs.push_back(seed3<N>(T.fin_x[k], 14 + 3 * static_cast<int>(k)));
            vs.push_back(seed3<N>(T.fin_v[k], 20 + 3 * static_cast<int>(k)));
        }
        const D mass = seed<N>(M.mass, 26);
        payload_finish(M, s, st, xs, vs, T.fin_lambda, mass, dt);
        double ub[N] = {};
        acc3(ub, s.v, Pb.v);
        acc3(ub, s.w, Pb.w);
        for (size_t k = 0; k < na; ++k) acc3(ub, vs[k], vb[M.att_nodes[k]]);
        // com and q pass through unchanged
        Pb_it.com = add(Pb.com, V3<double>{ub[0], ub[1], ub[2]});
        Pb_it.q = {Pb.q.w + ub[3], Pb.q.x + ub[4], Pb.q.y + ub[5], Pb.q.z + ub[6]};
        Pb_it.v = {0, 0, 0};
        Pb_it.w = {0, 0, 0};
        Pb_start.com = add(Pb_start.com, V3<double>{ub[7], ub[8], ub[9]});
        Pb_start.q = {Pb_start.q.w + ub[10], Pb_start.q.x + ub[11], Pb_start.q.y + ub[12], Pb_start.q.z + ub[13]};
        for (size_t k = 0; k < na; ++k) {
            xb[M.att_nodes[k]] = add(xb[M.att_nodes[k]], V3<double>{ub[14 + 3 * k], ub[15 + 3 * k], ub[16 + 3 * k]});
            vb[M.att_nodes[k]] = {ub[20 + 3 * k], ub[21 + 3 * k], ub[22 + 3 * k]};
        }
        G.mass += ub[26];
    }
    // ---- finalize --------------------------------------------------------------
    for (uint64_t i = 0; i < M.n; ++i) {
        if (M.w[i] == 0.0) continue;
        xb[i] = add(xb[i], mul(vb[i], inv));
        Xb_in[i] = sub(Xb_in[i], mul(vb[i], inv));
    }
    // ---- distance-type projection reverse ---------------------------------------
    auto dist_reverse = [&](uint64_t i, const std::array<V3<double>, 2>& in, double lam_in, double& lamb,
                            bool params) {
        constexpr int N = 9;  // xa, xb, lambda, rest, comp
        using D = Dual<N>;
        V3<D> a = seed3<N>(in[0], 0), b = seed3<N>(in[1], 3);
        D lam = seed<N>(lam_in, 6);
        const D rest = seed<N>(M.rest[i], 7), comp = seed<N>(M.comp[i], 8);
        project_distance(a, b, M.w[M.ca[i]], M.w[M.cb[i]], lam, rest, comp, M.kind[i], R.inv_dt2);
        double ub[N] = {};
        acc3(ub, a, xb[M.ca[i]]);
        acc3(ub, b, xb[M.cb[i]]);
        acc1(ub, lam, lamb);
        xb[M.ca[i]] = {ub[0], ub[1], ub[2]};
        xb[M.cb[i]] = {ub[3], ub[4], ub[5]};
        lamb = ub[6];
        if (params) {
            G.rest[i] += ub[7];
            G.comp[i] += ub[8];
        }
    };
    // ---- seam closing pass ------------------------------------------------------
    if (R.iterations > 0)
        for (size_t k = R.seams.size(); k-- > 0;) {
            double lamb = 0.0;
            dist_reverse(R.seams[k], T.seam_in[k], T.seam_lambda[k], lamb, true);
        }
    // ---- iterations -------------------------------------------------------------
    std::vector<double> lamb(M.m, 0.0), hlamb(M.h, 0.0), seglamb(ns, 0.0);
    for (int it = R.iterations - 1; it >= 0; --it) {
        // the ground plane closed the iteration: a node it moved keeps only
        // its position along the plane
        if (R.ground)
            for (uint64_t i = 0; i < M.n; ++i)
                if (T.ground_moved[static_cast<size_t>(it) * M.n + i])
                    xb[i] = sub(xb[i], mul(R.ground_normal, dot(R.ground_normal, xb[i])));
        // the line-line projections, last candidate first: each one's
        // Jacobian by forward mode at its taped inputs, its transpose applied
        // to the adjoints of its four end nodes
        for (size_t k = T.line_pairs.size(); k-- > 0;) {
            const auto& s1 = R.line_seg[T.line_pairs[k][0]];
            const auto& s2 = R.line_seg[T.line_pairs[k][1]];
            const uint64_t nd[4] = {s1[0], s1[1], s2[0], s2[1]};
            const auto& in = T.line_in[it * T.line_pairs.size() + k];
            V3<Dual<12>> q[4];
            for (int c = 0; c < 4; ++c) q[c] = seed3<12>(in[c], 3 * c);
            const double w[4] = {M.w[nd[0]], M.w[nd[1]], M.w[nd[2]], M.w[nd[3]]};
            project_line_pair(q[0], q[1], q[2], q[3], w, 2.0 * R.line_radius);
            double ob[12], ib[12] = {};
            for (int c = 0; c < 4; ++c) {
                ob[3 * c] = xb[nd[c]].x;
                ob[3 * c + 1] = xb[nd[c]].y;
                ob[3 * c + 2] = xb[nd[c]].z;
            }
            for (int c = 0; c < 4; ++c) {
                const Dual<12>* o[3] = {&q[c].x, &q[c].y, &q[c].z};
                for (int k3 = 0; k3 < 3; ++k3)
                    for (int j = 0; j < 12; ++j) ib[j] += ob[3 * c + k3] * o[k3]->d[j];
            }
            for (int c = 0; c < 4; ++c) xb[nd[c]] = {ib[3 * c], ib[3 * c + 1], ib[3 * c + 2]};
        }
        if (M.susp) {
            // inputs: com 3, q 4, lambda ns, xs 3*na, rest ns, mass 1
            constexpr int N = 3 + 4 + 2 + 6 + 2 + 1;
            if (ns > 2 || na > 2) {
                std::fprintf(stderr, "adjoint oracle: more than 2 segments\n");
                std::abort();
            }
            using D = Dual<N>;
            Payload<D> s;
            const Payload<double>& P0 = T.line_P[it];
            s.com = seed3<N>(P0.com, 0);
            s.q = {seed<N>(P0.q.w, 3), seed<N>(P0.q.x, 4), seed<N>(P0.q.y, 5), seed<N>(P0.q.z, 6)};
            s.v = {D(0.0), D(0.0), D(0.0)};
            s.w = {D(0.0), D(0.0), D(0.0)};
            std::vector<D> lam, rest;
            for (size_t k = 0; k < ns; ++k) lam.push_back(seed<N>(T.line_lambda[it][k], 7 + static_cast<int>(k)));
            std::vector<V3<D>> xs;
            for (size_t k = 0; k < na; ++k) xs.push_back(seed3<N>(T.line_x[it][k], 9 + 3 * static_cast<int>(k)));
            for (size_t k = 0; k < ns; ++k) rest.push_back(seed<N>(M.seg[k].rest, 15 + static_cast<int>(k)));
            const D mass = seed<N>(M.mass, 17);
            line_iteration(M, s, xs, lam, rest, mass, dt);
            double ub[N] = {};
            acc3(ub, s.com, Pb_it.com);
            acc1(ub, s.q.w, Pb_it.q.w);
            acc1(ub, s.q.x, Pb_it.q.x);
            acc1(ub, s.q.y, Pb_it.q.y);
            acc1(ub, s.q.z, Pb_it.q.z);
            for (size_t k = 0; k < ns; ++k) acc1(ub, lam[k], seglamb[k]);
            for (size_t k = 0; k < na; ++k) acc3(ub, xs[k], xb[M.att_nodes[k]]);
            Pb_it.com = {ub[0], ub[1], ub[2]};
            Pb_it.q = {ub[3], ub[4], ub[5], ub[6]};
            for (size_t k = 0; k < ns; ++k) seglamb[k] = ub[7 + k];
            for (size_t k = 0; k < na; ++k) xb[M.att_nodes[k]] = {ub[9 + 3 * k], ub[10 + 3 * k], ub[11 + 3 * k]};
            for (size_t k = 0; k < ns; ++k) G.seg_rest[M.seg[k].definition_index] += ub[15 + k];
            G.mass += ub[17];
        }
        for (uint64_t i = M.h; i-- > 0;) {
            constexpr int N = 14;  // 4 nodes, lambda, comp
            using D = Dual<N>;
            const auto& in = T.dih_in[it * M.h + i];
            V3<D> p[4];
            for (int k = 0; k < 4; ++k) p[k] = seed3<N>(in[k], 3 * k);
            D lam = seed<N>(T.dih_lambda[it * M.h + i], 12);
            const D comp = seed<N>(M.hcomp[i], 13);
            const double w[4] = {M.w[M.hn[i][0]], M.w[M.hn[i][1]], M.w[M.hn[i][2]], M.w[M.hn[i][3]]};
            project_dihedral(p, w, lam, D(M.hrest[i]), comp, R.inv_dt2);
            double ub[N] = {};
            for (int k = 0; k < 4; ++k) acc3(ub, p[k], xb[M.hn[i][k]]);
            acc1(ub, lam, hlamb[i]);
            for (int k = 0; k < 4; ++k) xb[M.hn[i][k]] = {ub[3 * k], ub[3 * k + 1], ub[3 * k + 2]};
            hlamb[i] = ub[12];
            G.hcomp[i] += ub[13];
        }
        for (uint64_t i = M.m; i-- > 0;) dist_reverse(i, T.dist_in[it * M.m + i], T.dist_lambda[it * M.m + i], lamb[i], true);
    }
    // ---- predict -------------------------------------------------------------------
    std::vector<V3<double>> fb(M.n, {0, 0, 0});
    std::vector<V3<double>> Vb_in(M.n, {0, 0, 0});
    for (uint64_t i = 0; i < M.n; ++i) {
        Xb_in[i] = add(Xb_in[i], xb[i]);
        if (M.w[i] == 0.0) continue;
        const V3<double> vpb = mul(xb[i], dt);          // adjoint of the predicted velocity
        Vb_in[i] = mul(vpb, R.damping);
        fb[i] = mul(vpb, R.damping * dt * M.w[i]);
    }
    // ---- pressure --------------------------------------------------------------------
    for (uint64_t t = 0; t < M.t; ++t) {
        if (M.pressure[t] == 0.0) continue;
        const uint64_t ia = M.tri[t][0], ib = M.tri[t][1], ic = M.tri[t][2];
        const V3<double> fsum = add(add(fb[ia], fb[ib]), fb[ic]);
        const V3<double> crossb = mul(fsum, M.pressure[t] / 3.0 * 0.5);
        const V3<double> u = sub(T.X[ib], T.X[ia]), w = sub(T.X[ic], T.X[ia]);
        const V3<double> ub = cross(w, crossb), wb = cross(crossb, u);
        Xb_in[ib] = add(Xb_in[ib], ub);
        Xb_in[ic] = add(Xb_in[ic], wb);
        Xb_in[ia] = sub(Xb_in[ia], add(ub, wb));
    }
    // ---- payload predict --------------------------------------------------------------
    Payload<double> Pb_in{{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0, 0}};
    if (M.susp) {
        constexpr int N = 3 + 4 + 3 + 3 + 1;
        using D = Dual<N>;
        Payload<D> s;
        s.com = seed3<N>(T.P.com, 0);
        s.q = {seed<N>(T.P.q.w, 3), seed<N>(T.P.q.x, 4), seed<N>(T.P.q.y, 5), seed<N>(T.P.q.z, 6)};
        s.v = seed3<N>(T.P.v, 7);
        s.w = seed3<N>(T.P.w, 10);
        const D mass = seed<N>(M.mass, 13);
        integrate_payload(M, s, mass, dt, R.g);
        double ub[N] = {};
        acc3(ub, s.com, Pb_it.com);
        acc1(ub, s.q.w, Pb_it.q.w);
        acc1(ub, s.q.x, Pb_it.q.x);
        acc1(ub, s.q.y, Pb_it.q.y);
        acc1(ub, s.q.z, Pb_it.q.z);
        Pb_in.com = add(Pb_start.com, V3<double>{ub[0], ub[1], ub[2]});
        Pb_in.q = {Pb_start.q.w + ub[3], Pb_start.q.x + ub[4], Pb_start.q.y + ub[5], Pb_start.q.z + ub[6]};
        Pb_in.v = {ub[7], ub[8], ub[9]};
        Pb_in.w = {ub[10], ub[11], ub[12]};
        G.mass += ub[13];
    }
    Xb = Xb_in;
    Vb = Vb_in;
    Pb = Pb_in;
}

thread_local std::string g_err;

}  // namespace

// ---- C interface (loaded by oracle/oracle.py) ----------------------------------
extern "C" {

const char* swa_last_error() { return g_err.c_str(); }

// Runs `steps` steps of the definition (its own insertion order is the sweep
// order) from `state` (node_count x (position xyz, velocity xyz), nullable:
// the definition's positions at rest) and `payload` (com xyz, orientation
// wxyz, linear and angular velocity xyz; nullable: the definition's initial
// pilot) with `forces` (node_count xyz, nullable) as the constant external
// load.  `step_states` / `step_payloads` (nullable; steps x node_count x 6
// and steps x 13 in the same layouts) restart every step s > 0 from a given
// trajectory, so that the reverse sweep runs along another solver's states.
// `ground` (nullable: none) is a frictionless ground plane (normal xyz, offset).
// `lines` (nullable: none) is line-line contact of the cable segments
// (radius, margin).
// Then evaluates the loss against `target` (node_count xyz) with node weights `weights` and its gradient.  Outputs
// (nullable): final positions (node_count xyz), d rest / d compliance per
// constraint, d compliance per dihedral, d rest per suspension segment
// (definition order), d pilot mass.  Returns 0 on success.
int swa_rollout_gradient(const swb_structure_definition* def, const swb_step_settings* st, int steps,
                         const double* state, const double* payload, const double* step_states,
                         const double* step_payloads, const double* forces, const double* target,
                         const double* weights, double* loss,
                         double* final_xyz, double* d_rest, double* d_comp, double* d_dihedral_comp,
                         double* d_segment_rest, double* d_mass, const double* ground, const double* lines) {
    try {
        Rollout R;
        if (!build_model(*def, R.M, g_err)) return 1;
        if (st->substeps != 1) {
            g_err = "one substep per step";
            return 1;
        }
        const Model& M = R.M;
        R.dt = st->time_step;
        R.inv_dt2 = 1.0 / (R.dt * R.dt);
        R.damping = std::exp(-st->velocity_damping * R.dt);
        R.g = fromabi(st->gravity);
        R.ref = fromabi(st->damping_reference_velocity);
        R.iterations = st->constraint_iterations;
        if (ground) {
            R.ground = true;
            R.ground_normal = {ground[0], ground[1], ground[2]};
            R.ground_offset = ground[3];
        }
        if (lines) {
            R.lines = true;
            R.line_radius = lines[0];
            R.line_reach = lines[0] + 0.5 * lines[1];
            for (uint64_t i = 0; i < M.m; ++i)
                if (M.kind[i] == SWB_CONSTRAINT_CABLE)
                    R.line_seg.push_back({std::min(M.ca[i], M.cb[i]), std::max(M.ca[i], M.cb[i])});
            std::sort(R.line_seg.begin(), R.line_seg.end());
            R.line_seg.erase(std::unique(R.line_seg.begin(), R.line_seg.end()), R.line_seg.end());
        }
        if (forces)
            for (uint64_t i = 0; i < M.n; ++i) R.M.pending[i] = {forces[3 * i], forces[3 * i + 1], forces[3 * i + 2]};
        for (uint64_t i = 0; i < M.m; ++i)
            if (M.kind[i] == SWB_CONSTRAINT_SEAM_STITCH) R.seams.push_back(i);
        R.X = M.x0;
        R.V = M.v0;
        R.P = {M.p_com, M.p_v, M.p_w, M.p_q};
        if (state)
            for (uint64_t i = 0; i < M.n; ++i) {
                R.X[i] = {state[6 * i], state[6 * i + 1], state[6 * i + 2]};
                R.V[i] = {state[6 * i + 3], state[6 * i + 4], state[6 * i + 5]};
            }
        if (payload && M.susp) {
            R.P.com = {payload[0], payload[1], payload[2]};
            R.P.q = {payload[3], payload[4], payload[5], payload[6]};
            R.P.v = {payload[7], payload[8], payload[9]};
            R.P.w = {payload[10], payload[11], payload[12]};
        }
        for (int s = 0; s < steps; ++s) {
            // optionally restart every step from a given trajectory (node
            // position and velocity, pilot), so that the reverse sweep is
            // evaluated along another solver's states
            if (step_states && s > 0)
                for (uint64_t i = 0; i < M.n; ++i) {
                    const double* q = step_states + (static_cast<size_t>(s) * M.n + i) * 6;
                    R.X[i] = {q[0], q[1], q[2]};
                    R.V[i] = {q[3], q[4], q[5]};
                }
            if (step_payloads && s > 0 && M.susp) {
                const double* q = step_payloads + static_cast<size_t>(s) * 13;
                R.P.com = {q[0], q[1], q[2]};
                R.P.q = {q[3], q[4], q[5], q[6]};
                R.P.v = {q[7], q[8], q[9]};
                R.P.w = {q[10], q[11], q[12]};
            }
            if (!forward_step(R, true)) {
                g_err = "forward step failed";
                return 1;
            }
        }
        double wsum = 0.0, L = 0.0;
        std::vector<V3<double>> Xb(M.n, {0, 0, 0}), Vb(M.n, {0, 0, 0});
        for (uint64_t i = 0; i < M.n; ++i) wsum += weights[i];
        for (uint64_t i = 0; i < M.n; ++i) {
            const V3<double> d = sub(R.X[i], V3<double>{target[3 * i], target[3 * i + 1], target[3 * i + 2]});
            L += weights[i] * dot(d, d);
            Xb[i] = mul(d, 2.0 * weights[i] / wsum);
        }
        if (loss) *loss = L / wsum;
        if (final_xyz)
            for (uint64_t i = 0; i < M.n; ++i) {
                final_xyz[3 * i] = R.X[i].x;
                final_xyz[3 * i + 1] = R.X[i].y;
                final_xyz[3 * i + 2] = R.X[i].z;
            }
        Grad G;
        G.rest.assign(M.m, 0.0);
        G.comp.assign(M.m, 0.0);
        G.hcomp.assign(M.h, 0.0);
        G.seg_rest.assign(M.seg.size(), 0.0);
        Payload<double> Pb{{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0, 0}};
        for (int s = steps - 1; s >= 0; --s) reverse_step(R, R.tape[s], Xb, Vb, Pb, G);
        if (d_rest) std::copy(G.rest.begin(), G.rest.end(), d_rest);
        if (d_comp) std::copy(G.comp.begin(), G.comp.end(), d_comp);
        if (d_dihedral_comp) std::copy(G.hcomp.begin(), G.hcomp.end(), d_dihedral_comp);
        if (d_segment_rest) std::copy(G.seg_rest.begin(), G.seg_rest.end(), d_segment_rest);
        if (d_mass) *d_mass = G.mass;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

}  // extern "C"
