// Checks the adjoint arithmetic of simwing_b200/csrc/adjoint_math.h on the
// host in double precision:
//  * dist_reverse and dihedral_reverse against central finite differences
//    of dist_forward / dihedral_forward, for every input (positions, lambda,
//    rest, compliance) and random output adjoints, in the regimes the
//    projections have (plain, cable taut, cable released, slack cable);
//  * the dual-number instantiations of the rigid-pilot functions against
//    central finite differences of their double instantiations.
// Prints one line per check; exits non-zero on the first failure.
#include "../../simwing_b200/csrc/adjoint_math.h"

#include <cstdio>
#include <random>
#include <vector>

using namespace swb::adj;

namespace {

int failures = 0;
std::mt19937_64 rng(7);
double gauss() { return std::normal_distribution<double>(0.0, 1.0)(rng); }
V3<double> gv(double s = 1.0) { return {s * gauss(), s * gauss(), s * gauss()}; }

void check(const char* what, double got, double want, double tol) {
    const double err = std::fabs(got - want) / std::max(1.0, std::fabs(want));
    const bool ok = err <= tol;
    if (!ok) {
        std::printf("FAIL %s: adjoint %.12e finite difference %.12e (error %.2e)\n", what, got, want, err);
        ++failures;
    }
}

// ---- distance ---------------------------------------------------------------
// `kink_lambda`: lambda sits on the slack cable's switch (lambda == 0 with
// the cable short), where the projection is not differentiable in lambda;
// that input is not compared.
void distance_case(const char* name, V3<double> a, V3<double> b, double lambda, double rest, double comp, bool cable,
                   bool kink_lambda = false) {
    const double wa = 2.0, wb = 3.0, inv_dt2 = 14400.0;
    const V3<double> ga = gv(), gb = gv();
    const double gl = gauss();
    auto f = [&](std::vector<double> u) {
        V3<double> A{u[0], u[1], u[2]}, B{u[3], u[4], u[5]};
        double l = u[6];
        dist_forward(A, B, wa, wb, l, u[7], u[8], cable, inv_dt2);
        return dot(ga, A) + dot(gb, B) + gl * l;
    };
    const std::vector<double> u0 = {a.x, a.y, a.z, b.x, b.y, b.z, lambda, rest, comp};
    DistanceGrad<double> g{ga, gb, gl, 0, 0};
    dist_reverse(a, b, wa, wb, lambda, rest, comp, cable, inv_dt2, g);
    const double adj[9] = {g.a.x, g.a.y, g.a.z, g.b.x, g.b.y, g.b.z, g.lambda, g.rest, g.comp};
    for (int j = 0; j < 9; ++j) {
        if (kink_lambda && j == 6) continue;
        const double h = j == 8 ? 1e-4 * comp : 1e-7;  // relative step for the compliance
        std::vector<double> up = u0, um = u0;
        up[j] += h;
        um[j] -= h;
        const double fd = (f(up) - f(um)) / (2 * h);
        char what[96];
        std::snprintf(what, sizeof what, "distance %s input %d", name, j);
        check(what, adj[j], fd, 1e-6);
    }
    std::printf("ok   distance %s\n", name);
}

// ---- dihedral ----------------------------------------------------------------
void dihedral_case(const char* name, const V3<double> p0[4], double lambda, double rest, double comp) {
    const double w[4] = {1.5, 2.0, 0.7, 3.0}, inv_dt2 = 14400.0;
    V3<double> gp[4];
    for (auto& v : gp) v = gv();
    const double gl = gauss();
    auto f = [&](std::vector<double> u) {
        V3<double> p[4];
        for (int k = 0; k < 4; ++k) p[k] = {u[3 * k], u[3 * k + 1], u[3 * k + 2]};
        double l = u[12];
        dihedral_forward(p, w, l, u[13], u[14], inv_dt2);
        double s = gl * l;
        for (int k = 0; k < 4; ++k) s += dot(gp[k], p[k]);
        return s;
    };
    std::vector<double> u0;
    for (int k = 0; k < 4; ++k) u0.insert(u0.end(), {p0[k].x, p0[k].y, p0[k].z});
    u0.insert(u0.end(), {lambda, rest, comp});
    DihedralGrad<double> G;
    for (int k = 0; k < 4; ++k) G.p[k] = gp[k];
    G.lambda = gl;
    dihedral_reverse(p0, w, lambda, rest, comp, inv_dt2, G);
    double adj[15];
    for (int k = 0; k < 4; ++k) {
        adj[3 * k] = G.p[k].x;
        adj[3 * k + 1] = G.p[k].y;
        adj[3 * k + 2] = G.p[k].z;
    }
    adj[12] = G.lambda;
    adj[13] = G.rest;
    adj[14] = G.comp;
    for (int j = 0; j < 15; ++j) {
        const double h = j == 14 ? 1e-4 * comp : 1e-7;
        std::vector<double> up = u0, um = u0;
        up[j] += h;
        um[j] -= h;
        const double fd = (f(up) - f(um)) / (2 * h);
        char what[96];
        std::snprintf(what, sizeof what, "dihedral %s input %d", name, j);
        check(what, adj[j], fd, 2e-6);
    }
    std::printf("ok   dihedral %s\n", name);
}

// ---- rigid pilot: dual numbers against finite differences -----------------------
PilotDef<double> pilot() {
    PilotDef<double> d{};
    d.com_local = {0.1, 0.0, -0.2};
    d.inertia = {12.0, 10.0, 6.0};
    d.segments = 2;
    for (int k = 0; k < 2; ++k) {
        d.from_node[k] = k;
        d.to_node[k] = -1;
        d.from_point[k] = -1;
        d.to_point[k] = k;
        d.stiffness[k] = 4e5;
        d.damping[k] = 40.0;
        d.hang_local[k] = {0.1 + (k ? 0.2 : -0.2), k ? 0.25 : -0.25, 0.2};
    }
    d.min_length = 1e-10;
    return d;
}

template <class T>
Q4<T> unitq(double w, double x, double y, double z) {
    const double n = std::sqrt(w * w + x * x + y * y + z * z);
    return {T(w / n), T(x / n), T(y / n), T(z / n)};
}

void pilot_checks() {
    const PilotDef<double> d = pilot();
    const double dt = 1.0 / 120.0;
    const V3<double> g = {0, 0, -9.81};
    const double ws[2] = {50.0, 60.0};
    // base state: pilot 0.45 m below two attachment nodes, lines slightly stretched
    const V3<double> com = {0.12, 0.01, -6.98};
    const Q4<double> q = unitq<double>(0.999, 0.02, -0.01, 0.03);
    const V3<double> v = {0.3, -0.1, -0.5}, w = {0.05, -0.02, 0.1};
    const V3<double> xs0[2] = {{0.0, -0.3, -6.4}, {0.3, 0.3, -6.45}};
    const V3<double> vs0[2] = {{0.2, 0.1, -0.4}, {0.1, -0.2, -0.6}};
    const double mass = 90.0;
    // input vector: com 3, q 4, v 3, w 3, xs 6, vs 6, lambda 2, rest 2, mass 1, start com 3, start q 4
    std::vector<double> u0 = {com.x, com.y, com.z, q.w, q.x, q.y, q.z, v.x, v.y, v.z, w.x, w.y, w.z};
    for (auto& x : xs0) u0.insert(u0.end(), {x.x, x.y, x.z});
    for (auto& x : vs0) u0.insert(u0.end(), {x.x, x.y, x.z});
    u0.insert(u0.end(), {0.01, 0.0, 0.45, 0.44, mass, 0.1, 0.0, -6.97});
    const Q4<double> q0 = unitq<double>(0.9995, 0.015, -0.012, 0.02);
    u0.insert(u0.end(), {q0.w, q0.x, q0.y, q0.z});
    const int nin = static_cast<int>(u0.size());
    std::vector<double> ybar(64);
    for (auto& y : ybar) y = gauss();

    // evaluates all three functions with scalar T, seeded along direction `dir`
    // (-1: none), returns the adjoint-weighted sum of the outputs
    auto run = [&](auto tag, const std::vector<double>& u, int dir, int which) {
        using T = decltype(tag);
        auto in = [&](int j) -> T {
            if constexpr (std::is_same_v<T, double>) return u[j];
            else return T(u[j], j == dir ? 1.0 : 0.0);
        };
        PilotState<T> s{{in(0), in(1), in(2)}, {in(7), in(8), in(9)}, {in(10), in(11), in(12)},
                        {in(3), in(4), in(5), in(6)}};
        V3<T> xs[2] = {{in(13), in(14), in(15)}, {in(16), in(17), in(18)}};
        V3<T> vs[2] = {{in(19), in(20), in(21)}, {in(22), in(23), in(24)}};
        T lam[2] = {in(25), in(26)};
        const T rest[2] = {in(27), in(28)};
        const T m = in(29);
        PilotState<T> start{{in(30), in(31), in(32)}, {T(0), T(0), T(0)}, {T(0), T(0), T(0)},
                            {in(33), in(34), in(35), in(36)}};
        T acc = T(0);
        int k = 0;
        auto add3 = [&](const V3<T>& a) {
            acc = acc + a.x * ybar[k] + a.y * ybar[k + 1] + a.z * ybar[k + 2];
            k += 3;
        };
        auto addq = [&](const Q4<T>& a) {
            acc = acc + a.w * ybar[k] + a.x * ybar[k + 1] + a.y * ybar[k + 2] + a.z * ybar[k + 3];
            k += 4;
        };
        bool ok = true;
        if (which == 0) {
            ok = payload_predict_t(d, s, m, dt, g);
            add3(s.com); addq(s.q); add3(s.v); add3(s.w);
        } else if (which == 1) {
            ok = line_iteration_t(d, s, xs, ws, lam, rest, m, dt);
            add3(s.com); addq(s.q); add3(xs[0]); add3(xs[1]);
            acc = acc + lam[0] * ybar[k] + lam[1] * ybar[k + 1];
        } else {
            const double lam_sign[2] = {1.0, 1.0};
            ok = payload_finish_t(d, s, start, xs, vs, ws, lam_sign, m, dt);
            add3(s.v); add3(s.w); add3(vs[0]); add3(vs[1]);
        }
        if (!ok) {
            std::printf("FAIL pilot function %d rejected its input\n", which);
            ++failures;
        }
        return acc;
    };
    const char* names[3] = {"payload predict", "line iteration", "payload finish"};
    for (int which = 0; which < 3; ++which) {
        for (int j = 0; j < nin; ++j) {
            const Dual<double> dv = run(Dual<double>(), u0, j, which);
            const double h = 1e-7;
            std::vector<double> up = u0, um = u0;
            up[j] += h;
            um[j] -= h;
            const double fd = (run(0.0, up, -1, which) - run(0.0, um, -1, which)) / (2 * h);
            char what[96];
            std::snprintf(what, sizeof what, "%s input %d", names[which], j);
            check(what, dv.d, fd, 2e-6);
        }
        std::printf("ok   %s\n", names[which]);
    }
}

}  // namespace

int main() {
    // distance: plain constraint stretched and compressed, cable taut, cable
    // released by the clamp, slack cable (skipped: identity)
    distance_case("stretched", {0, 0, 0}, {1.02, 0.03, -0.01}, -0.002, 1.0, 1e-6, false);
    distance_case("compressed", {0.1, 0, 0}, {0.95, 0.1, 0.02}, 0.001, 1.0, 1e-6, false);
    distance_case("cable taut", {0, 0, 0}, {1.01, 0.02, 0}, -0.001, 1.0, 1e-6, true);
    distance_case("cable released", {0, 0, 0}, {0.99, 0.02, 0}, -0.00001, 1.0, 1e-6, true);
    distance_case("cable slack", {0, 0, 0}, {0.9, 0.02, 0}, 0.0, 1.0, 1e-6, true, true);
    // dihedral: folded, nearly flat, strongly bent
    {
        const V3<double> p[4] = {{0, 0, 0}, {1, 0.1, 0}, {0.4, 0.9, 0.1}, {0.5, -0.8, 0.3}};
        dihedral_case("folded", p, 0.01, 0.2, 1e-3);
    }
    {
        const V3<double> p[4] = {{0, 0, 0}, {1, 0, 0.05}, {0.5, 1, 0.01}, {0.5, -1, -0.02}};
        dihedral_case("flat", p, -0.003, 0.0, 1e-3);
    }
    {
        const V3<double> p[4] = {{0, 0, 0}, {0.8, 0.3, 0}, {0.2, 0.5, 0.7}, {0.6, 0.1, 0.9}};
        dihedral_case("bent", p, 0.0, -0.5, 1e-2);
    }
    pilot_checks();
    return failures == 0 ? 0 : 1;
}
