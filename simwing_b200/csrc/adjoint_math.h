// Reverse-mode (adjoint) arithmetic of the XPBD step, shared by the device
// adjoint kernel and its host-side unit test.
//
//  * dist_reverse / dihedral_reverse: hand-written vector-Jacobian products
//    of one distance-type projection (soft_body.cpp:1598-1640) and one
//    dihedral projection (soft_body.cpp:1648-1711, 1754-1792) in the form
//    the device evaluates them (closed-form dihedral gradient), including
//    the compliance multiplier update.
//  * payload_predict_t / line_iteration_t / payload_finish_t: the rigid
//    pilot's prediction (suspension.cpp:1075-1102), unilateral line
//    iteration (suspension.cpp:2197-2274) and velocity reconstruction with
//    line damping (suspension.cpp:2386-2479), generic in the scalar type so
//    that a dual-number instantiation yields their Jacobians (forward mode,
//    one input direction per lane).
//
// Everything is templated on the scalar type and compiles as host code
// (g++) and device code (nvcc).
#pragma once

#include <cmath>
#include <cstdint>

#include "fast_math.h"

#if defined(__CUDACC__)
#define SWB_HD __host__ __device__ __forceinline__
#else
#define SWB_HD inline
#endif

namespace swb {
namespace adj {

// ---- scalars -------------------------------------------------------------------
template <class S>
struct Dual {
    S v, d;  // value and one directional derivative
    SWB_HD Dual() : v(0), d(0) {}
    SWB_HD Dual(S x) : v(x), d(0) {}  // NOLINT: constants promote
    SWB_HD Dual(S x, S dx) : v(x), d(dx) {}
};
template <class S> SWB_HD S val(S x) { return x; }
template <class S> SWB_HD S val(const Dual<S>& x) { return x.v; }

template <class S> SWB_HD Dual<S> operator+(Dual<S> a, Dual<S> b) { return {a.v + b.v, a.d + b.d}; }
template <class S> SWB_HD Dual<S> operator-(Dual<S> a, Dual<S> b) { return {a.v - b.v, a.d - b.d}; }
template <class S> SWB_HD Dual<S> operator-(Dual<S> a) { return {-a.v, -a.d}; }
template <class S> SWB_HD Dual<S> operator*(Dual<S> a, Dual<S> b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
template <class S> SWB_HD Dual<S> operator/(Dual<S> a, Dual<S> b) {
    const S r = a.v / b.v;
    return {r, (a.d - r * b.d) / b.v};
}
template <class S> SWB_HD Dual<S> operator+(Dual<S> a, S b) { return {a.v + b, a.d}; }
template <class S> SWB_HD Dual<S> operator+(S a, Dual<S> b) { return {a + b.v, b.d}; }
template <class S> SWB_HD Dual<S> operator-(Dual<S> a, S b) { return {a.v - b, a.d}; }
template <class S> SWB_HD Dual<S> operator-(S a, Dual<S> b) { return {a - b.v, -b.d}; }
template <class S> SWB_HD Dual<S> operator*(Dual<S> a, S b) { return {a.v * b, a.d * b}; }
template <class S> SWB_HD Dual<S> operator*(S a, Dual<S> b) { return {a * b.v, a * b.d}; }
template <class S> SWB_HD Dual<S> operator/(Dual<S> a, S b) { return {a.v / b, a.d / b}; }
template <class S> SWB_HD Dual<S> operator/(S a, Dual<S> b) {
    const S r = a / b.v;
    return {r, -r * b.d / b.v};
}

// math on plain scalars (float uses the single-precision functions)
#if defined(__CUDA_ARCH__)
SWB_HD float m_sqrt(float x) { return sqrtf(x); }
SWB_HD double m_sqrt(double x) { return sqrt(x); }
SWB_HD float m_sin(float x) { return sinf(x); }
SWB_HD double m_sin(double x) { return sin(x); }
SWB_HD float m_cos(float x) { return cosf(x); }
SWB_HD double m_cos(double x) { return cos(x); }
SWB_HD float m_atan2(float y, float x) { return atan2f(y, x); }
SWB_HD double m_atan2(double y, double x) { return atan2(y, x); }
SWB_HD float m_fabs(float x) { return fabsf(x); }
SWB_HD double m_fabs(double x) { return fabs(x); }
SWB_HD float m_copysign(float a, float b) { return copysignf(a, b); }
SWB_HD double m_copysign(double a, double b) { return copysign(a, b); }
SWB_HD float m_rint(float x) { return rintf(x); }
SWB_HD double m_rint(double x) { return rint(x); }
SWB_HD bool m_isfinite(float x) { return isfinite(x); }
SWB_HD bool m_isfinite(double x) { return isfinite(x); }
#else
template <class S> inline S m_sqrt(S x) { return std::sqrt(x); }
template <class S> inline S m_sin(S x) { return std::sin(x); }
template <class S> inline S m_cos(S x) { return std::cos(x); }
template <class S> inline S m_atan2(S y, S x) { return std::atan2(y, x); }
template <class S> inline S m_fabs(S x) { return std::fabs(x); }
template <class S> inline S m_copysign(S a, S b) { return std::copysign(a, b); }
template <class S> inline S m_rint(S x) { return std::rint(x); }
template <class S> inline bool m_isfinite(S x) { return std::isfinite(x); }
#endif

// The projections' scalar forms: in float the device step's own (approximate
// reciprocal, reciprocal square root, fast atan2), so that the reverse sweep
// recomputes exactly the forward values the step produced; in double exact.
SWB_HD float p_rcp(float x) { return fast_rcp(x); }
SWB_HD double p_rcp(double x) { return 1.0 / x; }
SWB_HD float p_rsqrt(float x) {
#if defined(__CUDA_ARCH__)
    return rsqrtf(x);
#else
    return 1.0f / std::sqrt(x);
#endif
}
SWB_HD double p_rsqrt(double x) { return 1.0 / m_sqrt(x); }
SWB_HD float p_atan2(float y, float x) { return fast_atan2(y, x); }
SWB_HD double p_atan2(double y, double x) { return m_atan2(y, x); }

template <class S> SWB_HD Dual<S> m_sqrt(Dual<S> a) {
    const S s = m_sqrt(a.v);
    return {s, a.d * S(0.5) / s};
}
template <class S> SWB_HD Dual<S> m_sin(Dual<S> a) { return {m_sin(a.v), a.d * m_cos(a.v)}; }
template <class S> SWB_HD Dual<S> m_cos(Dual<S> a) { return {m_cos(a.v), -a.d * m_sin(a.v)}; }
template <class S> SWB_HD Dual<S> m_atan2(Dual<S> y, Dual<S> x) {
    const S den = x.v * x.v + y.v * y.v;
    return {m_atan2(y.v, x.v), (x.v * y.d - y.v * x.d) / den};
}
template <class S> SWB_HD Dual<S> m_fabs(Dual<S> a) { return a.v < S(0) ? -a : a; }
template <class S> SWB_HD Dual<S> m_copysign(Dual<S> a, Dual<S> b) {
    return (a.v < S(0)) != (b.v < S(0)) ? -a : a;
}

// ---- vectors -------------------------------------------------------------------
template <class T> struct V3 { T x, y, z; };
template <class T> SWB_HD V3<T> operator+(const V3<T>& a, const V3<T>& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> SWB_HD V3<T> operator-(const V3<T>& a, const V3<T>& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> SWB_HD V3<T> operator-(const V3<T>& a) { return {-a.x, -a.y, -a.z}; }
template <class T, class U> SWB_HD V3<T> operator*(const V3<T>& a, const U& s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T, class U> SWB_HD V3<T> operator/(const V3<T>& a, const U& s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> SWB_HD T dot(const V3<T>& a, const V3<T>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> SWB_HD V3<T> cross(const V3<T>& a, const V3<T>& b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> SWB_HD T length(const V3<T>& a) { return m_sqrt(dot(a, a)); }
template <class T> SWB_HD bool finite3(const V3<T>& a) {
    return m_isfinite(val(a.x)) && m_isfinite(val(a.y)) && m_isfinite(val(a.z));
}

// ---- distance-type projection: forward and vector-Jacobian product ----------
// Inputs a, b (positions), wa, wb (inverse masses), lambda, rest, compliance
// (>= 0), cable flag.  Forward as the device step evaluates it.
template <class S>
struct DistanceGrad {
    V3<S> a, b;      // in: adjoints of the outputs; out: of the inputs
    S lambda;        // in: adjoint of lambda'; out: of lambda
    S rest, comp;    // out: adjoints of the rest length and the compliance
};

template <class S>
SWB_HD void dist_forward(V3<S>& a, V3<S>& b, S wa, S wb, S& lambda, S rest, S comp, bool cable, S inv_dt2) {
    const V3<S> d = b - a;
    const S l2 = dot(d, d);
    const S k = S(1.0e-12);
    if (!(l2 > k * k)) return;
    const S il = p_rsqrt(l2);
    const S l = l2 * il;
    if (l <= k) return;
    const S value = l - rest;
    if (cable && value <= S(0) && lambda == S(0)) return;
    const S W = wa + wb, alpha = comp * inv_dt2;
    if (W + alpha <= S(0)) return;
    const S dl = (-value - alpha * lambda) * p_rcp(W + alpha);
    S applied = dl;
    if (cable) {
        const S s = lambda + dl;
        const S nl = s < S(0) ? s : S(0);
        applied = nl - lambda;
        lambda = nl;
    } else {
        lambda = lambda + dl;
    }
    const S scale = applied * il;
    a = a - d * (wa * scale);
    b = b + d * (wb * scale);
}

// g holds the output adjoints on entry and the input adjoints on return.
template <class S>
SWB_HD void dist_reverse(V3<S> a, V3<S> b, S wa, S wb, S lambda, S rest, S comp, bool cable, S inv_dt2,
                         DistanceGrad<S>& g) {
    g.rest = S(0);
    g.comp = S(0);
    const V3<S> d = b - a;
    const S l2 = dot(d, d);
    const S k = S(1.0e-12);
    if (!(l2 > k * k)) return;
    const S il = p_rsqrt(l2);
    const S l = l2 * il;
    if (l <= k) return;
    const S value = l - rest;
    if (cable && value <= S(0) && lambda == S(0)) return;
    const S W = wa + wb, alpha = comp * inv_dt2;
    if (W + alpha <= S(0)) return;
    const S inv = p_rcp(W + alpha);
    const S dl = (-value - alpha * lambda) * inv;
    bool active = true;  // lambda' = lambda + dl, applied = dl
    S applied = dl;
    if (cable && !(lambda + dl < S(0))) {
        active = false;  // lambda' = 0, applied = -lambda
        applied = -lambda;
    }
    const S scale = applied * il;
    // a' = a - wa scale d, b' = b + wb scale d
    const S sbar = -wa * dot(d, g.a) + wb * dot(d, g.b);
    V3<S> dbar = (g.b * wb - g.a * wa) * scale;
    const S appliedbar = sbar * il;
    const S ilbar = sbar * applied;
    S dlbar = S(0), lambar = S(0);
    if (active) {
        dlbar = appliedbar + g.lambda;
        lambar = g.lambda;
    } else {
        lambar = -appliedbar;
    }
    const S valuebar = -dlbar * inv;
    lambar = lambar - alpha * dlbar * inv;
    const S alphabar = (-lambda - dl) * dlbar * inv;
    g.comp = alphabar * inv_dt2;
    g.rest = -valuebar;
    // l = |d|, il = 1/|d|
    dbar = dbar + d * (il * (valuebar - ilbar * il * il));
    g.a = g.a - dbar;
    g.b = g.b + dbar;
    g.lambda = lambar;
}

// ---- dihedral projection: forward and vector-Jacobian product ----------------
template <class S>
SWB_HD S wrap_2pi(S x) {
    const S two_pi = S(6.28318530717958647692);
    const S n = m_rint(x / two_pi);
    return x - n * two_pi;
}
// float: the device step's form (a branch within one turn, else remainderf)
SWB_HD float wrap_2pi(float x) {
    const float two_pi = 6.28318530717958647692f, half = 0.5f * two_pi;
    if (fabsf(x) <= two_pi) return x > half ? x - two_pi : (x < -half ? x + two_pi : x);
    return remainderf(x, two_pi);
}

template <class S>
struct DihedralGrad {
    V3<S> p[4];   // in: adjoints of the outputs; out: of the inputs
    S lambda;     // in/out
    S rest, comp; // out
};

template <class S>
SWB_HD void dihedral_forward(V3<S> p[4], const S w[4], S& lambda, S rest, S comp, S inv_dt2) {
    const V3<S> e = p[1] - p[0], u = p[2] - p[0], v = p[3] - p[0];
    const V3<S> A1 = cross(e, u), A2 = cross(v, e);
    const S e2 = dot(e, e), q1 = dot(A1, A1), q2 = dot(A2, A2);
    const S k2 = S(1.0e-24);
    if (!(e2 > k2) || !(q1 > k2 * e2) || !(q2 > k2 * e2)) return;
    const S iel = p_rsqrt(e2);
    const S el = e2 * iel;
    const S Sv = dot(e, cross(A1, A2)) * iel;
    const S Cv = dot(A1, A2);
    const S rq1 = p_rcp(q1), rq2 = p_rcp(q2);
    const S s1 = -el * rq1, s2 = -el * rq2;
    const V3<S> gc = A1 * s1, gd = A2 * s2;
    const S ie2 = iel * iel;
    const S t1 = dot(u, e) * ie2, t2 = dot(v, e) * ie2;
    const V3<S> gb = -(gc * t1 + gd * t2);
    const V3<S> ga = -((gb + gc) + gd);
    const V3<S> g[4] = {ga, gb, gc, gd};
    const S theta = p_atan2(Sv, Cv);
    S wg = S(0);
    for (int k = 0; k < 4; ++k) wg = wg + w[k] * dot(g[k], g[k]);
    const S alpha = comp * inv_dt2;
    const S den = wg + alpha;
    if (!(den > S(0)) || !m_isfinite(den)) return;
    const S value = wrap_2pi(theta - rest);
    const S dl = (-value - alpha * lambda) * p_rcp(den);
    if (!m_isfinite(dl)) return;
    for (int k = 0; k < 4; ++k) p[k] = p[k] + g[k] * (w[k] * dl);
    lambda = lambda + dl;
}

template <class S>
SWB_HD void dihedral_reverse(const V3<S> p[4], const S w[4], S lambda, S rest, S comp, S inv_dt2,
                             DihedralGrad<S>& G) {
    G.rest = S(0);
    G.comp = S(0);
    const V3<S> e = p[1] - p[0], u = p[2] - p[0], v = p[3] - p[0];
    const V3<S> A1 = cross(e, u), A2 = cross(v, e);
    const S e2 = dot(e, e), q1 = dot(A1, A1), q2 = dot(A2, A2);
    const S k2 = S(1.0e-24);
    if (!(e2 > k2) || !(q1 > k2 * e2) || !(q2 > k2 * e2)) return;
    const S iel = p_rsqrt(e2);
    const S el = e2 * iel;
    const V3<S> P = cross(A1, A2);
    const S Tv = dot(e, P);
    const S Sv = Tv * iel;
    const S Cv = dot(A1, A2);
    const S rq1 = p_rcp(q1), rq2 = p_rcp(q2);
    const S s1 = -el * rq1, s2 = -el * rq2;
    const V3<S> gc = A1 * s1, gd = A2 * s2;
    const S ie2 = iel * iel;
    const S ue = dot(u, e), ve = dot(v, e);
    const S t1 = ue * ie2, t2 = ve * ie2;
    const V3<S> gb = -(gc * t1 + gd * t2);
    const V3<S> ga = -((gb + gc) + gd);
    const V3<S> g[4] = {ga, gb, gc, gd};
    const S theta = p_atan2(Sv, Cv);
    S wg = S(0);
    for (int k = 0; k < 4; ++k) wg = wg + w[k] * dot(g[k], g[k]);
    const S alpha = comp * inv_dt2;
    const S den = wg + alpha;
    if (!(den > S(0)) || !m_isfinite(den)) return;
    const S iden = p_rcp(den);
    const S value = wrap_2pi(theta - rest);
    const S dl = (-value - alpha * lambda) * iden;
    if (!m_isfinite(dl)) return;
    // outputs: p_k' = p_k + w_k dl g_k, lambda' = lambda + dl
    S dlbar = G.lambda;
    V3<S> gbar[4];
    for (int k = 0; k < 4; ++k) {
        dlbar = dlbar + w[k] * dot(g[k], G.p[k]);
        gbar[k] = G.p[k] * (w[k] * dl);
    }
    S lambar = G.lambda;
    const S valuebar = -dlbar * iden;
    lambar = lambar - alpha * dlbar * iden;
    const S denbar = -dl * dlbar * iden;
    const S alphabar = -lambda * dlbar * iden + denbar;
    G.comp = alphabar * inv_dt2;
    G.rest = -valuebar;
    const S thetabar = valuebar;
    // wg
    for (int k = 0; k < 4; ++k) gbar[k] = gbar[k] + g[k] * (S(2) * w[k] * denbar);
    // theta = atan2(Sv, Cv)
    const S ir2 = p_rcp(Sv * Sv + Cv * Cv);
    const S Svbar = thetabar * Cv * ir2;
    const S Cvbar = -thetabar * Sv * ir2;
    // ga = -(gb + gc + gd)
    V3<S> gbb = gbar[1] - gbar[0], gcb = gbar[2] - gbar[0], gdb = gbar[3] - gbar[0];
    // gb = -(t1 gc + t2 gd)
    const S t1bar = -dot(gbb, gc), t2bar = -dot(gbb, gd);
    gcb = gcb - gbb * t1;
    gdb = gdb - gbb * t2;
    // t1 = ue ie2, t2 = ve ie2
    const S uebar = t1bar * ie2, vebar = t2bar * ie2;
    S ie2bar = t1bar * ue + t2bar * ve;
    V3<S> ebar = u * uebar + v * vebar;
    V3<S> ubar = e * uebar;
    V3<S> vbar = e * vebar;
    // gc = s1 A1, gd = s2 A2
    const S s1bar = dot(gcb, A1), s2bar = dot(gdb, A2);
    V3<S> A1bar = gcb * s1;
    V3<S> A2bar = gdb * s2;
    // s1 = -el / q1, s2 = -el / q2
    S elbar = -s1bar * rq1 - s2bar * rq2;
    const S q1bar = s1bar * el * rq1 * rq1;
    const S q2bar = s2bar * el * rq2 * rq2;
    // Cv = A1 . A2
    A1bar = A1bar + A2 * Cvbar;
    A2bar = A2bar + A1 * Cvbar;
    // Sv = (e . P) iel, P = A1 x A2
    const S Tbar = Svbar * iel;
    S ielbar = Svbar * Tv;
    ebar = ebar + P * Tbar;
    const V3<S> Pbar = e * Tbar;
    A1bar = A1bar + cross(A2, Pbar);
    A2bar = A2bar + cross(Pbar, A1);
    // ie2 = iel^2, el = e2 iel, iel = e2^-1/2
    ielbar = ielbar + S(2) * iel * ie2bar + elbar * e2;
    S e2bar = elbar * iel - S(0.5) * ielbar * iel * iel * iel;
    // q1 = A1.A1, q2 = A2.A2, e2 = e.e
    A1bar = A1bar + A1 * (S(2) * q1bar);
    A2bar = A2bar + A2 * (S(2) * q2bar);
    ebar = ebar + e * (S(2) * e2bar);
    // A1 = e x u, A2 = v x e
    ebar = ebar + cross(u, A1bar) + cross(A2bar, v);
    ubar = ubar + cross(A1bar, e);
    vbar = vbar + cross(e, A2bar);
    // e = p1 - p0, u = p2 - p0, v = p3 - p0
    G.p[1] = G.p[1] + ebar;
    G.p[2] = G.p[2] + ubar;
    G.p[3] = G.p[3] + vbar;
    G.p[0] = G.p[0] - ((ebar + ubar) + vbar);
    G.lambda = lambar;
}

// ---- rigid pilot, generic in the scalar type ------------------------------------
template <class T> struct Q4 { T w, x, y, z; };
template <class T> struct M3T { T m[9]; };

// The pilot's constant data as the generic functions use it.
template <class S>
struct PilotDef {
    V3<S> com_local;
    V3<S> inertia;        // principal, body frame
    int segments;
    int from_node[8], to_node[8], from_point[8], to_point[8];  // node: attachment slot index or -1
    S stiffness[8], damping[8];
    V3<S> hang_local[8];
    S min_length;
};

template <class T> SWB_HD Q4<T> q_mul(const Q4<T>& a, const Q4<T>& b) {
    return {a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z, a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
            a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x, a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w};
}
template <class T> SWB_HD bool q_canon(const Q4<T>& q, Q4<T>& out) {
    const T n2 = q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z;
    if (!(val(n2) > 1.0e-28)) return false;
    const T inv = T(1) / m_sqrt(n2);
    Q4<T> r = {q.w * inv, q.x * inv, q.y * inv, q.z * inv};
    const bool flip = val(r.w) < 0 || (val(r.w) == 0 && (val(r.x) < 0 || (val(r.x) == 0 && (val(r.y) < 0 ||
                                                                                          (val(r.y) == 0 && val(r.z) < 0)))));
    if (flip) r = {-r.w, -r.x, -r.y, -r.z};
    out = r;
    return true;
}
template <class T> SWB_HD bool q_rotation(const Q4<T>& o, M3T<T>& R) {
    Q4<T> q;
    if (!q_canon(o, q)) return false;
    const T xx = q.x * q.x, yy = q.y * q.y, zz = q.z * q.z, xy = q.x * q.y, xz = q.x * q.z, yz = q.y * q.z;
    const T wx = q.w * q.x, wy = q.w * q.y, wz = q.w * q.z;
    const T one = T(1), two = T(2);
    R.m[0] = one - two * (yy + zz); R.m[1] = two * (xy - wz); R.m[2] = two * (xz + wy);
    R.m[3] = two * (xy + wz); R.m[4] = one - two * (xx + zz); R.m[5] = two * (yz - wx);
    R.m[6] = two * (xz - wy); R.m[7] = two * (yz + wx); R.m[8] = one - two * (xx + yy);
    return true;
}
template <class T> SWB_HD V3<T> m3v(const M3T<T>& m, const V3<T>& v) {
    return {m.m[0] * v.x + m.m[1] * v.y + m.m[2] * v.z, m.m[3] * v.x + m.m[4] * v.y + m.m[5] * v.z,
            m.m[6] * v.x + m.m[7] * v.y + m.m[8] * v.z};
}
template <class T> SWB_HD bool q_increment(const V3<T>& r, Q4<T>& out) {
    const T angle = length(r);
    if (val(angle) < 1.0e-12) return q_canon(Q4<T>{T(1), r.x * T(0.5), r.y * T(0.5), r.z * T(0.5)}, out);
    const T half = T(0.5) * angle;
    const T s = m_sin(half) / angle;
    out = {m_cos(half), r.x * s, r.y * s, r.z * s};
    return true;
}
template <class T, class S> SWB_HD M3T<T> world_inertia(const M3T<T>& R, const V3<S>& I) {
    M3T<T> out;
    const S d[3] = {I.x, I.y, I.z};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            T s = T(0);
            for (int k = 0; k < 3; ++k) s = s + R.m[i * 3 + k] * d[k] * R.m[j * 3 + k];
            out.m[i * 3 + j] = s;
        }
    return out;
}
template <class T> SWB_HD bool m3_inverse(const M3T<T>& m, M3T<T>& out) {
    T scale = T(0);
    for (int i = 0; i < 9; ++i)
        if (m_fabs(val(m.m[i])) > val(scale)) scale = m_fabs(m.m[i]);
    if (!(val(scale) > 0)) return false;
    M3T<T> n;
    const T is = T(1) / scale;
    for (int i = 0; i < 9; ++i) n.m[i] = m.m[i] * is;
    const T c00 = n.m[4] * n.m[8] - n.m[5] * n.m[7];
    const T c01 = n.m[2] * n.m[7] - n.m[1] * n.m[8];
    const T c02 = n.m[1] * n.m[5] - n.m[2] * n.m[4];
    const T det = n.m[0] * c00 + n.m[3] * c01 + n.m[6] * c02;
    if (!(m_fabs(val(det)) > 1.0e-14)) return false;
    const T f = T(1) / (det * scale);
    out.m[0] = c00 * f; out.m[1] = c01 * f; out.m[2] = c02 * f;
    out.m[3] = (n.m[5] * n.m[6] - n.m[3] * n.m[8]) * f;
    out.m[4] = (n.m[0] * n.m[8] - n.m[2] * n.m[6]) * f;
    out.m[5] = (n.m[2] * n.m[3] - n.m[0] * n.m[5]) * f;
    out.m[6] = (n.m[3] * n.m[7] - n.m[4] * n.m[6]) * f;
    out.m[7] = (n.m[1] * n.m[6] - n.m[0] * n.m[7]) * f;
    out.m[8] = (n.m[0] * n.m[4] - n.m[1] * n.m[3]) * f;
    return true;
}

template <class T>
struct PilotState {
    V3<T> com, v, w;
    Q4<T> q;
};

// integratePayloadTorqueFree with force m g and no moment.
template <class T, class S>
SWB_HD bool payload_predict_t(const PilotDef<S>& d, PilotState<T>& s, const T& mass, S dt, const V3<S>& g) {
    Q4<T> q;
    if (!q_canon(s.q, q)) return false;
    s.q = q;
    M3T<T> R, invI;
    if (!q_rotation(s.q, R)) return false;
    M3T<T> I = world_inertia(R, d.inertia);
    const V3<T> L = m3v(I, s.w);
    const V3<T> force = {mass * g.x, mass * g.y, mass * g.z};
    s.v = s.v + force * (T(dt) / mass);
    if (!m3_inverse(I, invI)) return false;
    s.w = m3v(invI, L);
    s.com = s.com + s.v * T(dt);
    Q4<T> inc;
    if (!q_increment(s.w * T(dt), inc)) return false;
    if (!q_canon(q_mul(inc, s.q), s.q)) return false;
    if (!q_rotation(s.q, R)) return false;
    I = world_inertia(R, d.inertia);
    if (!m3_inverse(I, invI)) return false;
    s.w = m3v(invI, L);
    return true;
}

template <class T, class S>
SWB_HD bool pilot_point(const PilotDef<S>& d, const PilotState<T>& s, const V3<S>& local, V3<T>& out) {
    M3T<T> R;
    if (!q_rotation(s.q, R)) return false;
    const V3<S> l = local - d.com_local;
    out = s.com + m3v(R, V3<T>{T(l.x), T(l.y), T(l.z)});
    return true;
}

// One line iteration.  xs[k] = position of attachment slot k; ws[k] its
// inverse mass; lam/rest per segment.
template <class T, class S>
SWB_HD bool line_iteration_t(const PilotDef<S>& d, PilotState<T>& s, V3<T>* xs, const S* ws, T* lam,
                             const T* rest, const T& mass, S dt) {
    M3T<T> R, invI;
    if (!q_rotation(s.q, R)) return false;
    const M3T<T> I = world_inertia(R, d.inertia);
    if (!m3_inverse(I, invI)) return false;
    const T wp = T(1) / mass;
    for (int k = 0; k < d.segments; ++k) {
        V3<T> p[2], off[2];
        T w[2];
        bool rigid[2], fixed[2];
        const int node[2] = {d.from_node[k], d.to_node[k]};
        const int point[2] = {d.from_point[k], d.to_point[k]};
        for (int e = 0; e < 2; ++e) {
            off[e] = {T(0), T(0), T(0)};
            if (node[e] >= 0) {
                p[e] = xs[node[e]];
                w[e] = T(ws[node[e]]);
                fixed[e] = ws[node[e]] == S(0);
                rigid[e] = false;
            } else {
                if (!pilot_point(d, s, d.hang_local[point[e]], p[e])) return false;
                off[e] = p[e] - s.com;
                rigid[e] = true;
                fixed[e] = false;
                w[e] = wp;
            }
        }
        const V3<T> diff = p[1] - p[0];
        const T l = length(diff);
        if (!(val(l) > val(d.min_length))) return false;
        const V3<T> dir = diff / l;
        const V3<T> grad[2] = {dir, -dir};
        T eff = T(0);
        for (int e = 0; e < 2; ++e) {
            T r = w[e];
            if (rigid[e] && !fixed[e] && val(w[e]) > 0) {
                const V3<T> rot = cross(off[e], grad[e]);
                r = r + dot(rot, m3v(invI, rot));
            }
            eff = eff + r;
        }
        const S at = S(1) / (d.stiffness[k] * dt * dt);
        const T gap = rest[k] - l;
        const T cand = lam[k] + (-gap - T(at) * lam[k]) / (eff + T(at));
        const T acc = val(cand) > 0 ? cand : T(0);
        const T inc = acc - lam[k];
        lam[k] = acc;
        for (int e = 0; e < 2; ++e) {
            if (fixed[e]) continue;
            if (node[e] >= 0) {
                xs[node[e]] = xs[node[e]] + grad[e] * (w[e] * inc);
            } else {
                s.com = s.com + grad[e] * (w[e] * inc);
                const V3<T> rot = m3v(invI, cross(off[e], grad[e])) * inc;
                Q4<T> qi;
                if (!q_increment(rot, qi) || !q_canon(q_mul(qi, s.q), s.q)) return false;
            }
        }
    }
    return true;
}

// Velocity reconstruction and bounded line damping.  xs/vs: attachment
// slot positions and velocities; lam: segment multipliers (sign only).
template <class T, class S>
SWB_HD bool payload_finish_t(const PilotDef<S>& d, PilotState<T>& s, const PilotState<T>& start, const V3<T>* xs,
                             V3<T>* vs, const S* ws, const S* lam, const T& mass, S dt) {
    s.v = (s.com - start.com) / T(dt);
    const Q4<T> conj = {start.q.w, -start.q.x, -start.q.y, -start.q.z};
    Q4<T> delta;
    if (!q_canon(q_mul(s.q, conj), delta)) return false;
    const T sn = m_sqrt(delta.x * delta.x + delta.y * delta.y + delta.z * delta.z);
    const T half = m_atan2(sn, delta.w);
    if (val(sn) < 1.0e-12) {
        s.w = V3<T>{delta.x, delta.y, delta.z} * T(S(2) / dt);
    } else {
        s.w = V3<T>{delta.x, delta.y, delta.z} * (T(2) * half / (T(dt) * sn));
    }
    M3T<T> R, invI;
    if (!q_rotation(s.q, R)) return false;
    const M3T<T> I = world_inertia(R, d.inertia);
    if (!m3_inverse(I, invI)) return false;
    for (int k = 0; k < d.segments; ++k) {
        if (!(lam[k] > S(0)) || !(d.damping[k] > S(0))) continue;
        V3<T> pts[2], vel[2];
        const int node[2] = {d.from_node[k], d.to_node[k]};
        const int point[2] = {d.from_point[k], d.to_point[k]};
        for (int e = 0; e < 2; ++e) {
            if (node[e] >= 0) {
                pts[e] = xs[node[e]];
                vel[e] = vs[node[e]];
            } else {
                const V3<S> l = d.hang_local[point[e]] - d.com_local;
                const V3<T> offset = m3v(R, V3<T>{T(l.x), T(l.y), T(l.z)});
                pts[e] = s.com + offset;
                vel[e] = s.v + cross(s.w, offset);
            }
        }
        const V3<T> df = pts[1] - pts[0];
        const T m = length(df);
        const V3<T> dir = val(m) > 0 ? df / m : V3<T>{T(0), T(0), T(0)};
        const T rel = dot(vel[1] - vel[0], dir);
        T eff = T(0);
        for (int e = 0; e < 2; ++e) {
            if (node[e] >= 0) {
                eff = eff + T(ws[node[e]]);
            } else {
                const V3<T> rxn = cross(pts[e] - s.com, dir);
                eff = eff + (T(1) / mass + dot(rxn, m3v(invI, rxn)));
            }
        }
        if (!(val(eff) > 0) || val(rel) == 0) continue;
        const T req = T(d.damping[k]) * m_fabs(rel) * T(dt);
        const T stop = m_fabs(rel) / eff;
        const T mag = m_copysign(val(stop) < val(req) ? stop : req, rel);
        const V3<T> imp[2] = {dir * mag, -(dir * mag)};
        for (int e = 0; e < 2; ++e) {
            if (node[e] >= 0) {
                if (ws[node[e]] > S(0)) vs[node[e]] = vs[node[e]] + imp[e] * T(ws[node[e]]);
            } else {
                s.v = s.v + imp[e] / mass;
                s.w = s.w + m3v(invI, cross(pts[e] - s.com, imp[e]));
            }
        }
    }
    return true;
}

}  // namespace adj
}  // namespace swb
