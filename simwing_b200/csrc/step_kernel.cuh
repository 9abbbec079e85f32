// Persistent XPBD step kernel (one launch per substep).
//
// Restates, in FP32 on the device, the reference substep
// SoftBody::integrateSubstepTrial (src/softwing/soft_body.cpp:1175-1460):
//   prologue   accumulatePressureForces (gather form, ascending triangle
//              order, :1511-1533), SuspensionSystem::beginSubstep payload
//              prediction (suspension.cpp:2170-2181), predictPositions
//              (:1536-1566), multiplier reset (:1207-1218);
//   iterations distance/cable/tie/seam sweep (projectDistanceConstraint
//              :1598-1640), dihedral sweep (solveDihedralConstraint
//              :1754-1792), suspension line iteration
//              (suspension.cpp:2197-2274);
//   epilogue   final seam-stitch projections (:1389-1405),
//              finalizeVelocities (:1568-1585), payload velocity
//              reconstruction, line damping and certification
//              (suspension.cpp:2324-2479), payload line wrench (:2582-2589).
// The sweep order is the schedule's (see schedule.h); it equals the
// reference's serial sweep with its constraint lists permuted into it.
#pragma once

#include "fast_math.h"
#include "step_params.h"

namespace swb {
namespace dev {

constexpr float kMinimumLengthF = 1.0e-12f;
constexpr float kTwoPiF = 6.28318530717958647692f;

// remainder(x, 2*pi) as IEEE remainderf(x, kTwoPiF).  For |x| <= kTwoPiF the
// quotient rounds to n in {-1, 0, 1} (a tie at |x| = pi rounds to the even
// n = 0) and x - n*kTwoPiF is exact by Sterbenz' lemma, so the fast path
// returns the same bits as remainderf; larger |x| takes remainderf.
__device__ __forceinline__ float wrap_two_pi(float x) {
    const float half = 0.5f * kTwoPiF;
    if (fabsf(x) <= kTwoPiF) return x > half ? x - kTwoPiF : (x < -half ? x + kTwoPiF : x);
    return remainderf(x, kTwoPiF);
}

// projectDistanceConstraint (soft_body.cpp:1598-1640) on float4 nodes
// (xyz, w = inverse mass).  comp carries the cable flag in its sign bit.
// The length and the two divisions use the reciprocal square root and the
// approximate reciprocal (an ulp or two each) instead of IEEE sqrt and
// division.
__device__ __forceinline__ void project_distance(float4& pa, float4& pb, float rest, float comp_raw,
                                                 float& lambda, float inv_dt2) {
    const float dx = pb.x - pa.x, dy = pb.y - pa.y, dz = pb.z - pa.z;
    const float l2 = dx * dx + dy * dy + dz * dz;
    if (!(l2 > kMinimumLengthF * kMinimumLengthF)) return;
    const float il = rsqrtf(l2);
    const float l = l2 * il;
    if (l <= kMinimumLengthF) return;
    const float value = l - rest;
    const bool cable = signbit(comp_raw);
    if (cable && value <= 0.0f && lambda == 0.0f) return;
    const float wsum = pa.w + pb.w;
    const float alpha = fabsf(comp_raw) * inv_dt2;
    if (wsum + alpha <= 0.0f) return;
    const float dl = (-value - alpha * lambda) * fast_rcp(wsum + alpha);
    float applied = dl;
    if (cable) {
        const float sum = lambda + dl;
        const float nl = sum < 0.0f ? sum : 0.0f;  // std::min(0.0, x)
        applied = nl - lambda;
        lambda = nl;
    } else {
        lambda += dl;
    }
    const float scale = applied * il;
    const float sa = pa.w * scale, sb = pb.w * scale;
    pa.x -= sa * dx; pa.y -= sa * dy; pa.z -= sa * dz;
    pb.x += sb * dx; pb.y += sb * dy; pb.z += sb * dz;
}

// evaluateDihedral + solveDihedralConstraint (soft_body.cpp:1648-1711,
// 1754-1792): one XPBD projection of the signed hinge angle.
//
// The angle uses fast_atan2 (fast_math.h, within 4e-7 rad of atan2) and the
// divisions the approximate reciprocal.
// The reference evaluates theta = atan2(e.(n1 x n2), n1.n2) from unit
// vectors and its gradient by reverse mode through the normalisations.  The
// same function and gradient are evaluated here in closed form (an identity,
// checked against the reference evaluation in the tests): with the face
// areas A1 = e x (c - a), A2 = (d - a) x e and the hinge e = b - a,
//   theta = atan2(e.(A1 x A2) / |e|, A1.A2)      (atan2 is scale-invariant),
//   grad_c = -|e| / |A1|^2 A1,   grad_d = -|e| / |A2|^2 A2,
//   grad_b = -t1 grad_c - t2 grad_d,   grad_a = -(grad_b + grad_c + grad_d),
// where t1, t2 are the projections of c and d on the hinge
// ((c - a).e / |e|^2, (d - a).e / |e|^2).  The degeneracy gates are the
// reference's (|e|, |A1|/|e|, |A2|/|e| above 1e-12).
__device__ __forceinline__ void project_dihedral(float4& A, float4& B, float4& C, float4& D, float rest,
                                                 float comp, float& lambda, float inv_dt2) {
    const float3 a = f3(A), b = f3(B), c = f3(C), d = f3(D);
    const float3 edge = b - a;
    const float3 toC = c - a;
    const float3 toD = d - a;
    const float3 A1 = cross(edge, toC);
    const float3 A2 = cross(toD, edge);
    const float e2 = dot(edge, edge), q1 = dot(A1, A1), q2 = dot(A2, A2);
    const float k2 = kMinimumLengthF * kMinimumLengthF;
    if (!(e2 > k2) || !(q1 > k2 * e2) || !(q2 > k2 * e2)) return;
    const float iel = rsqrtf(e2);
    const float el = e2 * iel;
    const float sine = dot(edge, cross(A1, A2)) * iel;
    const float cosine = dot(A1, A2);
    const float s1 = -el * fast_rcp(q1), s2 = -el * fast_rcp(q2);
    const float3 gc = A1 * s1;
    const float3 gd = A2 * s2;
    const float ie2 = iel * iel;
    const float t1 = dot(toC, edge) * ie2, t2 = dot(toD, edge) * ie2;
    const float3 gb = -(gc * t1 + gd * t2);
    const float3 ga = -((gb + gc) + gd);
    const float angle = fast_atan2(sine, cosine);
    // The reference skips a hinge whose angle or gradient is not finite.  A
    // non-finite gradient component makes wg (and den) non-finite, and a
    // non-finite angle makes dl non-finite, so the two checks below reject
    // exactly those cases without testing each component.
    const float wg = A.w * dot(ga, ga) + B.w * dot(gb, gb) + C.w * dot(gc, gc) + D.w * dot(gd, gd);
    const float alpha = comp * inv_dt2;
    const float den = wg + alpha;
    if (!(den > 0.0f) || !isfinite(den) || !isfinite(wg)) return;
    const float value = wrap_two_pi(angle - rest);
    const float dl = (-value - alpha * lambda) * fast_rcp(den);
    if (!isfinite(dl)) return;
    const float sa = A.w * dl, sb = B.w * dl, sc = C.w * dl, sd = D.w * dl;
    A.x += sa * ga.x; A.y += sa * ga.y; A.z += sa * ga.z;
    B.x += sb * gb.x; B.y += sb * gb.y; B.z += sb * gb.z;
    C.x += sc * gc.x; C.y += sc * gc.y; C.z += sc * gc.z;
    D.x += sd * gd.x; D.y += sd * gd.y; D.z += sd * gd.z;
    lambda += dl;
}

// ---- rigid payload (suspension.cpp:538-690, 1018-1163) in FP32 -----------
struct M3 { float m[9]; };

__device__ __forceinline__ float4 q_mul(float4 a, float4 b) {
    return make_float4(a.x * b.x - a.y * b.y - a.z * b.z - a.w * b.w,
                       a.x * b.y + a.y * b.x + a.z * b.w - a.w * b.z,
                       a.x * b.z - a.y * b.w + a.z * b.x + a.w * b.y,
                       a.x * b.w + a.y * b.z - a.z * b.y + a.w * b.x);
}
// float4 quaternion layout: (x=w, y=x, z=y, w=z)
__device__ __forceinline__ bool q_canon(float4 q, float4& out) {
    const float n2 = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
    if (!isfinite(q.x) || !isfinite(q.y) || !isfinite(q.z) || !isfinite(q.w) || !(n2 > 1.0e-28f)) return false;
    const float inv = rsqrtf(n2);
    float4 r = make_float4(q.x * inv, q.y * inv, q.z * inv, q.w * inv);
    const bool flip = r.x < 0.0f ||
                      (r.x == 0.0f && (r.y < 0.0f || (r.y == 0.0f && (r.z < 0.0f || (r.z == 0.0f && r.w < 0.0f)))));
    if (flip) r = make_float4(-r.x, -r.y, -r.z, -r.w);
    out = r;
    return true;
}
__device__ __forceinline__ bool q_rotation(float4 o, M3& R) {
    float4 q;
    if (!q_canon(o, q)) return false;
    const float w = q.x, x = q.y, y = q.z, z = q.w;
    const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z;
    const float wx = w * x, wy = w * y, wz = w * z;
    R.m[0] = 1.0f - 2.0f * (yy + zz); R.m[1] = 2.0f * (xy - wz); R.m[2] = 2.0f * (xz + wy);
    R.m[3] = 2.0f * (xy + wz); R.m[4] = 1.0f - 2.0f * (xx + zz); R.m[5] = 2.0f * (yz - wx);
    R.m[6] = 2.0f * (xz - wy); R.m[7] = 2.0f * (yz + wx); R.m[8] = 1.0f - 2.0f * (xx + yy);
    return true;
}
__device__ __forceinline__ float3 m3v(const M3& m, float3 v) {
    return make_float3(m.m[0] * v.x + m.m[1] * v.y + m.m[2] * v.z, m.m[3] * v.x + m.m[4] * v.y + m.m[5] * v.z,
                       m.m[6] * v.x + m.m[7] * v.y + m.m[8] * v.z);
}
// rotationIncrement (suspension.cpp:669-684).  Below a half angle of 0.02
// rad (an iteration's increment is far smaller) sin(h) / (2 h) and cos(h)
// come from their Taylor series to h^4 and h^6: the truncation error is
// under 1e-14 relative, below FP32 rounding.
__device__ __forceinline__ bool q_increment(float3 r, float4& out) {
    if (!finite3(r)) return false;
    const float angle = length(r);
    if (angle < 1.0e-12f) return q_canon(make_float4(1.0f, 0.5f * r.x, 0.5f * r.y, 0.5f * r.z), out);
    const float half = 0.5f * angle;
    float s, c;
    if (half < 0.02f) {
        const float h2 = half * half;
        s = 0.5f * (1.0f - h2 * (1.0f / 6.0f - h2 * (1.0f / 120.0f)));
        c = 1.0f - h2 * (0.5f - h2 * (1.0f / 24.0f - h2 * (1.0f / 720.0f)));
    } else {
        s = sinf(half) / angle;
        c = cosf(half);
    }
    out = make_float4(c, r.x * s, r.y * s, r.z * s);
    return true;
}
// R diag(I) R^T
__device__ __forceinline__ M3 world_inertia(const M3& R, float3 I) {
    M3 out;
    const float d[3] = {I.x, I.y, I.z};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            float s = 0.0f;
            for (int k = 0; k < 3; ++k) s += R.m[i * 3 + k] * d[k] * R.m[j * 3 + k];
            out.m[i * 3 + j] = s;
        }
    return out;
}
// Mat3 inverse with max-magnitude scaling (suspension.cpp:567-595).
__device__ __forceinline__ bool m3_inverse(const M3& m, M3& out) {
    float scale = 0.0f;
    for (int i = 0; i < 9; ++i) scale = fmaxf(scale, fabsf(m.m[i]));
    if (!(scale > 0.0f) || !isfinite(scale)) return false;
    M3 n;
    const float is = 1.0f / scale;
    for (int i = 0; i < 9; ++i) n.m[i] = m.m[i] * is;
    const float c00 = n.m[4] * n.m[8] - n.m[5] * n.m[7];
    const float c01 = n.m[2] * n.m[7] - n.m[1] * n.m[8];
    const float c02 = n.m[1] * n.m[5] - n.m[2] * n.m[4];
    const float det = n.m[0] * c00 + n.m[3] * c01 + n.m[6] * c02;
    if (!isfinite(det) || fabsf(det) <= 1.0e-14f) return false;
    const float f = 1.0f / (det * scale);
    out.m[0] = c00 * f; out.m[1] = c01 * f; out.m[2] = c02 * f;
    out.m[3] = (n.m[5] * n.m[6] - n.m[3] * n.m[8]) * f;
    out.m[4] = (n.m[0] * n.m[8] - n.m[2] * n.m[6]) * f;
    out.m[5] = (n.m[2] * n.m[3] - n.m[0] * n.m[5]) * f;
    out.m[6] = (n.m[3] * n.m[7] - n.m[4] * n.m[6]) * f;
    out.m[7] = (n.m[1] * n.m[6] - n.m[0] * n.m[7]) * f;
    out.m[8] = (n.m[0] * n.m[4] - n.m[1] * n.m[3]) * f;
    return true;
}

__device__ __forceinline__ void susp_fail(int* status, int code) {
    if (atomicOr(status, kStatusSuspension) == 0) status[1] = code;
    else atomicCAS(status + 1, 0, code);
}

// integratePayloadTorqueFree (suspension.cpp:1075-1102) with force
// m*g and no applied wrench (the structural adapter applies none).
__device__ bool payload_predict(const DevPayloadDef& d, DevPayloadState& s, float dt, float3 g) {
    float4 q;
    if (!q_canon(s.q, q)) return false;
    s.q = q;
    M3 R, I, invI;
    if (!q_rotation(s.q, R)) return false;
    I = world_inertia(R, d.inertia);
    float3 L = m3v(I, s.w);
    const float3 force = g * d.mass;
    s.v = s.v + force * (dt / d.mass);
    if (!m3_inverse(I, invI)) return false;
    s.w = m3v(invI, L);
    s.com = s.com + s.v * dt;
    float4 inc;
    if (!q_increment(s.w * dt, inc)) return false;
    if (!q_canon(q_mul(inc, s.q), s.q)) return false;
    if (!q_rotation(s.q, R)) return false;
    I = world_inertia(R, d.inertia);
    if (!m3_inverse(I, invI)) return false;
    s.w = m3v(invI, L);
    return finite3(s.com) && finite3(s.v) && finite3(s.w);
}

__device__ __forceinline__ bool payload_point(const DevPayloadDef& d, const DevPayloadState& s, float3 local,
                                              float3& out) {
    M3 R;
    if (!q_rotation(s.q, R)) return false;
    out = s.com + m3v(R, local - d.com_local);
    return true;
}

// solveLineIteration (suspension.cpp:2197-2274): serial unilateral
// projection of every segment with the rigid-endpoint effective mass.
// Nodes are level-1 local indices into x (the owner CTA's patch).
__device__ __noinline__ void line_iteration(const DevPayloadDef& d, DevPayloadState& s, float4* x, float dt, int* status) {
    M3 R, I, invI;
    if (!q_rotation(s.q, R)) { susp_fail(status, kSuspOrientation); return; }
    I = world_inertia(R, d.inertia);
    if (!m3_inverse(I, invI)) { susp_fail(status, kSuspEffectiveMass); return; }
    const float wp = 1.0f / d.mass;
    for (int k = 0; k < d.segments; ++k) {
        float3 p[2], off[2];
        float w[2];
        bool rigid[2], fixed[2];
        const int node[2] = {d.from_node[k], d.to_node[k]};
        const int point[2] = {d.from_point[k], d.to_point[k]};
        for (int e = 0; e < 2; ++e) {
            off[e] = make_float3(0.0f, 0.0f, 0.0f);
            if (node[e] >= 0) {
                const float4 X = x[node[e]];
                p[e] = f3(X);
                w[e] = X.w;
                fixed[e] = X.w == 0.0f;
                rigid[e] = false;
            } else {
                if (!payload_point(d, s, d.hang_local[point[e]], p[e])) { susp_fail(status, kSuspOrientation); return; }
                off[e] = p[e] - s.com;
                rigid[e] = true;
                fixed[e] = false;
                w[e] = wp;
            }
        }
        const float3 diff = p[1] - p[0];
        const float l = length(diff);
        if (!isfinite(l) || l <= d.min_length) { susp_fail(status, kSuspLineGeometry | ((k + 1) << 8)); return; }
        const float3 dir = diff * fast_rcp(l);
        const float lam = s.lambda[k];
        // projectUnilateralLine (suspension.cpp:1125-1163).  The unit-gradient
        // check uses an FP32 tolerance.
        if (!(l > 0.0f) || !(d.rest[k] > 0.0f) || !(d.stiffness[k] > 0.0f) || !(lam >= 0.0f) || !isfinite(lam) ||
            fabsf(length(dir) - 1.0f) > 1.0e-5f) {
            susp_fail(status, kSuspLineInput);
            return;
        }
        const float3 grad[2] = {dir, -dir};
        float eff = 0.0f;
        for (int e = 0; e < 2; ++e) {
            float r = w[e];
            if (rigid[e] && !fixed[e] && w[e] > 0.0f) {
                const float3 rot = cross(off[e], grad[e]);
                r += dot(rot, m3v(invI, rot));
            }
            eff += r;
        }
        const float at = fast_rcp(d.stiffness[k] * dt * dt);
        if (!(eff + at > 0.0f)) { susp_fail(status, kSuspEffectiveMass); return; }
        const float gap = d.rest[k] - l;
        const float cand = lam + (-gap - at * lam) * fast_rcp(eff + at);
        const float acc = 0.0f < cand ? cand : 0.0f;
        const float inc = acc - lam;
        s.lambda[k] = acc;
        for (int e = 0; e < 2; ++e) {
            if (fixed[e]) continue;
            if (node[e] >= 0) {
                float4 X = x[node[e]];
                const float sc = w[e] * inc;
                X.x += grad[e].x * sc; X.y += grad[e].y * sc; X.z += grad[e].z * sc;
                x[node[e]] = X;
            } else {
                s.com = s.com + grad[e] * (w[e] * inc);
                const float3 rot = m3v(invI, cross(off[e], grad[e])) * inc;
                float4 qi;
                if (!q_increment(rot, qi) || !q_canon(q_mul(qi, s.q), s.q)) { susp_fail(status, kSuspOrientation); return; }
            }
        }
    }
}

// reconstructPayloadVelocity, applyLineDamping, certifySubstep and the
// payload line wrench of finishSubstep (suspension.cpp:2324-2589).  The
// half angle of the orientation increment is evaluated as
// atan2(|xyz|, w), which equals the reference's acos(w) on unit
// quaternions and keeps FP32 accuracy for small rotations.
// A suspension endpoint's position and velocity: a node, or a harness point
// of the payload.
__device__ __forceinline__ bool payload_endpoint(const DevPayloadDef& d, const DevPayloadState& s, const float4* x,
                                                 const float4* v, int node, int point, float3& pos, float3& vel) {
    if (node >= 0) {
        pos = f3(x[node]);
        vel = f3(v[node]);
        return true;
    }
    const float3 local = d.hang_local[point] - d.com_local;
    M3 RR;
    if (!q_rotation(s.q, RR)) return false;
    const float3 offset = m3v(RR, local);
    pos = s.com + offset;
    vel = s.v + cross(s.w, offset);
    return true;
}

// reconstructPayloadVelocity and applyLineDamping (suspension.cpp:2413-2479):
// the first half of the payload's substep finish.  Returns false after a
// failure (status set).
__device__ bool payload_reconstruct_damp(const DevPayloadDef& d, DevPayloadState& s, const DevPayloadState& start,
                                         const float4* x, float4* v, float dt, int* status) {
    s.v = (s.com - start.com) / dt;
    float4 delta;
    const float4 conj = make_float4(start.q.x, -start.q.y, -start.q.z, -start.q.w);
    if (!q_canon(q_mul(s.q, conj), delta)) { susp_fail(status, kSuspFinish); return false; }
    const float sn = sqrtf(delta.y * delta.y + delta.z * delta.z + delta.w * delta.w);
    const float half = atan2f(sn, delta.x);
    if (sn < 1.0e-12f) {
        s.w = make_float3(delta.y, delta.z, delta.w) * (2.0f / dt);
    } else {
        s.w = make_float3(delta.y, delta.z, delta.w) * (2.0f * half / (dt * sn));
    }
    M3 R, I, invI;
    if (!q_rotation(s.q, R)) { susp_fail(status, kSuspFinish); return false; }
    I = world_inertia(R, d.inertia);
    if (!m3_inverse(I, invI)) { susp_fail(status, kSuspFinish); return false; }
    auto endpoint = [&](int node, int point, float3& pos, float3& vel) -> bool {
        return payload_endpoint(d, s, x, v, node, point, pos, vel);
    };
    // applyLineDamping (suspension.cpp:2413-2479)
    for (int k = 0; k < d.segments; ++k) {
        if (!(s.lambda[k] > 0.0f) || !(d.damping[k] > 0.0f)) continue;
        float3 from, to, vf, vt;
        if (!endpoint(d.from_node[k], d.from_point[k], from, vf) || !endpoint(d.to_node[k], d.to_point[k], to, vt)) {
            susp_fail(status, kSuspFinish);
            return false;
        }
        const float3 df = to - from;
        const float m = length(df);
        const float3 dir = m > 0.0f ? df / m : make_float3(0.0f, 0.0f, 0.0f);
        const float rel = dot(vt - vf, dir);
        float eff = 0.0f;
        const int nodes[2] = {d.from_node[k], d.to_node[k]};
        const float3 pts[2] = {from, to};
        for (int e = 0; e < 2; ++e) {
            if (nodes[e] >= 0) {
                eff += x[nodes[e]].w;
            } else {
                const float3 rxn = cross(pts[e] - s.com, dir);
                eff += 1.0f / d.mass + dot(rxn, m3v(invI, rxn));
            }
        }
        if (!(eff > 0.0f) || rel == 0.0f) continue;
        const float req = d.damping[k] * fabsf(rel) * dt;
        const float stop = fabsf(rel) / eff;
        const float mag = copysignf(stop < req ? stop : req, rel);
        const float3 imp[2] = {dir * mag, -(dir * mag)};
        for (int e = 0; e < 2; ++e) {
            if (nodes[e] >= 0) {
                const float w = x[nodes[e]].w;
                if (w > 0.0f) {
                    float4 V = v[nodes[e]];
                    V.x += imp[e].x * w; V.y += imp[e].y * w; V.z += imp[e].z * w;
                    v[nodes[e]] = V;
                }
            } else {
                s.v = s.v + imp[e] / d.mass;
                s.w = s.w + m3v(invI, cross(pts[e] - s.com, imp[e]));
            }
        }
    }
    return true;
}

// certifySubstep and finishSubstep (suspension.cpp:2324-2359, 2481-2610):
// the second half of the payload's substep finish.
__device__ void payload_certify_finish(const DevPayloadDef& d, DevPayloadState& s, const float4* x, const float4* v,
                                       float dt, int* status) {
    auto endpoint = [&](int node, int point, float3& pos, float3& vel) -> bool {
        return payload_endpoint(d, s, x, v, node, point, pos, vel);
    };
    // certifySubstep (suspension.cpp:2324-2359); the unit-norm gate uses an
    // FP32 tolerance.
    const float qn = s.q.x * s.q.x + s.q.y * s.q.y + s.q.z * s.q.z + s.q.w * s.q.w;
    if (!finite3(s.com) || !finite3(s.v) || !finite3(s.w) || !(fabsf(qn - 1.0f) <= 1.0e-5f)) {
        susp_fail(status, kSuspPayload);
        return;
    }
    float maxres = 0.0f;
    s.line_force = make_float3(0.0f, 0.0f, 0.0f);
    s.line_moment = make_float3(0.0f, 0.0f, 0.0f);
    for (int k = 0; k < d.segments; ++k) {
        float3 from, to, vf, vt;
        endpoint(d.from_node[k], d.from_point[k], from, vf);
        endpoint(d.to_node[k], d.to_point[k], to, vt);
        const float3 df = to - from;
        const float l = length(df);
        if (!isfinite(l)) { susp_fail(status, kSuspCertifyLength | ((k + 1) << 8)); return; }
        const float stretch = fmaxf(0.0f, l - d.rest[k]);
        const float cs = s.lambda[k] / (d.stiffness[k] * dt * dt);
        maxres = fmaxf(maxres, fabsf(stretch - cs));
        // finishSubstep payload line wrench
        const float3 dir = l > 0.0f ? df / l : make_float3(0.0f, 0.0f, 0.0f);
        const float3 fimp = dir * (s.lambda[k] / dt);
        if (d.from_point[k] >= 0 || d.to_point[k] >= 0) {
            const bool to_payload = d.to_point[k] >= 0;
            const float3 impulse = to_payload ? -fimp : fimp;
            const float3 pt = to_payload ? to : from;
            s.line_force = s.line_force + impulse / dt;
            s.line_moment = s.line_moment + cross(pt - s.com, impulse / dt);
        }
    }
    s.max_residual = maxres;
    if (maxres > d.max_residual) susp_fail(status, kSuspResidual);
}


// The payload's substep finish: velocity reconstruction, line damping,
// certification and the line wrench.
__device__ void payload_finish(const DevPayloadDef& d, DevPayloadState& s, const DevPayloadState& start,
                               const float4* x, float4* v, float dt, int* status) {
    if (payload_reconstruct_damp(d, s, start, x, v, dt, status)) payload_certify_finish(d, s, x, v, dt, status);
}

// ---- the kernel -------------------------------------------------------------

__device__ __forceinline__ void run_local_stages(const DevTable& t, int kind, int b, unsigned char* smem, float4* x,
                                                 float inv_dt2) {
    const uint32_t* so = t.stage_offsets + static_cast<size_t>(b) * (t.stages + 1);
    const uint32_t* ab = reinterpret_cast<const uint32_t*>(smem + t.smem_ab);
    const float* rest = reinterpret_cast<const float*>(smem + t.smem_rest);
    const float* comp = reinterpret_cast<const float*>(smem + t.smem_comp);
    float* lambda = reinterpret_cast<float*>(smem + t.smem_lambda);
    if (kind == 0) {
        for (int s = 0; s < t.stages; ++s) {
            const uint32_t lo = __ldg(so + s), hi = __ldg(so + s + 1);
            for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
                const uint32_t v = ab[i];
                const uint32_t ia = v & 0xffffu, ib = v >> 16;
                float4 pa = x[ia], pb = x[ib];
                float lam = lambda[i];
                project_distance(pa, pb, rest[i], comp[i], lam, inv_dt2);
                x[ia] = pa;
                x[ib] = pb;
                lambda[i] = lam;
            }
            __syncthreads();
        }
    } else {
        const uint32_t* cd = reinterpret_cast<const uint32_t*>(smem + t.smem_cd);
        for (int s = 0; s < t.stages; ++s) {
            const uint32_t lo = __ldg(so + s), hi = __ldg(so + s + 1);
            for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
                const uint32_t v0 = ab[i], v1 = cd[i];
                const uint32_t ia = v0 & 0xffffu, ib = v0 >> 16, ic = v1 & 0xffffu, id = v1 >> 16;
                float4 A = x[ia], B = x[ib], C = x[ic], D = x[id];
                float lam = lambda[i];
                project_dihedral(A, B, C, D, rest[i], comp[i], lam, inv_dt2);
                x[ia] = A; x[ib] = B; x[ic] = C; x[id] = D;
                lambda[i] = lam;
            }
            __syncthreads();
        }
    }
}

__device__ __forceinline__ void run_global_colour(const DevGlobal& g, int kind, int colour, float4* pos, float inv_dt2) {
    const uint32_t lo = __ldg(g.colour_offsets + colour), hi = __ldg(g.colour_offsets + colour + 1);
    const uint32_t stride = blockDim.x * gridDim.x;
    for (uint32_t i = lo + blockIdx.x * blockDim.x + threadIdx.x; i < hi; i += stride) {
        if (kind == 0) {
            const uint32_t a = __ldg(g.a + i), b = __ldg(g.b + i);
            float4 pa = __ldcg(pos + a), pb = __ldcg(pos + b);
            float lam = __ldcg(g.lambda + i);
            project_distance(pa, pb, __ldg(g.rest + i), __ldg(g.comp + i), lam, inv_dt2);
            __stcg(pos + a, pa);
            __stcg(pos + b, pb);
            __stcg(g.lambda + i, lam);
        } else {
            const uint32_t a = __ldg(g.a + i), b = __ldg(g.b + i), c = __ldg(g.c + i), d = __ldg(g.d + i);
            float4 A = __ldcg(pos + a), B = __ldcg(pos + b), C = __ldcg(pos + c), D = __ldcg(pos + d);
            float lam = __ldcg(g.lambda + i);
            project_dihedral(A, B, C, D, __ldg(g.rest + i), __ldg(g.comp + i), lam, inv_dt2);
            __stcg(pos + a, A); __stcg(pos + b, B); __stcg(pos + c, C); __stcg(pos + d, D);
            __stcg(g.lambda + i, lam);
        }
    }
}

__device__ __forceinline__ void iface_flush(const StepParams& p, int b, const float4* x1, uint32_t base) {
    const uint32_t lo = __ldg(p.iface_begin + b), hi = __ldg(p.iface_begin + b + 1);
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const uint32_t l = __ldg(p.iface_local + i);
        __stcg(p.pos_out + base + l, x1[l]);
    }
}
__device__ __forceinline__ void iface_reload(const StepParams& p, int b, float4* x1, uint32_t base) {
    const uint32_t lo = __ldg(p.iface_begin + b), hi = __ldg(p.iface_begin + b + 1);
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const uint32_t l = __ldg(p.iface_local + i);
        x1[l] = __ldcg(p.pos_out + base + l);
    }
}

__global__ void __launch_bounds__(1024) xpbd_step_kernel(const __grid_constant__ StepParams p) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint64_t bar;
    __shared__ DevPayloadState pay;
    const int b = blockIdx.x;
    const int tid = threadIdx.x;
    float4* x1 = reinterpret_cast<float4*>(smem + p.smem_x1);
    float4* prev1 = reinterpret_cast<float4*>(smem + p.smem_prev1);
    float4* f1 = reinterpret_cast<float4*>(smem + p.smem_f1);
    float4* x2 = reinterpret_cast<float4*>(smem + p.smem_x2);
    const uint32_t base = __ldg(p.l1_begin + b);
    const uint32_t n1 = __ldg(p.l1_begin + b + 1) - base;
    const bool owner = b == p.susp_block;

    // ---- stage the patch and the constraint tables (bulk copies) ----------
    if (tid == 0) mbar_init(&bar, 1);
    __syncthreads();
    if (tid == 0) {
        uint32_t bytes = n1 * 16u;
        for (int l = 0; l < p.levels; ++l)
            for (int k = 0; k < 2; ++k) {
                const DevTable& t = p.tab[l][k];
                const uint32_t cnt = __ldg(t.block_begin + b + 1) - __ldg(t.block_begin + b);
                bytes += cnt * 4u * (k == 0 ? 3u : 4u);
            }
        mbar_expect_tx(&bar, bytes);
        if (n1) bulk_load(x1, p.pos_in + base, n1 * 16u, &bar);
        for (int l = 0; l < p.levels; ++l)
            for (int k = 0; k < 2; ++k) {
                const DevTable& t = p.tab[l][k];
                const uint32_t bb = __ldg(t.block_begin + b);
                const uint32_t cnt = __ldg(t.block_begin + b + 1) - bb;
                if (!cnt) continue;
                bulk_load(smem + t.smem_ab, t.ab + bb, cnt * 4u, &bar);
                if (k == 1) bulk_load(smem + t.smem_cd, t.cd + bb, cnt * 4u, &bar);
                bulk_load(smem + t.smem_rest, t.rest + bb, cnt * 4u, &bar);
                bulk_load(smem + t.smem_comp, t.comp + bb, cnt * 4u, &bar);
            }
    }
    // multipliers restart every substep (soft_body.cpp:1207-1218)
    for (int l = 0; l < p.levels; ++l)
        for (int k = 0; k < 2; ++k) {
            const DevTable& t = p.tab[l][k];
            const uint32_t cnt = __ldg(t.block_begin + b + 1) - __ldg(t.block_begin + b);
            float* lam = reinterpret_cast<float*>(smem + t.smem_lambda);
            for (uint32_t i = tid; i < cnt; i += blockDim.x) lam[i] = 0.0f;
        }
    for (int k = 0; k < 2; ++k) {
        const DevGlobal& g = p.glob[k];
        for (uint32_t i = b * blockDim.x + tid; i < g.count; i += blockDim.x * gridDim.x) g.lambda[i] = 0.0f;
    }
    // pressure gather: external force plus the faces in ascending order
    for (uint32_t i = tid; i < n1; i += blockDim.x) {
        const uint32_t slot = base + i;
        float3 f = f3(__ldg(p.force + slot));
        const uint32_t lo = __ldg(p.tri_offsets + slot), hi = __ldg(p.tri_offsets + slot + 1);
        for (uint32_t q = lo; q < hi; ++q) {
            const uint4 t = __ldg(p.tri + __ldg(p.tri_list + q));
            const float3 pa = f3(__ldg(p.pos_in + t.x));
            const float3 pb = f3(__ldg(p.pos_in + t.y));
            const float3 pc = f3(__ldg(p.pos_in + t.z));
            const float3 area = 0.5f * cross(pb - pa, pc - pa);
            f = f + (__uint_as_float(t.w) * area) / 3.0f;
        }
        f1[i] = make_float4(f.x, f.y, f.z, 0.0f);
    }
    if (owner && tid == 0) pay = *p.payload_in;
    {
        const bool ok = mbar_wait(&bar, 0, p.copy_budget);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicOr(p.status, kStatusCopyTimeout);
                mbar_wait(&bar, 0, p.copy_budget);
            }
            __syncthreads();
            return;
        }
    }
    // ---- predict (soft_body.cpp:1536-1566) and payload prediction ----------
    for (uint32_t i = tid; i < n1; i += blockDim.x) {
        float4 X = x1[i];
        prev1[i] = X;
        if (X.w == 0.0f) continue;
        const float4 V0 = __ldg(p.vel_in + base + i);
        const float4 F = f1[i];
        const float ax = p.gravity.x + F.x * X.w, ay = p.gravity.y + F.y * X.w, az = p.gravity.z + F.z * X.w;
        const float wx = (V0.x + ax * p.dt) - p.ref_velocity.x;
        const float vx = p.ref_velocity.x + (wx - wx * p.damping_loss);
        const float wy = (V0.y + ay * p.dt) - p.ref_velocity.y;
        const float vy = p.ref_velocity.y + (wy - wy * p.damping_loss);
        const float wz = (V0.z + az * p.dt) - p.ref_velocity.z;
        const float vz = p.ref_velocity.z + (wz - wz * p.damping_loss);
        X.x += vx * p.dt;
        X.y += vy * p.dt;
        X.z += vz * p.dt;
        x1[i] = X;
    }
    if (owner && tid == 0) {
        for (int k = 0; k < 8; ++k) pay.lambda[k] = 0.0f;
        if (!payload_predict(*p.payload_def, pay, p.dt, p.gravity)) susp_fail(p.status, kSuspPredict);
    }
    __syncthreads();

    // ---- constraint iterations ------------------------------------------------
    bool has_outer[2];
    for (int k = 0; k < 2; ++k) {
        has_outer[k] = p.glob[k].colours > 0;
        for (int l = 1; l < p.levels; ++l) has_outer[k] = has_outer[k] || p.tab[l][k].stages > 0;
    }
    bool dirty = false;
    bool alive = true;
    for (int it = 0; it < p.iterations && alive; ++it) {
        for (int k = 0; k < 2 && alive; ++k) {
            if (dirty) {
                iface_reload(p, b, x1, base);
                __syncthreads();
                dirty = false;
            }
            if (k == 0 && it > 0 && owner) {
                if (tid == 0) line_iteration(*p.payload_def, pay, x1, p.dt, p.status);
                __syncthreads();
            }
            if (p.levels > 0) run_local_stages(p.tab[0][k], k, b, smem, x1, p.inv_dt2);
            if (!has_outer[k]) continue;
            iface_flush(p, b, x1, base);
            if (!grid_sync(p.barrier)) { alive = false; break; }
            for (int l = 1; l < p.levels && alive; ++l) {
                const DevTable& t = p.tab[l][k];
                if (t.stages == 0) continue;
                const uint32_t lo = __ldg(p.patch_begin[l] + b), hi = __ldg(p.patch_begin[l] + b + 1);
                for (uint32_t i = lo + tid; i < hi; i += blockDim.x)
                    x2[i - lo] = __ldcg(p.pos_out + __ldg(p.patch_slots[l] + i));
                __syncthreads();
                run_local_stages(t, k, b, smem, x2, p.inv_dt2);
                for (uint32_t i = lo + tid; i < hi; i += blockDim.x)
                    __stcg(p.pos_out + __ldg(p.patch_slots[l] + i), x2[i - lo]);
                if (!grid_sync(p.barrier)) alive = false;
            }
            for (int c = 0; c < p.glob[k].colours && alive; ++c) {
                run_global_colour(p.glob[k], k, c, p.pos_out, p.inv_dt2);
                if (!grid_sync(p.barrier)) alive = false;
            }
            dirty = true;
        }
    }
    if (!alive) return;
    if (dirty) {
        iface_reload(p, b, x1, base);
        __syncthreads();
    }
    if (p.iterations > 0 && owner) {
        if (tid == 0) line_iteration(*p.payload_def, pay, x1, p.dt, p.status);
        __syncthreads();
    }
    // ---- final seam-stitch projections (soft_body.cpp:1389-1405) ----------
    if (p.iterations > 0 && p.seam_stages > 0) {
        iface_flush(p, b, x1, base);
        if (!grid_sync(p.barrier)) return;
        for (int s = 0; s < p.seam_stages; ++s) {
            const uint32_t lo = __ldg(p.seam_offsets + s), hi = __ldg(p.seam_offsets + s + 1);
            for (uint32_t i = lo + b * blockDim.x + tid; i < hi; i += blockDim.x * gridDim.x) {
                const uint32_t a = __ldg(p.seam_a + i), c = __ldg(p.seam_b + i);
                float4 pa = __ldcg(p.pos_out + a), pb = __ldcg(p.pos_out + c);
                float lam = 0.0f;  // stitches are rigid: alpha = 0, lambda unused
                project_distance(pa, pb, 0.0f, 0.0f, lam, p.inv_dt2);
                __stcg(p.pos_out + a, pa);
                __stcg(p.pos_out + c, pb);
            }
            if (!grid_sync(p.barrier)) return;
        }
        iface_reload(p, b, x1, base);
        __syncthreads();
    }
    // ---- finalize (soft_body.cpp:1568-1585) --------------------------------
    for (uint32_t i = tid; i < n1; i += blockDim.x) {
        const float4 X = x1[i], P = prev1[i];
        float4 V = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (X.w != 0.0f) V = make_float4((X.x - P.x) * p.inv_dt, (X.y - P.y) * p.inv_dt, (X.z - P.z) * p.inv_dt, 0.0f);
        f1[i] = V;
    }
    __syncthreads();
    if (owner && tid == 0) payload_finish(*p.payload_def, pay, *p.payload_in, x1, f1, p.dt, p.status);
    // ---- re-centring shift (payload centre of mass) --------------------------
    float3 shift = make_float3(0.0f, 0.0f, 0.0f);
    if (p.recentre) {
        if (owner && tid == 0) {
            float3 s = make_float3(0.0f, 0.0f, 0.0f);
            if (fmaxf(fabsf(pay.com.x), fmaxf(fabsf(pay.com.y), fabsf(pay.com.z))) > 0.25f && finite3(pay.com))
                s = make_float3(rintf(pay.com.x * 256.0f) / 256.0f, rintf(pay.com.y * 256.0f) / 256.0f,
                                rintf(pay.com.z * 256.0f) / 256.0f);
            *p.shift_out = s;
        }
        if (!grid_sync(p.barrier)) return;
        const volatile float* sv = reinterpret_cast<const volatile float*>(p.shift_out);
        shift = make_float3(sv[0], sv[1], sv[2]);
    }
    // ---- write the trial state --------------------------------------------
    int bad = 0;
    for (uint32_t i = tid; i < n1; i += blockDim.x) {
        float4 X = x1[i], P = prev1[i];
        const float4 V = f1[i];
        X.x -= shift.x; X.y -= shift.y; X.z -= shift.z;
        P.x -= shift.x; P.y -= shift.y; P.z -= shift.z;
        bad |= !(isfinite(X.x) && isfinite(X.y) && isfinite(X.z) && isfinite(V.x) && isfinite(V.y) && isfinite(V.z));
        p.pos_out[base + i] = X;
        p.prev_out[base + i] = P;
        p.vel_out[base + i] = V;
    }
    if (__syncthreads_or(bad) && tid == 0) atomicOr(p.status, kStatusNonFinite);
    if (owner && tid == 0) {
        pay.com = pay.com - shift;
        *p.payload_out = pay;
    }
    if (b == 0 && tid == 0) {
        p.origin_out[0] = p.origin_in[0] + static_cast<double>(shift.x);
        p.origin_out[1] = p.origin_in[1] + static_cast<double>(shift.y);
        p.origin_out[2] = p.origin_in[2] + static_cast<double>(shift.z);
    }
}

}  // namespace dev
}  // namespace swb
