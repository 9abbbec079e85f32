// Orthotropic membrane elements on the device (FP32): the XPBD projection of
// one element and its normalized residual, as the reference states them
// (SoftBody::membraneElementCorrections and solveMembraneElement,
// src/softwing/soft_body.cpp:1822-1929; evaluateMembraneElement,
// soft_body.cpp:204-270; updateMembraneSolverDiagnostics,
// soft_body.cpp:2366-2404; effectiveMembraneStiffness and the symmetric
// 3x3 inverse, src/softwing/membrane.cpp:208-296).
//
// An element's Green strain (warp, weft, engineering shear) is taken from the
// deformation F = [e1 e2] Dm^-1 of its triangle, Dm the chart's edge matrix;
// the constraint value is sqrt(A) times the strain and the compliance the
// inverse of the material stiffness (state dependent under compression
// softening).  The three strain components are solved together: a 3x3
// system (1 + gamma) J W J^T + alpha~ with damping gamma = damping time / dt.
#pragma once

#include "cluster_params.h"
#include "step_kernel.cuh"

namespace swb {
namespace dev {

struct MembraneConst {
    float i00, i01, i10, i11;  // inverse chart matrix
    float area_scale;          // sqrt(reference area)
    float damping_time, ratio, warp_pre, weft_pre;
    float c[6];                // compliance xx yy zz xy xz yz
    float k[4];                // stiffness xx yy zz xy (xz = yz = 0)
};

__device__ __forceinline__ MembraneConst load_membrane(const float4* aux, uint32_t r) {
    const float4 q0 = __ldg(aux + static_cast<size_t>(r) * kMembraneAux);
    const float4 q1 = __ldg(aux + static_cast<size_t>(r) * kMembraneAux + 1);
    const float4 q2 = __ldg(aux + static_cast<size_t>(r) * kMembraneAux + 2);
    const float4 q3 = __ldg(aux + static_cast<size_t>(r) * kMembraneAux + 3);
    const float4 q4 = __ldg(aux + static_cast<size_t>(r) * kMembraneAux + 4);
    MembraneConst m;
    m.i00 = q0.x; m.i01 = q0.y; m.i10 = q0.z; m.i11 = q0.w;
    m.area_scale = q1.x; m.damping_time = q1.y; m.ratio = q1.z; m.warp_pre = q1.w;
    m.weft_pre = q2.x; m.c[0] = q2.y; m.c[1] = q2.z; m.c[2] = q2.w;
    m.c[3] = q3.x; m.c[4] = q3.y; m.c[5] = q3.z; m.k[0] = q3.w;
    m.k[1] = q4.x; m.k[2] = q4.y; m.k[3] = q4.z;
    return m;
}

// Green strain and its gradients g[component][corner] (unscaled).
__device__ __forceinline__ float3 membrane_strain(float3 a, float3 b, float3 c, const MembraneConst& m,
                                                  float3 g[3][3]) {
    const float3 e1 = b - a, e2 = c - a;
    const float3 warp = e1 * m.i00 + e2 * m.i10;
    const float3 weft = e1 * m.i01 + e2 * m.i11;
    const float3 s = make_float3(0.5f * (dot(warp, warp) - 1.0f) + m.warp_pre,
                                 0.5f * (dot(weft, weft) - 1.0f) + m.weft_pre, dot(warp, weft));
    // d/d(warp) and d/d(weft) of the three components: (warp, 0), (0, weft), (weft, warp)
    const float3 first[3] = {warp * m.i00, weft * m.i01, weft * m.i00 + warp * m.i01};
    const float3 second[3] = {warp * m.i10, weft * m.i11, weft * m.i10 + warp * m.i11};
    for (int k = 0; k < 3; ++k) {
        g[k][0] = -(first[k] + second[k]);
        g[k][1] = first[k];
        g[k][2] = second[k];
    }
    return s;
}

// Inverse of a symmetric 3x3 (xx yy zz xy xz yz) by cofactors; false when
// the determinant is zero or not finite.
__device__ __forceinline__ bool sym3_inverse(const float* m, float* out) {
    const float c0 = m[1] * m[2] - m[5] * m[5], c1 = m[0] * m[2] - m[4] * m[4], c2 = m[0] * m[1] - m[3] * m[3];
    const float c3 = m[4] * m[5] - m[3] * m[2], c4 = m[3] * m[5] - m[4] * m[1], c5 = m[3] * m[4] - m[0] * m[5];
    const float det = m[0] * c0 + m[3] * c3 + m[4] * c4;
    if (!(det != 0.0f) || !isfinite(det)) return false;
    const float id = 1.0f / det;
    out[0] = c0 * id; out[1] = c1 * id; out[2] = c2 * id;
    out[3] = c3 * id; out[4] = c4 * id; out[5] = c5 * id;
    return true;
}
__device__ __forceinline__ float3 sym3_mul(const float* m, float3 v) {
    return make_float3(m[0] * v.x + m[3] * v.y + m[4] * v.z, m[3] * v.x + m[1] * v.y + m[5] * v.z,
                       m[4] * v.x + m[5] * v.y + m[2] * v.z);
}

// One membrane projection on the element's corners (w = inverse mass);
// pa/pb/pc: the corners' positions at the start of the step (read only when
// the material has damping).  `mult` holds the element's three multipliers.
// Returns false when the element's system has no inverse.
__device__ __forceinline__ bool project_membrane(float4& A, float4& B, float4& C, float3 pa, float3 pb, float3 pc,
                                                 const MembraneConst& m, float* mult, float inv_dt, float inv_dt2) {
    float3 g[3][3];
    const float3 s = membrane_strain(f3(A), f3(B), f3(C), m, g);
    const float w[3] = {A.w, B.w, C.w};
    float3 J[3][3];
    for (int k = 0; k < 3; ++k)
        for (int q = 0; q < 3; ++q) J[k][q] = g[k][q] * m.area_scale;
    float M[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    for (int q = 0; q < 3; ++q) {
        M[0] += w[q] * dot(J[0][q], J[0][q]);
        M[1] += w[q] * dot(J[1][q], J[1][q]);
        M[2] += w[q] * dot(J[2][q], J[2][q]);
        M[3] += w[q] * dot(J[0][q], J[1][q]);
        M[4] += w[q] * dot(J[0][q], J[2][q]);
        M[5] += w[q] * dot(J[1][q], J[2][q]);
    }
    const float gamma = m.damping_time * inv_dt;
    float3 damping = make_float3(0.0f, 0.0f, 0.0f);
    if (gamma != 0.0f) {
        const float3 disp[3] = {f3(A) - pa, f3(B) - pb, f3(C) - pc};
        for (int q = 0; q < 3; ++q) {
            damping.x += dot(J[0][q], disp[q]);
            damping.y += dot(J[1][q], disp[q]);
            damping.z += dot(J[2][q], disp[q]);
        }
    }
    float comp[6];
    if (m.ratio == 1.0f) {
        for (int i = 0; i < 6; ++i) comp[i] = m.c[i];
    } else {
        // effectiveMembraneStiffness: compressed directions scaled by sqrt(ratio)
        const float retained = sqrtf(m.ratio);
        const float ws = s.x < 0.0f ? retained : 1.0f, fs = s.y < 0.0f ? retained : 1.0f;
        const float ss = sqrtf(ws * fs);
        const float k[6] = {m.k[0] * ws * ws, m.k[1] * fs * fs, m.k[2] * ss * ss, m.k[3] * ws * fs, 0.0f, 0.0f};
        if (!sym3_inverse(k, comp)) return false;
    }
    float sys[6], alpha[6];
    for (int i = 0; i < 6; ++i) {
        alpha[i] = inv_dt2 * comp[i];
        sys[i] = (1.0f + gamma) * M[i] + alpha[i];
    }
    const float3 lam = make_float3(mult[0], mult[1], mult[2]);
    const float3 rhs = (-(s * m.area_scale) - sym3_mul(alpha, lam)) - damping * gamma;
    float inv[6];
    if (!(isfinite(rhs.x) && isfinite(rhs.y) && isfinite(rhs.z)) || !sym3_inverse(sys, inv)) return false;
    const float3 dl = sym3_mul(inv, rhs);
    float3 corr[3];
    for (int q = 0; q < 3; ++q) corr[q] = (J[0][q] * dl.x + J[1][q] * dl.y + J[2][q] * dl.z) * w[q];
    A.x += corr[0].x; A.y += corr[0].y; A.z += corr[0].z;
    B.x += corr[1].x; B.y += corr[1].y; B.z += corr[1].z;
    C.x += corr[2].x; C.y += corr[2].y; C.z += corr[2].z;
    mult[0] = lam.x + dl.x;
    mult[1] = lam.y + dl.y;
    mult[2] = lam.z + dl.z;
    return true;
}

// The element's normalized residual after the substep's iterations
// (with the material's constant compliance, as the reference reports it).
__device__ __forceinline__ float membrane_residual(float3 a, float3 b, float3 c, float3 pa, float3 pb, float3 pc,
                                                   const MembraneConst& m, const float* mult, float inv_dt,
                                                   float inv_dt2) {
    float3 g[3][3];
    const float3 s = membrane_strain(a, b, c, m, g);
    const float gamma = m.damping_time * inv_dt;
    float3 damping = make_float3(0.0f, 0.0f, 0.0f);
    if (gamma != 0.0f) {
        const float3 disp[3] = {a - pa, b - pb, c - pc};
        for (int q = 0; q < 3; ++q) {
            damping.x += m.area_scale * dot(g[0][q], disp[q]);
            damping.y += m.area_scale * dot(g[1][q], disp[q]);
            damping.z += m.area_scale * dot(g[2][q], disp[q]);
        }
    }
    float alpha[6];
    for (int i = 0; i < 6; ++i) alpha[i] = inv_dt2 * m.c[i];
    const float3 r = (s * m.area_scale + sym3_mul(alpha, make_float3(mult[0], mult[1], mult[2]))) + damping * gamma;
    return length(r) / m.area_scale;
}

}  // namespace dev
}  // namespace swb
