// Line-line contact (swb_structure_set_line_contact): the suspension
// lines' cable segments kept 2 x radius apart, in the cluster step.
//
// Once per substep, after the prediction, every CTA of the cluster boxes
// the segments at their predicted positions and tests the pairs of
// segments that share no node; a pair whose boxes, widened by `reach`,
// overlap becomes a candidate.  Rank 0's block sorts the candidates by
// key (first segment, then second).  After every iteration one thread of
// rank 0 projects the candidates in key order: the closest points of the
// two segments (the segment-segment closest-point method of Ericson, Real-
// Time Collision Detection, 5.1.9) pushed apart along their separation to
// 2 x radius, rigidly, the correction shared by the four end nodes in
// proportion to their inverse masses and barycentric weights.  Parity is
// pinned to the FP64 port's restatement (the reference's structural step
// has no line-line contact: it rejects segment contact).
#pragma once

#include <cooperative_groups.h>

#include "cluster_params.h"
#include "contact_phase.cuh"
#include "device_common.cuh"

namespace swb {
namespace dev {

struct SegmentClosest {
    float s, t;
};

// Parameters of the closest points p1 + s d1 and p2 + t d2 of two segments.
__device__ __forceinline__ SegmentClosest segment_closest(float3 p1, float3 d1, float3 p2, float3 d2) {
    constexpr float eps = 1.0e-12f;
    const float3 r = p1 - p2;
    const float a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    SegmentClosest out{0.0f, 0.0f};
    if (a <= eps && e <= eps) return out;
    if (a <= eps) {
        out.t = fminf(fmaxf(f / e, 0.0f), 1.0f);
        return out;
    }
    const float c = dot(d1, r);
    if (e <= eps) {
        out.s = fminf(fmaxf(-c / a, 0.0f), 1.0f);
        return out;
    }
    const float b = dot(d1, d2), denom = a * e - b * b;
    float s = denom != 0.0f ? fminf(fmaxf((b * f - c * e) / denom, 0.0f), 1.0f) : 0.0f;
    float t = (b * s + f) / e;
    if (t < 0.0f) {
        t = 0.0f;
        s = fminf(fmaxf(-c / a, 0.0f), 1.0f);
    } else if (t > 1.0f) {
        t = 1.0f;
        s = fminf(fmaxf((b - c) / a, 0.0f), 1.0f);
    }
    out.s = s;
    out.t = t;
    return out;
}

// The substep's candidate pairs (every thread of every CTA; a cluster
// barrier inside, and one must follow before rank 0 sorts them).
template <class Addr>
__device__ void line_broadphase(const LineContactDev& L, uint32_t me, uint32_t ctas,
                                cooperative_groups::cluster_group& cluster, Addr addr, int* status) {
    const uint32_t gt = me * blockDim.x + threadIdx.x, stride = ctas * blockDim.x;
    for (uint32_t i = gt; i < L.segments; i += stride) {
        const uint32_t ab = L.seg[i];
        const float4 A = ld_node(addr(ab & 0xffffu)), B = ld_node(addr(ab >> 16));
        L.box[2 * i] = make_float4(fminf(A.x, B.x) - L.reach, fminf(A.y, B.y) - L.reach, fminf(A.z, B.z) - L.reach, 0.0f);
        L.box[2 * i + 1] =
            make_float4(fmaxf(A.x, B.x) + L.reach, fmaxf(A.y, B.y) + L.reach, fmaxf(A.z, B.z) + L.reach, 0.0f);
    }
    cluster.sync();
    for (uint32_t i = gt; i < L.segments; i += stride) {
        const float4 lo = __ldcg(L.box + 2 * i), hi = __ldcg(L.box + 2 * i + 1);
        const uint2 ni = L.seg_nodes[i];
        for (uint32_t j = i + 1; j < L.segments; ++j) {
            const float4 lo2 = __ldcg(L.box + 2 * j), hi2 = __ldcg(L.box + 2 * j + 1);
            if (lo.x > hi2.x || lo2.x > hi.x || lo.y > hi2.y || lo2.y > hi.y || lo.z > hi2.z || lo2.z > hi.z) continue;
            const uint2 nj = L.seg_nodes[j];
            if (ni.x == nj.x || ni.x == nj.y || ni.y == nj.x || ni.y == nj.y) continue;
            const uint32_t k = atomicAdd(L.count, 1u);
            if (k < L.capacity)
                L.pair[k] = (i << 16) | j;
            else
                contact_fail(status, kContactLinePairs);
        }
    }
}

// Rank 0's block: the candidates into key order (a rank sort; the keys are
// distinct).  Reads the count after the cluster barrier that followed the
// broadphase.
__device__ void line_sort(const LineContactDev& L, uint32_t* scratch) {
    const uint32_t n = min(*L.count, L.capacity);
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) scratch[k] = L.pair[k];
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
        const uint32_t mine = scratch[k];
        uint32_t rank = 0;
        for (uint32_t q = 0; q < n; ++q) rank += scratch[q] < mine ? 1u : 0u;
        L.pair[rank] = mine;
    }
    __syncthreads();
}

// One thread: the candidates' projections in key order.
template <class Addr>
__device__ void line_project(const LineContactDev& L, Addr addr) {
    const uint32_t n = min(*L.count, L.capacity);
    const float gap = 2.0f * L.radius;
    for (uint32_t k = 0; k < n; ++k) {
        const uint32_t pr = L.pair[k];
        const uint32_t s1 = L.seg[pr >> 16], s2 = L.seg[pr & 0xffffu];
        const uint32_t aa = addr(s1 & 0xffffu), ab = addr(s1 >> 16), ac = addr(s2 & 0xffffu), ad = addr(s2 >> 16);
        float4 A = ld_node(aa), B = ld_node(ab), Cn = ld_node(ac), D = ld_node(ad);
        const float3 d1 = f3(B) - f3(A), d2 = f3(D) - f3(Cn);
        const SegmentClosest q = segment_closest(f3(A), d1, f3(Cn), d2);
        const float3 diff = (f3(A) + d1 * q.s) - (f3(Cn) + d2 * q.t);
        const float dist = length(diff);
        if (!(dist < gap) || !(dist > 0.0f)) continue;
        const float3 nrm = diff / dist;
        const float wa = A.w * (1.0f - q.s), wb = B.w * q.s, wc = Cn.w * (1.0f - q.t), wd = D.w * q.t;
        const float W = wa * (1.0f - q.s) + wb * q.s + wc * (1.0f - q.t) + wd * q.t;
        if (!(W > 0.0f)) continue;
        const float dl = (gap - dist) / W;
        A.x += nrm.x * wa * dl; A.y += nrm.y * wa * dl; A.z += nrm.z * wa * dl;
        B.x += nrm.x * wb * dl; B.y += nrm.y * wb * dl; B.z += nrm.z * wb * dl;
        Cn.x -= nrm.x * wc * dl; Cn.y -= nrm.y * wc * dl; Cn.z -= nrm.z * wc * dl;
        D.x -= nrm.x * wd * dl; D.y -= nrm.y * wd * dl; D.z -= nrm.z * wd * dl;
        st_node(aa, A);
        st_node(ab, B);
        st_node(ac, Cn);
        st_node(ad, D);
    }
}

}  // namespace dev
}  // namespace swb
