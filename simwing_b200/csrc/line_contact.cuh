// Line-line contact (swb_structure_set_line_contact): the suspension
// lines' cable segments kept 2 x radius apart, in the cluster step.
//
// Once per substep, after the prediction, every CTA of the cluster boxes
// the segments at their predicted positions and tests the pairs of
// segments that share no node; a pair whose boxes, widened by `reach`,
// overlap becomes a candidate.  Rank 0's block sorts the candidates by key
// (first segment, then second) and into levels of candidates that share
// no node.  After every iteration rank 0's first warp projects the
// candidates level by level, which gives the key-order sweep's results:
// the closest points of the two segments (the segment-segment
// closest-point method of Ericson, Real-Time Collision Detection, 5.1.9)
// pushed apart along their separation to 2 x radius, rigidly, the
// correction shared by the four end nodes in proportion to their inverse
// masses and barycentric weights.  Rollouts tape each step's candidates
// and the projections' inputs, and the reverse kernel runs each
// projection's vector-Jacobian product.  Parity is pinned to the FP64
// port's restatement (the reference's structural step has no line-line
// contact: it rejects segment contact).
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
// barrier inside, and one must follow before rank 0 sorts them).  The pair
// tests are spread evenly: the triangle of pairs is cut into runs of equal
// length, one per warp, whose lanes take the run's pairs in turn.
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
    // the triangle of pairs (i < j), row by row, cut into equal runs, one
    // per warp of the cluster; a warp's lanes take its pairs in turn, so
    // that they read neighbouring boxes together
    const uint64_t S = L.segments, P = S * (S - 1) / 2;
    const uint64_t warps = stride / 32, chunk = (P + warps - 1) / warps;
    const uint64_t run = gt / 32, lane = gt % 32;
    const uint64_t p0 = run * chunk + lane, end = min(P, run * chunk + chunk);
    if (p0 >= end) return;
    auto row_start = [&](uint64_t i) { return i * (2 * S - i - 1) / 2; };
    const double b = 2.0 * static_cast<double>(S) - 1.0;
    uint64_t i = static_cast<uint64_t>(max(0.0, floor((b - sqrt(max(0.0, b * b - 8.0 * static_cast<double>(p0)))) * 0.5)));
    i = min(i, S - 2);
    while (i > 0 && row_start(i) > p0) --i;
    while (i + 2 < S && row_start(i + 1) <= p0) ++i;
    uint64_t j = i + 1 + (p0 - row_start(i));
    float4 lo = __ldcg(L.box + 2 * i), hi = __ldcg(L.box + 2 * i + 1);
    uint2 ni = L.seg_nodes[i];
    for (uint64_t p = p0; p < end; p += 32) {
        const float4 lo2 = __ldcg(L.box + 2 * j), hi2 = __ldcg(L.box + 2 * j + 1);
        if (!(lo.x > hi2.x || lo2.x > hi.x || lo.y > hi2.y || lo2.y > hi.y || lo.z > hi2.z || lo2.z > hi.z)) {
            const uint2 nj = L.seg_nodes[j];
            if (!(ni.x == nj.x || ni.x == nj.y || ni.y == nj.x || ni.y == nj.y)) {
                const uint32_t k = atomicAdd(L.count, 1u);
                if (k < L.capacity)
                    L.pair[k] = (static_cast<uint32_t>(i) << 16) | static_cast<uint32_t>(j);
                else
                    contact_fail(status, kContactLinePairs);
            }
        }
        // the pair 32 places on, across row ends
        j += 32;
        bool moved = false;
        while (j >= S && i + 2 < S) {
            const uint64_t over = j - S;
            ++i;
            j = i + 1 + over;
            moved = true;
        }
        if (j >= S) break;  // past the last pair
        if (moved) {
            lo = __ldcg(L.box + 2 * i);
            hi = __ldcg(L.box + 2 * i + 1);
            ni = L.seg_nodes[i];
        }
    }
}

// Rank 0's block: the candidates into key order (a rank sort; the keys are
// distinct), then each candidate's level: one more than the highest level
// of the earlier candidates (in key order) that share a node with it, 0
// when none does.  Candidates of one level share no node, and every node
// meets its candidates in key order level by level, so projecting the
// levels in turn, each level's candidates side by side, gives the serial
// key-order sweep's results exactly.  Each candidate's predecessors (per
// node, the latest earlier candidate with that node) are found once; the
// levels then follow by sweeps until none changes (as many sweeps as the
// longest chain, plus one).  They go to `scratch`, their count to
// count[1], and the candidates, ordered by level, to `order`.  Reads
// the candidate count after the cluster barrier that followed the
// broadphase.
__device__ __forceinline__ uint4 line_pair_nodes(const LineContactDev& L, uint32_t pr) {
    const uint2 a = L.seg_nodes[pr >> 16], b = L.seg_nodes[pr & 0xffffu];
    return make_uint4(a.x, a.y, b.x, b.y);
}
__device__ void line_sort(const LineContactDev& L, uint32_t* scratch) {
    const uint32_t n = min(L.count[0], L.capacity);
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) scratch[k] = L.pair[k];
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
        const uint32_t mine = scratch[k];
        uint32_t rank = 0;
        for (uint32_t q = 0; q < n; ++q) rank += scratch[q] < mine ? 1u : 0u;
        L.pair[rank] = mine;
    }
    __syncthreads();
    // each candidate's predecessors: for each of its four nodes the latest
    // earlier candidate (key order) that has the node, ~0u for none
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
        const uint4 mine = line_pair_nodes(L, L.pair[k]);
        const uint32_t v[4] = {mine.x, mine.y, mine.z, mine.w};
        uint32_t pred[4] = {~0u, ~0u, ~0u, ~0u};
        uint32_t open = 4;
        for (uint32_t q = k; q-- > 0 && open > 0;) {
            const uint4 o = line_pair_nodes(L, L.pair[q]);
            for (int c = 0; c < 4; ++c)
                if (pred[c] == ~0u && (v[c] == o.x || v[c] == o.y || v[c] == o.z || v[c] == o.w)) {
                    pred[c] = q;
                    --open;
                }
        }
        for (int c = 0; c < 4; ++c) __stcg(L.pred + 4 * k + c, pred[c]);
        __stcg(scratch + k, 0u);
    }
    __syncthreads();
    // the levels: sweeps of level = 1 + the predecessors' highest level
    // until none changes (as many as the longest chain, plus one)
    uint32_t top = 0;
    for (uint32_t sweep = 0; sweep <= n; ++sweep) {
        bool changed = false;
        for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
            uint32_t lv = 0;
            for (int c = 0; c < 4; ++c) {
                const uint32_t q = __ldcg(L.pred + 4 * k + c);
                if (q != ~0u) lv = max(lv, __ldcg(scratch + q) + 1u);
            }
            if (lv != __ldcg(scratch + k)) changed = true;
            top = max(top, lv);
            // the block barrier below orders this store before the next
            // sweep's reads; a read in this sweep sees the old level or the
            // new one, and either only moves the sweep towards the fixpoint
            __stcg(scratch + k, lv);
        }
        if (!__syncthreads_or(changed)) break;
    }
    // the level count: the largest level plus one
    __shared__ uint32_t s_top;
    if (threadIdx.x == 0) s_top = 0;
    __syncthreads();
    atomicMax(&s_top, top);
    __syncthreads();
    const uint32_t levels = n ? s_top + 1u : 0u;
    // the level offsets: counts by level, then their exclusive scan
    for (uint32_t l = threadIdx.x; l <= levels; l += blockDim.x) __stcg(L.level_off + l, 0u);
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) atomicAdd(L.level_off + __ldcg(scratch + k) + 1, 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (uint32_t l = 0; l <= levels; ++l) {
            acc += __ldcg(L.level_off + l);
            L.level_off[l] = acc;
        }
        L.count[1] = levels;
    }
    __syncthreads();
    // the candidates by level, key order within a level
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
        const uint32_t lv = __ldcg(scratch + k);
        uint32_t r = 0;
        for (uint32_t q = 0; q < k; ++q) r += __ldcg(scratch + q) == lv ? 1u : 0u;
        L.order[L.level_off[lv] + r] = L.pair[k];
    }
    __syncthreads();
}

// One candidate's projection: the closest points of its two segments
// pushed apart to 2 x radius, rigidly, the correction shared by the four
// end nodes by inverse mass and barycentric weight.
template <class Addr>
__device__ __forceinline__ void line_project_one(const LineContactDev& L, uint32_t pr, Addr addr, float4* tape) {
    const float gap = 2.0f * L.radius;
    const uint32_t s1 = __ldg(L.seg + (pr >> 16)), s2 = __ldg(L.seg + (pr & 0xffffu));
    const uint32_t aa = addr(s1 & 0xffffu), ab = addr(s1 >> 16), ac = addr(s2 & 0xffffu), ad = addr(s2 >> 16);
    float4 A = ld_node(aa), B = ld_node(ab), Cn = ld_node(ac), D = ld_node(ad);
    if (tape) {
        tape[0] = A;
        tape[1] = B;
        tape[2] = Cn;
        tape[3] = D;
    }
    const float3 d1 = f3(B) - f3(A), d2 = f3(D) - f3(Cn);
    const SegmentClosest q = segment_closest(f3(A), d1, f3(Cn), d2);
    const float3 diff = (f3(A) + d1 * q.s) - (f3(Cn) + d2 * q.t);
    const float dist = length(diff);
    if (!(dist < gap) || !(dist > 0.0f)) return;
    const float3 nrm = diff / dist;
    const float wa = A.w * (1.0f - q.s), wb = B.w * q.s, wc = Cn.w * (1.0f - q.t), wd = D.w * q.t;
    const float W = wa * (1.0f - q.s) + wb * q.s + wc * (1.0f - q.t) + wd * q.t;
    if (!(W > 0.0f)) return;
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

// Rank 0's block: the candidates' projections, level by level (line_sort
// left them ordered by level, with the levels' offsets), on the block's
// first warp: most levels hold fewer candidates than a warp has lanes, and
// a warp barrier between levels costs far less than a block barrier (the
// widest levels take a few rounds of the warp instead).  Taping launches
// pass `tape` ([capacity][4] of this iteration): each candidate's four end
// nodes before its projection, at its place in that order.  The caller's
// cluster barrier publishes the result.
template <class Addr>
__device__ void line_project(const LineContactDev& L, Addr addr, float4* tape = nullptr) {
    if (threadIdx.x >= 32) return;
    const uint32_t lane = threadIdx.x, top = L.count[1];
    // each lane's first candidate of the next level is looked up before the
    // current level's projections (the lists stay fixed for the substep)
    uint32_t next = ~0u;
    if (top > 0 && L.level_off[0] + lane < L.level_off[1]) next = L.order[L.level_off[0] + lane];
    for (uint32_t lv = 0; lv < top; ++lv) {
        const uint32_t lo = L.level_off[lv], hi = L.level_off[lv + 1];
        const uint32_t cur = next;
        next = ~0u;
        if (lv + 1 < top) {
            const uint32_t nlo = L.level_off[lv + 1], nhi = L.level_off[lv + 2];
            if (nlo + lane < nhi) next = L.order[nlo + lane];
        }
        if (cur != ~0u) line_project_one(L, cur, addr, tape ? tape + 4 * (lo + lane) : nullptr);
        for (uint32_t k = lo + lane + 32; k < hi; k += 32)
            line_project_one(L, L.order[k], addr, tape ? tape + 4 * k : nullptr);
        __syncwarp();
    }
}

// Taping launches, rank 0's block after line_sort: the step's candidates
// in level order, the level offsets and the counts into the tape; false
// when they exceed its capacity, and then the tape holds no candidate (its
// reverse does nothing; the step's failure is reported).
__device__ bool line_tape_step(const LineContactDev& L, const TapeStep& t) {
    const uint32_t n = min(L.count[0], L.capacity), top = L.count[1];
    if (n > t.line_cap) {
        if (threadIdx.x == 0) {
            t.line_count[0] = 0;
            t.line_count[1] = 0;
        }
        return false;
    }
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) t.line_pairs[k] = L.order[k];
    for (uint32_t l = threadIdx.x; l <= top; l += blockDim.x) t.line_level_off[l] = L.level_off[l];
    if (threadIdx.x == 0) {
        t.line_count[0] = n;
        t.line_count[1] = top;
    }
    return true;
}

// Double-precision 3-vectors of the reverse below.
struct LV3 {
    double x, y, z;
};
__device__ __forceinline__ LV3 lv3(float4 a) { return {a.x, a.y, a.z}; }
__device__ __forceinline__ LV3 lv3(float3 a) { return {a.x, a.y, a.z}; }
__device__ __forceinline__ LV3 operator+(LV3 a, LV3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ LV3 operator-(LV3 a, LV3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ LV3 operator*(LV3 a, double k) { return {a.x * k, a.y * k, a.z * k}; }
__device__ __forceinline__ double dot(LV3 a, LV3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// The reverse of one candidate's projection: `in` its four end nodes
// before it (taped), g[4] the adjoints of the four nodes after it on entry
// and before it on return.  The closest-point parameters s and t and the
// branch taken are the forward's (FP32); the vector-Jacobian product of
// that map is evaluated in FP64, where ill-conditioned terms (nearly
// parallel segments) cost FP32 most.  s and t depend on the nodes where
// they lie inside (0, 1): there the closest points satisfy d1 . (P - Q) = 0
// (s free) and d2 . (P - Q) = 0 (t free), and their adjoints pass through
// those conditions (implicit function).
__device__ __forceinline__ void line_reverse_one(const float4 in[4], float gap_f, float3 g3[4]) {
    const SegmentClosest q = segment_closest(f3(in[0]), f3(in[1]) - f3(in[0]), f3(in[2]), f3(in[3]) - f3(in[2]));
    {
        // the forward's own test, in its own arithmetic
        const float3 d1 = f3(in[1]) - f3(in[0]), d2 = f3(in[3]) - f3(in[2]);
        const float3 df = (f3(in[0]) + d1 * q.s) - (f3(in[2]) + d2 * q.t);
        const float dist = length(df);
        if (!(dist < gap_f) || !(dist > 0.0f)) return;
        const float Wf = in[0].w * (1.0f - q.s) * (1.0f - q.s) + in[1].w * q.s * q.s +
                         in[2].w * (1.0f - q.t) * (1.0f - q.t) + in[3].w * q.t * q.t;
        if (!(Wf > 0.0f)) return;
    }
    const double gap = gap_f, s = q.s, t = q.t;
    const LV3 A = lv3(in[0]), B = lv3(in[1]), C = lv3(in[2]), D = lv3(in[3]);
    LV3 g[4] = {lv3(g3[0]), lv3(g3[1]), lv3(g3[2]), lv3(g3[3])};
    const LV3 d1 = B - A, d2 = D - C;
    const LV3 diff = (A + d1 * s) - (C + d2 * t);
    const double dist = sqrt(dot(diff, diff));
    const LV3 n = diff * (1.0 / dist);
    const double wA = in[0].w, wB = in[1].w, wC = in[2].w, wD = in[3].w;
    const double wa = wA * (1.0 - s), wb = wB * s, wc = wC * (1.0 - t), wd = wD * t;
    const double W = wa * (1.0 - s) + wb * s + wc * (1.0 - t) + wd * t;
    const double dl = (gap - dist) / W;
    const LV3 u = n * dl;
    // A' = A + wa u, B' = B + wb u, C' = C - wc u, D' = D - wd u
    const LV3 ub = g[0] * wa + g[1] * wb - g[2] * wc - g[3] * wd;
    double wab = dot(g[0], u), wbb = dot(g[1], u), wcb = -dot(g[2], u), wdb = -dot(g[3], u);
    const double dlb = dot(ub, n);
    const LV3 nb = ub * dl;
    // dl = (gap - dist) / W
    const double distb = -dlb / W, Wb = -dlb * dl / W;
    wab += Wb * (1.0 - s);
    wbb += Wb * s;
    wcb += Wb * (1.0 - t);
    wdb += Wb * t;
    double sb = Wb * (wb - wa) - wA * wab + wB * wbb;
    double tb = Wb * (wd - wc) - wC * wcb + wD * wdb;
    // n = diff / dist, dist = |diff|
    const LV3 diffb = (nb - n * dot(n, nb)) * (1.0 / dist) + n * distb;
    // diff = A (1 - s) + B s - C (1 - t) - D t
    g[0] = g[0] + diffb * (1.0 - s);
    g[1] = g[1] + diffb * s;
    g[2] = g[2] - diffb * (1.0 - t);
    g[3] = g[3] - diffb * t;
    sb += dot(diffb, d1);
    tb -= dot(diffb, d2);
    const bool fs = s > 0.0 && s < 1.0, ft = t > 0.0 && t < 1.0;
    double l1 = 0.0, l2 = 0.0;
    if (fs && ft) {
        const double a = dot(d1, d1), b = dot(d1, d2), e = dot(d2, d2), det = a * e - b * b;
        l1 = (-sb * e - b * tb) / det;
        l2 = (a * tb + b * sb) / det;
    } else if (fs) {
        l1 = -sb / dot(d1, d1);
    } else if (ft) {
        l2 = tb / dot(d2, d2);
    }
    // F1 = d1 . diff, F2 = d2 . diff, by node
    g[0] = g[0] + (d1 * (1.0 - s) - diff) * l1 + d2 * ((1.0 - s) * l2);
    g[1] = g[1] + (diff + d1 * s) * l1 + d2 * (s * l2);
    g[2] = g[2] - d1 * ((1.0 - t) * l1) - (diff + d2 * (1.0 - t)) * l2;
    g[3] = g[3] - d1 * (t * l1) + (diff - d2 * t) * l2;
    for (int c = 0; c < 4; ++c)
        g3[c] = make_float3(static_cast<float>(g[c].x), static_cast<float>(g[c].y), static_cast<float>(g[c].z));
}

// The reverse of an iteration's line-line projections, on rank 0's first
// warp: the taped levels from the last, each level's candidates side by
// side, on the node adjoints (`addr` gives a node's adjoint in the cluster
// window).  The caller's cluster barrier publishes the result.  Not
// inlined: the reverse kernel's main loop keeps its registers.
template <class Addr>
__device__ __noinline__ void line_contact_reverse(const LineContactDev& L, const TapeStep& t, int it, Addr addr) {
    const uint32_t top = t.line_count[1];
    const float gap = 2.0f * L.radius;
    const float4* in_it = t.line_in + static_cast<size_t>(it) * t.line_cap * 4;
    if (threadIdx.x >= 32 || t.line_count[0] > t.line_cap || top > t.line_count[0]) return;
    for (uint32_t lv = top; lv-- > 0;) {
        const uint32_t lo = t.line_level_off[lv], hi = t.line_level_off[lv + 1];
        for (uint32_t k = lo + threadIdx.x; k < hi; k += 32) {
            const uint32_t pr = t.line_pairs[k];
            const uint32_t s1 = L.seg[pr >> 16], s2 = L.seg[pr & 0xffffu];
            const uint32_t ad[4] = {addr(s1 & 0xffffu), addr(s1 >> 16), addr(s2 & 0xffffu), addr(s2 >> 16)};
            float4 in[4], G[4];
            float3 g[4];
            for (int c = 0; c < 4; ++c) {
                in[c] = in_it[4 * k + c];
                G[c] = ld_node(ad[c]);
                g[c] = f3(G[c]);
            }
            line_reverse_one(in, gap, g);
            for (int c = 0; c < 4; ++c) st_node(ad[c], make_float4(g[c].x, g[c].y, g[c].z, G[c].w));
        }
        __syncwarp();
    }
}

}  // namespace dev
}  // namespace swb
