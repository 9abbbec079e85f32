// Reverse sweep of one XPBD step on a thread-block cluster: the discrete
// adjoint of the taping step (xpbd_cluster_tape_kernel) on the same
// schedule, stage by stage in reverse order.
//
// State of the sweep, per node in distributed shared memory: the adjoint of
// the node's current position (xyz, with the node's inverse mass in w) and
// the adjoint of its final velocity, later the accumulator of the adjoint of
// its step-start position; per record in shared memory: the adjoint of its
// multiplier and its parameter adjoints.  The rigid pilot's reverse runs on
// one warp of the CTA that owns the suspension nodes: each lane evaluates the
// pilot function in forward mode along one input direction and contracts the
// result with the output adjoints, which gives one entry of the input adjoint
// (the function's Jacobian is never stored).
//
// Reverse order (the forward substep, soft_body.cpp:1175-1460, read
// backwards): payload finish -> finalize -> seam closing pass -> for each
// iteration, last first: line iteration, then the colour stages from last to
// first -> predict -> pressure gather -> payload prediction.
#pragma once

#include "adjoint_math.h"
#include "cluster_kernel.cuh"

namespace swb {
namespace dev {

using DualF = adj::Dual<float>;

// ---- pilot reverse on one warp ---------------------------------------------------
constexpr int kPilotMaxIn = 15 + 6 * 16 + 1;
constexpr int kPilotMaxOut = 7 + 8 + 3 * 16;

__device__ __forceinline__ adj::PilotDef<float> pilot_def(const AdjointPilot& a) {
    adj::PilotDef<float> d;
    d.com_local = {a.com_local.x, a.com_local.y, a.com_local.z};
    d.inertia = {a.inertia.x, a.inertia.y, a.inertia.z};
    d.segments = a.segments;
    for (int k = 0; k < 8; ++k) {
        d.from_node[k] = a.from_slot[k];
        d.to_node[k] = a.to_slot[k];
        d.from_point[k] = a.from_point[k];
        d.to_point[k] = a.to_point[k];
        d.stiffness[k] = a.stiffness[k];
        d.damping[k] = a.damping[k];
        d.hang_local[k] = {a.hang_local[k].x, a.hang_local[k].y, a.hang_local[k].z};
    }
    d.min_length = a.min_length;
    return d;
}

// ubar[j] = sum_k ybar[k] d out_k / d u_j for j < nin, computed by the calling
// warp (all 32 lanes), one input direction per lane.  `fn(in, out)` evaluates
// the function on dual numbers.
template <class Fn>
__device__ void warp_vjp(int nin, int nout, const float* u, const float* ybar, float* ubar, Fn fn) {
    const int lane = threadIdx.x & 31;
    for (int base = 0; base < nin; base += 32) {
        const int j = base + lane;
        DualF in[kPilotMaxIn];
        DualF out[kPilotMaxOut];
        for (int k = 0; k < nin; ++k) in[k] = DualF(u[k], k == j ? 1.0f : 0.0f);
        for (int k = 0; k < nout; ++k) out[k] = DualF(0.0f);
        fn(in, out);
        float s = 0.0f;
        for (int k = 0; k < nout; ++k) s += ybar[k] * out[k].d;
        if (j < nin) ubar[j] = s;
    }
    __syncwarp();
}

// Shared state of the pilot reverse (owner CTA).
struct PilotAdjoint {
    float pb[13];         // adjoint of the pilot (com, q, v, w)
    float pb_start[7];    // adjoint of the step-start com and q collected by the finish
    float seg_lambda[8];  // adjoint of the segment multipliers
    float seg_rest[8];    // parameter adjoints
    float mass;
    float u[kPilotMaxIn];
    float ybar[kPilotMaxOut];
    float ubar[kPilotMaxIn];
};

// Payload finish: inputs com_end 3, q_end 4, com_start 3, q_start 4, xs 3S,
// vs 3S, mass; outputs v 3, w 3, vs' 3S.
__device__ void finish_reverse(PilotAdjoint& A, const AdjointPilot& ap, const PilotTape& t,
                               const DevPayloadState& start, float4* xb, float4* vb, float dt) {
    const int lane = threadIdx.x & 31;
    const int S = ap.slots;
    const int nin = 15 + 6 * S, nout = 6 + 3 * S;
    if (lane == 0) {
        for (int k = 0; k < 3; ++k) A.u[k] = t.com[k];
        for (int k = 0; k < 4; ++k) A.u[3 + k] = t.q[k];
        A.u[7] = start.com.x; A.u[8] = start.com.y; A.u[9] = start.com.z;
        A.u[10] = start.q.x; A.u[11] = start.q.y; A.u[12] = start.q.z; A.u[13] = start.q.w;
        for (int s = 0; s < S; ++s) {
            A.u[14 + 3 * s] = t.xs[s].x; A.u[15 + 3 * s] = t.xs[s].y; A.u[16 + 3 * s] = t.xs[s].z;
            A.u[14 + 3 * S + 3 * s] = t.vs[s].x; A.u[15 + 3 * S + 3 * s] = t.vs[s].y;
            A.u[16 + 3 * S + 3 * s] = t.vs[s].z;
        }
        A.u[14 + 6 * S] = ap.mass;
        for (int k = 0; k < 6; ++k) A.ybar[k] = A.pb[7 + k];
        for (int s = 0; s < S; ++s) {
            const float4 V = vb[ap.slot_node[s]];
            A.ybar[6 + 3 * s] = V.x; A.ybar[7 + 3 * s] = V.y; A.ybar[8 + 3 * s] = V.z;
        }
    }
    __syncwarp();
    const adj::PilotDef<float> d = pilot_def(ap);
    warp_vjp(nin, nout, A.u, A.ybar, A.ubar, [&](DualF* in, DualF* out) {
        adj::PilotState<DualF> s, st;
        s.com = {in[0], in[1], in[2]};
        s.q = {in[3], in[4], in[5], in[6]};
        s.v = {DualF(0.0f), DualF(0.0f), DualF(0.0f)};
        s.w = s.v;
        st.com = {in[7], in[8], in[9]};
        st.q = {in[10], in[11], in[12], in[13]};
        st.v = s.v;
        st.w = s.v;
        adj::V3<DualF> xs[16], vs[16];
        for (int k = 0; k < S; ++k) {
            xs[k] = {in[14 + 3 * k], in[15 + 3 * k], in[16 + 3 * k]};
            vs[k] = {in[14 + 3 * S + 3 * k], in[15 + 3 * S + 3 * k], in[16 + 3 * S + 3 * k]};
        }
        adj::payload_finish_t(d, s, st, xs, vs, ap.slot_w, t.lambda, in[14 + 6 * S], dt);
        out[0] = s.v.x; out[1] = s.v.y; out[2] = s.v.z;
        out[3] = s.w.x; out[4] = s.w.y; out[5] = s.w.z;
        for (int k = 0; k < S; ++k) {
            out[6 + 3 * k] = vs[k].x; out[7 + 3 * k] = vs[k].y; out[8 + 3 * k] = vs[k].z;
        }
    });
    if (lane == 0) {
        for (int k = 0; k < 7; ++k) A.pb[k] += A.ubar[k];           // com, q of the end state
        for (int k = 0; k < 7; ++k) A.pb_start[k] += A.ubar[7 + k];
        for (int k = 7; k < 13; ++k) A.pb[k] = 0.0f;                // v, w consumed
        for (int s = 0; s < S; ++s) {
            float4& X = xb[ap.slot_node[s]];
            X.x += A.ubar[14 + 3 * s]; X.y += A.ubar[15 + 3 * s]; X.z += A.ubar[16 + 3 * s];
            float4& V = vb[ap.slot_node[s]];
            V.x = A.ubar[14 + 3 * S + 3 * s]; V.y = A.ubar[15 + 3 * S + 3 * s]; V.z = A.ubar[16 + 3 * S + 3 * s];
        }
        A.mass += A.ubar[14 + 6 * S];
    }
    __syncwarp();
}

// Line iteration: inputs com 3, q 4, lambda ns, xs 3S, rest ns, mass;
// outputs com 3, q 4, lambda ns, xs 3S.  Its Jacobian depends only on the
// taped inputs, so the kernel's prologue computes every iteration's Jacobian
// at once (one warp per iteration, one input direction per lane, dual
// numbers) and the sweep itself only contracts it with the output adjoints.
__device__ __forceinline__ int line_inputs(const AdjointPilot& ap) { return 8 + 2 * ap.segments + 3 * ap.slots; }
__device__ __forceinline__ int line_outputs(const AdjointPilot& ap) { return 7 + ap.segments + 3 * ap.slots; }

// J[k * nin + j] = d out_k / d in_j at the taped inputs, by the calling warp.
__device__ void line_jacobian(const AdjointPilot& ap, const PilotTape& t, float dt, float* J) {
    const int lane = threadIdx.x & 31;
    const int S = ap.slots, ns = ap.segments;
    const int nin = line_inputs(ap), nout = line_outputs(ap);
    float u[kPilotMaxIn];
    for (int k = 0; k < 3; ++k) u[k] = t.com[k];
    for (int k = 0; k < 4; ++k) u[3 + k] = t.q[k];
    for (int k = 0; k < ns; ++k) u[7 + k] = t.lambda[k];
    for (int s = 0; s < S; ++s) {
        u[7 + ns + 3 * s] = t.xs[s].x; u[8 + ns + 3 * s] = t.xs[s].y; u[9 + ns + 3 * s] = t.xs[s].z;
    }
    for (int k = 0; k < ns; ++k) u[7 + ns + 3 * S + k] = ap.rest[k];
    u[7 + 2 * ns + 3 * S] = ap.mass;
    const adj::PilotDef<float> d = pilot_def(ap);
    for (int base = 0; base < nin; base += 32) {
        const int j = base + lane;
        DualF in[kPilotMaxIn];
        DualF out[kPilotMaxOut];
        for (int k = 0; k < nin; ++k) in[k] = DualF(u[k], k == j ? 1.0f : 0.0f);
        adj::PilotState<DualF> s;
        s.com = {in[0], in[1], in[2]};
        s.q = {in[3], in[4], in[5], in[6]};
        s.v = {DualF(0.0f), DualF(0.0f), DualF(0.0f)};
        s.w = s.v;
        DualF lam[8], rest[8];
        adj::V3<DualF> xs[16];
        for (int k = 0; k < ns; ++k) {
            lam[k] = in[7 + k];
            rest[k] = in[7 + ns + 3 * S + k];
        }
        for (int k = 0; k < S; ++k) xs[k] = {in[7 + ns + 3 * k], in[8 + ns + 3 * k], in[9 + ns + 3 * k]};
        adj::line_iteration_t(d, s, xs, ap.slot_w, lam, rest, in[7 + 2 * ns + 3 * S], dt);
        out[0] = s.com.x; out[1] = s.com.y; out[2] = s.com.z;
        out[3] = s.q.w; out[4] = s.q.x; out[5] = s.q.y; out[6] = s.q.z;
        for (int k = 0; k < ns; ++k) out[7 + k] = lam[k];
        for (int k = 0; k < S; ++k) {
            out[7 + ns + 3 * k] = xs[k].x; out[8 + ns + 3 * k] = xs[k].y; out[9 + ns + 3 * k] = xs[k].z;
        }
        if (j < nin)
            for (int k = 0; k < nout; ++k) J[k * nin + j] = out[k].d;
    }
}

// Reverse of one line iteration through its Jacobian J (from the prologue):
// ubar_j = sum_k ybar_k J[k][j], summed in the order of warp_vjp.
__device__ void line_reverse(PilotAdjoint& A, const AdjointPilot& ap, const float* J, float4* xb) {
    const int lane = threadIdx.x & 31;
    const int S = ap.slots, ns = ap.segments;
    const int nin = line_inputs(ap), nout = line_outputs(ap);
    if (lane == 0) {
        for (int k = 0; k < 7; ++k) A.ybar[k] = A.pb[k];
        for (int k = 0; k < ns; ++k) A.ybar[7 + k] = A.seg_lambda[k];
        for (int s = 0; s < S; ++s) {
            const float4 X = xb[ap.slot_node[s]];
            A.ybar[7 + ns + 3 * s] = X.x; A.ybar[8 + ns + 3 * s] = X.y; A.ybar[9 + ns + 3 * s] = X.z;
        }
    }
    __syncwarp();
    for (int j = lane; j < nin; j += 32) {
        float s = 0.0f;
        for (int k = 0; k < nout; ++k) s += A.ybar[k] * __ldcg(J + k * nin + j);
        A.ubar[j] = s;
    }
    __syncwarp();
    if (lane == 0) {
        for (int k = 0; k < 7; ++k) A.pb[k] = A.ubar[k];
        for (int k = 0; k < ns; ++k) A.seg_lambda[k] = A.ubar[7 + k];
        for (int s = 0; s < S; ++s) {
            float4& X = xb[ap.slot_node[s]];
            X.x = A.ubar[7 + ns + 3 * s]; X.y = A.ubar[8 + ns + 3 * s]; X.z = A.ubar[9 + ns + 3 * s];
        }
        for (int k = 0; k < ns; ++k) A.seg_rest[k] += A.ubar[7 + ns + 3 * S + k];
        A.mass += A.ubar[7 + 2 * ns + 3 * S];
    }
    __syncwarp();
}

// Payload prediction: inputs com 3, q 4, v 3, w 3, mass; outputs com 3, q 4
// (the predicted v and w are overwritten by the finish, so carry no adjoint).
__device__ void predict_reverse(PilotAdjoint& A, const AdjointPilot& ap, const DevPayloadState& start, float dt,
                                float3 g, float* pb_in) {
    const int lane = threadIdx.x & 31;
    if (lane == 0) {
        A.u[0] = start.com.x; A.u[1] = start.com.y; A.u[2] = start.com.z;
        A.u[3] = start.q.x; A.u[4] = start.q.y; A.u[5] = start.q.z; A.u[6] = start.q.w;
        A.u[7] = start.v.x; A.u[8] = start.v.y; A.u[9] = start.v.z;
        A.u[10] = start.w.x; A.u[11] = start.w.y; A.u[12] = start.w.z;
        A.u[13] = ap.mass;
        for (int k = 0; k < 7; ++k) A.ybar[k] = A.pb[k];
    }
    __syncwarp();
    const adj::PilotDef<float> d = pilot_def(ap);
    const adj::V3<float> grav = {g.x, g.y, g.z};
    warp_vjp(14, 7, A.u, A.ybar, A.ubar, [&](DualF* in, DualF* out) {
        adj::PilotState<DualF> s;
        s.com = {in[0], in[1], in[2]};
        s.q = {in[3], in[4], in[5], in[6]};
        s.v = {in[7], in[8], in[9]};
        s.w = {in[10], in[11], in[12]};
        adj::payload_predict_t(d, s, in[13], dt, grav);
        out[0] = s.com.x; out[1] = s.com.y; out[2] = s.com.z;
        out[3] = s.q.w; out[4] = s.q.x; out[5] = s.q.y; out[6] = s.q.z;
    });
    if (lane == 0) {
        for (int k = 0; k < 7; ++k) pb_in[k] = A.pb_start[k] + A.ubar[k];
        for (int k = 7; k < 13; ++k) pb_in[k] = A.ubar[k];
        A.mass += A.ubar[13];
    }
    __syncwarp();
}

// ---- projections ----------------------------------------------------------------
__device__ __forceinline__ adj::V3<float> v3a(float4 a) { return {a.x, a.y, a.z}; }

// The tape entries of record i of this iteration: position and multiplier of
// the first node, then the other nodes' positions (2 entries for a distance
// record, 4 for a dihedral).
struct RecordTape {
    float4 t[4];
};
__device__ __forceinline__ RecordTape load_tape(int kind, const TapeStep& tp, int it, uint32_t i) {
    const uint32_t rtotal = kind ? tp.r1 : tp.r0;
    const float4* tape = (kind ? tp.dih : tp.dist) + static_cast<size_t>(it) * (kind ? 4 : 2) * rtotal;
    RecordTape t;
    t.t[0] = __ldcs(tape + i);
    t.t[1] = __ldcs(tape + rtotal + i);
    if (kind) {
        t.t[2] = __ldcs(tape + 2 * rtotal + i);
        t.t[3] = __ldcs(tape + 3 * rtotal + i);
    } else {
        t.t[2] = t.t[3] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    return t;
}

__device__ __forceinline__ void reverse_record(const ClusterRecord& r, int kind, uint32_t me, uint32_t x_base,
                                               const RecordTape& tp, float* lamb, float* acc_r, float* acc_c,
                                               uint32_t first, float inv_dt2) {
    const uint32_t pa = node_addr(r.ab & 0xffffu, me, 0u, x_base);
    const uint32_t pb = node_addr(r.ab >> 16, me, 0u, x_base);
    const uint32_t slot = r.index - first;
    if (kind == 0) {
        const float4 A4 = tp.t[0], B4 = tp.t[1];
        const float4 XA = ld_node(pa), XB = ld_node(pb);
        adj::DistanceGrad<float> g{v3a(XA), v3a(XB), lamb[slot], 0.0f, 0.0f};
        adj::dist_reverse(v3a(A4), v3a(B4), XA.w, XB.w, A4.w, r.rest, fabsf(r.comp), signbit(r.comp) != 0, inv_dt2,
                          g);
        st_node(pa, make_float4(g.a.x, g.a.y, g.a.z, XA.w));
        st_node(pb, make_float4(g.b.x, g.b.y, g.b.z, XB.w));
        lamb[slot] = g.lambda;
        acc_r[slot] += g.rest;
        acc_c[slot] += g.comp;
    } else {
        const uint32_t pc = node_addr(r.cd & 0xffffu, me, 0u, x_base);
        const uint32_t pd = node_addr(r.cd >> 16, me, 0u, x_base);
        const float4 A4 = tp.t[0], B4 = tp.t[1], C4 = tp.t[2], D4 = tp.t[3];
        const float4 XA = ld_node(pa), XB = ld_node(pb), XC = ld_node(pc), XD = ld_node(pd);
        const adj::V3<float> p[4] = {v3a(A4), v3a(B4), v3a(C4), v3a(D4)};
        const float w[4] = {XA.w, XB.w, XC.w, XD.w};
        adj::DihedralGrad<float> G;
        G.p[0] = v3a(XA); G.p[1] = v3a(XB); G.p[2] = v3a(XC); G.p[3] = v3a(XD);
        G.lambda = lamb[slot];
        adj::dihedral_reverse(p, w, A4.w, r.rest, r.comp, inv_dt2, G);
        st_node(pa, make_float4(G.p[0].x, G.p[0].y, G.p[0].z, XA.w));
        st_node(pb, make_float4(G.p[1].x, G.p[1].y, G.p[1].z, XB.w));
        st_node(pc, make_float4(G.p[2].x, G.p[2].y, G.p[2].z, XC.w));
        st_node(pd, make_float4(G.p[3].x, G.p[3].y, G.p[3].z, XD.w));
        lamb[slot] = G.lambda;
        acc_c[slot] += G.comp;
    }
}

// kMaxThreads: the launch bound.  Up to 512 threads a thread has the
// registers (128) to prefetch the next stage's record and tape entries; the
// 768-thread instantiation (80 registers) loads them when it reaches them.
// kLines: the instantiation that reverses line-line contact (the others
// carry none of its code, so their registers stay as they were).
template <int kMaxThreads, bool kLines = false>
__global__ void __launch_bounds__(kMaxThreads) xpbd_cluster_adjoint_kernel_t(const __grid_constant__ AdjointParams p) {
    constexpr bool kPrefetch = kMaxThreads <= 512;
    namespace cg = cooperative_groups;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ PilotAdjoint pa;
    cg::cluster_group cluster = cg::this_cluster();
    const uint32_t me = cluster.block_rank();
    const ClusterInstance& I = *p.inst;
    const int tid = threadIdx.x;
    float4* xb = reinterpret_cast<float4*>(smem + p.smem_xb);
    float4* vb = reinterpret_cast<float4*>(smem + p.smem_vb);
    float* lam[2] = {reinterpret_cast<float*>(smem + p.smem_lam0), reinterpret_cast<float*>(smem + p.smem_lam1)};
    float* acc0r = reinterpret_cast<float*>(smem + p.smem_acc0r);
    float* acc_c[2] = {reinterpret_cast<float*>(smem + p.smem_acc0c), reinterpret_cast<float*>(smem + p.smem_acc1c)};
    const uint32_t base = __ldg(I.patch_begin + me);
    const uint32_t n = __ldg(I.patch_begin + me + 1) - base;
    const bool owner = static_cast<int>(me) == I.susp_cta;
    const bool pilot_warp = owner && tid < 32;
    const uint32_t x_base = smem_addr(xb);
    const AdjointPilot* ap = p.tape.pilot;

    // stage offsets of this CTA
    const int S0 = I.kind[0].stages, S1 = I.kind[1].stages, S = S0 + S1;
    uint32_t* soff = reinterpret_cast<uint32_t*>(smem + p.smem_offsets);
    for (int i = tid; i <= S0; i += blockDim.x)
        soff[i] = __ldg(I.kind[0].offsets + static_cast<size_t>(me) * (S0 + 1) + i);
    for (int i = tid; i <= S1; i += blockDim.x)
        soff[S0 + 1 + i] = __ldg(I.kind[1].offsets + static_cast<size_t>(me) * (S1 + 1) + i);
    // adjoint state of the step's outputs
    for (uint32_t i = tid; i < n; i += blockDim.x) {
        const float4 X = __ldg(I.pos_in + base + i);
        const float4 B = p.xb_out[base + i];
        xb[i] = make_float4(B.x, B.y, B.z, X.w);
        vb[i] = p.vb_out[base + i];
    }
    __syncthreads();
    const uint32_t first[2] = {soff[0], soff[S0 + 1]};
    const uint32_t count[2] = {soff[S0] - soff[0], soff[S0 + 1 + S1] - soff[S0 + 1]};
    // multiplier and parameter adjoints start at zero
    for (int k = 0; k < 2; ++k)
        for (uint32_t i = tid; i < count[k]; i += blockDim.x) {
            lam[k][i] = 0.0f;
            acc_c[k][i] = 0.0f;
            if (k == 0) acc0r[i] = 0.0f;
        }
    if (owner && tid < 13) pa.pb[tid] = p.pb_out[tid];
    if (owner && tid < 8) {
        pa.seg_lambda[tid] = 0.0f;
        pa.seg_rest[tid] = 0.0f;
        if (tid < 7) pa.pb_start[tid] = 0.0f;
    }
    if (owner && tid == 0) pa.mass = 0.0f;
    __syncthreads();
    auto stage_lo = [&](int g) { return g < S0 ? soff[g] : soff[S0 + 1 + (g - S0)]; };
    auto stage_hi = [&](int g) { return g < S0 ? soff[g + 1] : soff[S0 + 2 + (g - S0)]; };

    // ---- line-iteration Jacobians of every iteration (all warps but the
    // pilot warp, one iteration each; the pilot warp too when it is the only
    // warp); read after the cluster barriers below
    const int line_block = I.susp_cta >= 0 ? line_inputs(*ap) * line_outputs(*ap) : 0;
    if (I.susp_cta >= 0) {
        const int warps = static_cast<int>(blockDim.x >> 5);
        const int total = p.ctas * warps;
        const int workers = total > 1 ? total - 1 : 1;
        int w = static_cast<int>(me) * warps + (tid >> 5);
        const int pilot_at = I.susp_cta * warps;  // the pilot warp's index
        if (total == 1 || w != pilot_at) {
            if (total > 1 && w > pilot_at) --w;
            for (int it = w; it < p.iterations; it += workers)
                line_jacobian(*ap, p.tape.line[it], p.dt, p.line_jac + static_cast<size_t>(it) * line_block);
        }
    }
    // ---- payload finish ------------------------------------------------------------
    if (I.susp_cta >= 0) {
        if (pilot_warp) finish_reverse(pa, *ap, *p.tape.finish, *I.payload_in, xb, vb, p.dt);
        __syncthreads();
    }
    // ---- finalize: v = (x - X) / dt --------------------------------------------------
    for (uint32_t i = tid; i < n; i += blockDim.x) {
        float4 X = xb[i];
        const float4 V = vb[i];
        if (X.w != 0.0f) {
            X.x += V.x * p.inv_dt; X.y += V.y * p.inv_dt; X.z += V.z * p.inv_dt;
            vb[i] = make_float4(-V.x * p.inv_dt, -V.y * p.inv_dt, -V.z * p.inv_dt, 0.0f);
        } else {
            vb[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        xb[i] = X;
    }
    cluster.sync();
    // ---- seam closing pass, last stage first ----------------------------------------
    if (p.iterations > 0) {
        for (int s = I.seam_stages - 1; s >= 0; --s) {
            const uint32_t* off = I.seam_offsets + static_cast<size_t>(me) * (I.seam_stages + 1);
            for (uint32_t i = __ldg(off + s) + tid; i < __ldg(off + s + 1); i += blockDim.x) {
                const uint32_t r = __ldg(I.seam_ab + i);
                const uint32_t a = node_addr(r & 0xffffu, me, 0u, x_base);
                const uint32_t b = node_addr(r >> 16, me, 0u, x_base);
                const float4 A4 = __ldcs(p.tape.seam + i), B4 = __ldcs(p.tape.seam + p.tape.rs + i);
                const float4 XA = ld_node(a), XB = ld_node(b);
                adj::DistanceGrad<float> g{v3a(XA), v3a(XB), 0.0f, 0.0f, 0.0f};
                adj::dist_reverse(v3a(A4), v3a(B4), XA.w, XB.w, 0.0f, 0.0f, 0.0f, false, p.inv_dt2, g);
                st_node(a, make_float4(g.a.x, g.a.y, g.a.z, XA.w));
                st_node(b, make_float4(g.b.x, g.b.y, g.b.z, XB.w));
            }
            cluster.sync();
        }
    }
    // ---- iterations, last first --------------------------------------------------------
    // In the narrow instantiation each thread prefetches its first record of
    // the next stage visited and that record's tape entries before it works on
    // the current one, so the loads from L2 and DRAM overlap the stage and its
    // barrier.  The record arrays' pointers are held in registers.
    const uint4* rec[2] = {I.kind[0].rec, I.kind[1].rec};
    ClusterRecord next;
    next.index = ~0u;
    RecordTape next_tape{};
    auto prefetch = [&](int it, int g) {
        const int kind = g < S0 ? 0 : 1;
        next = load_record(rec[kind], stage_lo(g) + tid, stage_hi(g));
        if (next.index != ~0u) next_tape = load_tape(kind, p.tape, it, next.index);
    };
    if (kPrefetch && p.iterations > 0 && S > 0) prefetch(p.iterations - 1, S - 1);
    // The forward ran the line iteration beside its last two stages (neither
    // touches a riser attachment node); the reverse of the line iteration runs
    // beside the reverse of those two stages, on the same idle last warp of
    // the suspension CTA: it arrives at the first reverse stage's barrier,
    // runs, then waits, and its writes are released by its arrival at the
    // second one's barrier.
    const int line_stage = I.susp_cta >= 0 ? I.line_stage : -1;
    const bool line_warp = line_stage >= 0 && owner && (tid >> 5) == static_cast<int>(blockDim.x >> 5) - 1;
    const uint32_t slots = __ldg(I.patch_begin + p.ctas);
    for (int it = p.iterations - 1; it >= 0; --it) {
        // the ground plane closed the forward iteration: a node it moved
        // kept only its position along the plane (x' = x - n (n.x - off)),
        // so its adjoint loses the normal component
        if (p.ground) {
            const uint8_t* moved = p.tape.ground + static_cast<size_t>(it) * slots + base;
            const float3 nrm = p.ground_normal;
            for (uint32_t i = tid; i < n; i += blockDim.x) {
                if (!moved[i]) continue;
                float4 B = xb[i];
                const float d = nrm.x * B.x + nrm.y * B.y + nrm.z * B.z;
                B.x -= d * nrm.x;
                B.y -= d * nrm.y;
                B.z -= d * nrm.z;
                xb[i] = B;
            }
            cluster.sync();
        }
        // the line-line projections followed the pilot's line iteration
        if constexpr (kLines) {
            if (me == 0)
                line_contact_reverse(*I.lines, p.tape, it,
                                     [&](uint32_t ref) { return node_addr(ref, me, 0u, x_base); });
            cluster.sync();
        }
        if (I.susp_cta >= 0 && line_stage < 0) {
            if (pilot_warp) line_reverse(pa, *ap, p.line_jac + static_cast<size_t>(it) * line_block, xb);
            cluster.sync();
        }
        for (int g = S - 1; g >= 0; --g) {
            const int kind = g < S0 ? 0 : 1;
            uint32_t i = stage_lo(g) + tid;
            if constexpr (kPrefetch) {
                const ClusterRecord cur = next;
                const RecordTape cur_tape = next_tape;
                if (g > 0)
                    prefetch(it, g - 1);
                else if (it > 0)
                    prefetch(it - 1, S - 1);
                if (cur.index != ~0u)
                    reverse_record(cur, kind, me, x_base, cur_tape, lam[kind], kind ? acc_c[1] : acc0r, acc_c[kind],
                                   first[kind], p.inv_dt2);
                i += blockDim.x;
            }
            for (; i < stage_hi(g); i += blockDim.x)
                reverse_record(load_record(rec[kind], i, stage_hi(g)), kind, me, x_base, load_tape(kind, p.tape, it, i),
                               lam[kind], kind ? acc_c[1] : acc0r, acc_c[kind], first[kind], p.inv_dt2);
            if (g == line_stage + 1 && line_warp) {
                cluster_arrive();
                line_reverse(pa, *ap, p.line_jac + static_cast<size_t>(it) * line_block, xb);
                cluster_wait();
            } else {
                cluster.sync();
            }
        }
    }
    // ---- predict: x = X + dt (ref + (V + (g + f w) dt - ref) damping) --------------------
    const float vscale = p.damping * p.dt;
    for (uint32_t i = tid; i < n; i += blockDim.x) {
        const float4 X = xb[i];
        float4 acc = vb[i];
        acc.x += X.x; acc.y += X.y; acc.z += X.z;
        vb[i] = acc;
        float4 Vb = make_float4(0.0f, 0.0f, 0.0f, 0.0f), Fb = Vb;
        if (X.w != 0.0f) {
            Vb = make_float4(X.x * vscale, X.y * vscale, X.z * vscale, 0.0f);
            const float fs = vscale * p.dt * X.w;
            Fb = make_float4(X.x * fs, X.y * fs, X.z * fs, 0.0f);
        }
        p.vb_in[base + i] = Vb;
        p.fbar[base + i] = Fb;
    }
    cluster.sync();
    // ---- pressure gather: f_i += sum_t dp_t area_t / 3 ------------------------------------
    for (uint32_t i = tid; i < n; i += blockDim.x) {
        const uint32_t slot = base + i;
        float4 acc = vb[i];
        const uint32_t lo = __ldg(I.tri_offsets + slot), hi = __ldg(I.tri_offsets + slot + 1);
        for (uint32_t q = lo; q < hi; ++q) {
            const uint4 t = __ldg(I.tri + __ldg(I.tri_list + q));
            const float4 fa = __ldcg(p.fbar + t.x), fb = __ldcg(p.fbar + t.y), fc = __ldcg(p.fbar + t.z);
            const float s = __uint_as_float(t.w) * (0.5f / 3.0f);
            const float3 cb = make_float3((fa.x + fb.x + fc.x) * s, (fa.y + fb.y + fc.y) * s, (fa.z + fb.z + fc.z) * s);
            const float3 xa = f3(__ldg(I.pos_in + t.x)), xbp = f3(__ldg(I.pos_in + t.y)), xc = f3(__ldg(I.pos_in + t.z));
            const float3 u = xbp - xa, w = xc - xa;
            const float3 ub = cross(w, cb), wb = cross(cb, u);
            float3 d;
            if (slot == t.x) d = -(ub + wb);
            else if (slot == t.y) d = ub;
            else d = wb;
            acc.x += d.x; acc.y += d.y; acc.z += d.z;
        }
        p.xb_in[slot] = make_float4(acc.x, acc.y, acc.z, 0.0f);
    }
    // ---- payload prediction, parameter adjoints ---------------------------------------------
    if (I.susp_cta >= 0 && pilot_warp) predict_reverse(pa, *ap, *I.payload_in, p.dt, p.gravity, p.pb_in);
    for (int k = 0; k < 2; ++k)
        for (uint32_t i = tid; i < count[k]; i += blockDim.x) {
            if (k == 0) {
                p.g_rest0[first[0] + i] += acc0r[i];
                p.g_comp0[first[0] + i] += acc_c[0][i];
            } else {
                p.g_comp1[first[1] + i] += acc_c[1][i];
            }
        }
    if (pilot_warp && tid == 0) {
        for (int k = 0; k < ap->segments; ++k) p.g_seg_rest[k] += pa.seg_rest[k];
        p.g_mass[0] += pa.mass;
    }
    if (I.susp_cta < 0 && me == 0 && tid < 13) p.pb_in[tid] = 0.0f;
    cluster.sync();  // no CTA leaves while a peer may still read its memory
}

inline constexpr auto xpbd_cluster_adjoint_kernel = &xpbd_cluster_adjoint_kernel_t<kClusterMaxThreads>;
inline constexpr auto xpbd_cluster_adjoint_kernel_narrow = &xpbd_cluster_adjoint_kernel_t<512>;
inline constexpr auto xpbd_cluster_adjoint_lines_kernel = &xpbd_cluster_adjoint_kernel_t<kClusterMaxThreads, true>;
inline constexpr auto xpbd_cluster_adjoint_lines_kernel_narrow = &xpbd_cluster_adjoint_kernel_t<512, true>;

}  // namespace dev
}  // namespace swb
