// Cluster XPBD step kernel: one thread-block cluster (up to 16 CTAs)
// steps one structure, with every node resident in the distributed shared
// memory of the cluster for the whole substep.
//
// Same substep as xpbd_step_kernel (SoftBody::integrateSubstepTrial,
// src/softwing/soft_body.cpp:1175-1460) with a different schedule: every
// colour of the whole mesh is one stage, each CTA executes the stage's
// constraints it owns, nodes of other CTAs are read and written through
// distributed shared memory, and a cluster barrier (not a device-wide one)
// separates stages.  A launch may carry several independent clusters; the
// cluster index selects the instance (see ClusterInstance).
#pragma once

#include <cooperative_groups.h>

#include "cluster_params.h"
#include "membrane.cuh"
#include "contact_phase.cuh"
#include "line_contact.cuh"
#include "step_kernel.cuh"

namespace swb {

namespace dev {

// `ref` names a node by (instance rank << 12 | local index); `rank_base` is
// the instance's first rank in the cluster (0 unless several structures
// share the cluster).
__device__ __forceinline__ float4* node_at(uint32_t ref, uint32_t me, uint32_t rank_base, float4* x,
                                           float4* const* peers) {
    const uint32_t r = ref >> 12;
    return (r == me ? x : peers[r + rank_base]) + (ref & 0xfffu);
}

// One constraint record held in registers between its prefetch and its use.
struct ClusterRecord {
    uint32_t ab, cd;
    float rest, comp;
    uint32_t index;  // record index (global), or ~0u when the slot is empty
};

__device__ __forceinline__ ClusterRecord load_record(const uint4* rec, uint32_t i, uint32_t hi) {
    ClusterRecord r;
    r.index = ~0u;
    if (i < hi) {
        const uint4 q = __ldg(rec + i);
        r.ab = q.x;
        r.cd = q.y;
        r.rest = __uint_as_float(q.z);
        r.comp = __uint_as_float(q.w);
        r.index = i;
    }
    return r;
}
__device__ __forceinline__ ClusterRecord load_record(const ClusterKindDev& K, int, uint32_t i, uint32_t hi) {
    return load_record(K.rec, i, hi);
}

// Cluster-window address of node `ref`: the node arrays sit at the same
// shared-memory offset in every CTA, so a peer's node is this CTA's address
// mapped to the peer's rank (mapa); a local node keeps its own address,
// which is valid in the cluster window.
__device__ __forceinline__ uint32_t node_addr(uint32_t ref, uint32_t me, uint32_t rank_base, uint32_t x_base) {
    const uint32_t rank = ref >> 12;
    const uint32_t local = x_base + (ref & 0xfffu) * 16u;
    if (rank == me) return local;
    uint32_t remote;
    asm("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(local), "r"(rank + rank_base));
    return remote;
}

// The two halves of a cluster barrier, for a warp that works between its
// arrival and its wait (arrive releases, wait acquires; every lane of the
// warp executes both).
__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.aligned;" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.aligned;" ::: "memory"); }

// ---- momentum guard of free structures (soft_body.cpp:119-190) -------------
// Sums over a CTA's free nodes, in double: [0] mass, [1..3] sum m x,
// [4..6] sum m v, [7..9] sum m x cross v, [10..15] sum m x x^T (xx yy zz xy
// xz yz), m = 1 / inverse mass.
constexpr int kMomentumFields = 16;
constexpr int kMaxWarps = kClusterMaxThreads / 32;

// This CTA's sums into out[16] (shared), by the whole block.
__device__ __noinline__ void cta_momentum_sums(const float4* x, const float4* vel, uint32_t n, double* out,
                                               double* scratch) {
    double acc[kMomentumFields];
    for (int f = 0; f < kMomentumFields; ++f) acc[f] = 0.0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const float4 X = x[i], V = vel[i];
        if (!(X.w > 0.0f)) continue;
        const double m = 1.0 / static_cast<double>(X.w);
        const double px = X.x, py = X.y, pz = X.z, vx = V.x, vy = V.y, vz = V.z;
        acc[0] += m;
        acc[1] += m * px; acc[2] += m * py; acc[3] += m * pz;
        acc[4] += m * vx; acc[5] += m * vy; acc[6] += m * vz;
        acc[7] += m * (py * vz - pz * vy); acc[8] += m * (pz * vx - px * vz); acc[9] += m * (px * vy - py * vx);
        acc[10] += m * px * px; acc[11] += m * py * py; acc[12] += m * pz * pz;
        acc[13] += m * px * py; acc[14] += m * px * pz; acc[15] += m * py * pz;
    }
    for (int f = 0; f < kMomentumFields; ++f)
        for (int off = 16; off > 0; off >>= 1) acc[f] += __shfl_down_sync(0xffffffffu, acc[f], off);
    const int warp = static_cast<int>(threadIdx.x >> 5);
    if ((threadIdx.x & 31) == 0)
        for (int f = 0; f < kMomentumFields; ++f) scratch[warp * kMomentumFields + f] = acc[f];
    __syncthreads();
    if (threadIdx.x < kMomentumFields) {
        double s = 0.0;
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) s += scratch[w * kMomentumFields + threadIdx.x];
        out[threadIdx.x] = s;
    }
    __syncthreads();
}

// Cluster totals of the sums in `sums` (the same shared offset in every CTA
// of the structure), added in rank order so every CTA holds the same values;
// after a cluster barrier.
__device__ __forceinline__ void cluster_momentum_totals(cooperative_groups::cluster_group& cluster, double* sums,
                                                        int ctas, uint32_t rank_base, double* total) {
    if (threadIdx.x < kMomentumFields) {
        double s = 0.0;
        for (int r = 0; r < ctas; ++r)
            s += cluster.map_shared_rank(sums, r + static_cast<int>(rank_base))[threadIdx.x];
        total[threadIdx.x] = s;
    }
    __syncthreads();
}

// Momentum about the centre of mass from the totals: com, linear momentum
// and angular momentum about com.
struct MomentumTotals {
    double mass, com[3], p[3], L[3];
};
__device__ __forceinline__ MomentumTotals momentum_of(const double* t) {
    MomentumTotals r;
    r.mass = t[0];
    for (int k = 0; k < 3; ++k) {
        r.com[k] = t[0] > 0.0 ? t[1 + k] / t[0] : 0.0;
        r.p[k] = t[4 + k];
    }
    // sum m (x - c) x v = sum m x x v - c x sum m v
    r.L[0] = t[7] - (r.com[1] * t[6] - r.com[2] * t[5]);
    r.L[1] = t[8] - (r.com[2] * t[4] - r.com[0] * t[6]);
    r.L[2] = t[9] - (r.com[0] * t[5] - r.com[1] * t[4]);
    return r;
}

// isPositiveDefinite and checkedSolve of a symmetric 3x3 (xx yy zz xy xz yz)
// as the reference's membrane math states them (membrane.cpp:153-257);
// false when the matrix is not positive definite or the inverse is rejected.
__device__ bool guard_solve(const double* m, const double* rhs, double* out) {
    if (!isfinite(m[0]) || !isfinite(m[1]) || !isfinite(m[2]) || !isfinite(m[3]) || !isfinite(m[4]) ||
        !isfinite(m[5]) || !(m[0] > 0.0) || !(m[1] > 0.0) || !(m[2] > 0.0))
        return false;
    const double sx = sqrt(m[0]), sy = sqrt(m[1]), sz = sqrt(m[2]);
    const double l10 = m[3] / sx / sy, l20 = m[4] / sx / sz;
    const double p1 = 1.0 - l10 * l10;
    if (!isfinite(p1) || !(p1 > 0.0)) return false;
    const double l11 = sqrt(p1);
    const double l21 = (m[5] / sy / sz - l20 * l10) / l11;
    const double p2 = 1.0 - l20 * l20 - l21 * l21;
    if (!isfinite(p2) || !(p2 > 0.0)) return false;
    double scale = 0.0;
    for (int k = 0; k < 6; ++k) scale = fmax(scale, fabs(m[k]));
    const double det = m[0] * (m[1] * m[2] - m[5] * m[5]) - m[3] * (m[3] * m[2] - m[5] * m[4]) +
                       m[4] * (m[3] * m[5] - m[1] * m[4]);
    if (!isfinite(det) || fabs(det) <= 128.0 * 2.220446049250313e-16 * scale * scale * scale) return false;
    const double id = 1.0 / det;
    const double ixx = (m[1] * m[2] - m[5] * m[5]) * id, iyy = (m[0] * m[2] - m[4] * m[4]) * id,
                 izz = (m[0] * m[1] - m[3] * m[3]) * id, ixy = (m[4] * m[5] - m[3] * m[2]) * id,
                 ixz = (m[3] * m[5] - m[4] * m[1]) * id, iyz = (m[3] * m[4] - m[0] * m[5]) * id;
    out[0] = ixx * rhs[0] + ixy * rhs[1] + ixz * rhs[2];
    out[1] = ixy * rhs[0] + iyy * rhs[1] + iyz * rhs[2];
    out[2] = ixz * rhs[0] + iyz * rhs[1] + izz * rhs[2];
    return true;
}

// Projects one membrane record: its three corners through the cluster
// window like apply_record, the step-start positions (damping) from global
// memory by slot (pbeg = the structure's patch starts).  False when the
// element's system has no inverse (the corners are then left as they were).
__device__ __noinline__ bool apply_membrane(const ClusterRecord& r, uint32_t me, uint32_t rank_base,
                                            uint32_t x_base, float* lam, uint32_t first, const float4* aux,
                                            const float4* pos_in, const uint32_t* pbeg, float inv_dt,
                                            float inv_dt2) {
    const uint32_t ra = r.ab & 0xffffu, rb = r.ab >> 16, rc = r.cd & 0xffffu;
    const uint32_t pa = node_addr(ra, me, rank_base, x_base);
    const uint32_t pb = node_addr(rb, me, rank_base, x_base);
    const uint32_t pc = node_addr(rc, me, rank_base, x_base);
    float4 A = ld_node(pa), B = ld_node(pb), C = ld_node(pc);
    const MembraneConst m = load_membrane(aux, r.index);
    float3 PA = make_float3(0.0f, 0.0f, 0.0f), PB = PA, PC = PA;
    if (m.damping_time != 0.0f) {
        PA = f3(__ldg(pos_in + pbeg[ra >> 12] + (ra & 0xfffu)));
        PB = f3(__ldg(pos_in + pbeg[rb >> 12] + (rb & 0xfffu)));
        PC = f3(__ldg(pos_in + pbeg[rc >> 12] + (rc & 0xfffu)));
    }
    const bool ok = project_membrane(A, B, C, PA, PB, PC, m, lam + 3 * (r.index - first), inv_dt, inv_dt2);
    st_node(pa, A);
    st_node(pb, B);
    st_node(pc, C);
    return ok;
}

// Projects one record.  Taping launches first store the record's inputs
// (node positions and multiplier) at its index in this iteration's tape
// blocks of `rtotal` entries.
template <bool kTape = false>
__device__ __forceinline__ void apply_record(const ClusterRecord& r, int kind, uint32_t me, uint32_t rank_base,
                                             uint32_t x_base, float* lam, uint32_t first, float inv_dt2,
                                             float4* tape = nullptr, uint32_t rtotal = 0) {
    const uint32_t pa = node_addr(r.ab & 0xffffu, me, rank_base, x_base);
    const uint32_t pb = node_addr(r.ab >> 16, me, rank_base, x_base);
    float l = lam[r.index - first];
    if (kind == 0) {
        float4 A = ld_node(pa), B = ld_node(pb);
        if constexpr (kTape) {
            tape[r.index] = make_float4(A.x, A.y, A.z, l);
            tape[rtotal + r.index] = B;
        }
        project_distance(A, B, r.rest, r.comp, l, inv_dt2);
        st_node(pa, A);
        st_node(pb, B);
    } else {
        const uint32_t pc = node_addr(r.cd & 0xffffu, me, rank_base, x_base);
        const uint32_t pd = node_addr(r.cd >> 16, me, rank_base, x_base);
        float4 A = ld_node(pa), B = ld_node(pb), C = ld_node(pc), D = ld_node(pd);
        if constexpr (kTape) {
            tape[r.index] = make_float4(A.x, A.y, A.z, l);
            tape[rtotal + r.index] = B;
            tape[2 * rtotal + r.index] = C;
            tape[3 * rtotal + r.index] = D;
        }
        project_dihedral(A, B, C, D, r.rest, r.comp, l, inv_dt2);
        st_node(pa, A);
        st_node(pb, B);
        st_node(pc, C);
        st_node(pd, D);
    }
    lam[r.index - first] = l;
}

// Records the pilot's inputs of a line iteration (or of the finish).
__device__ __forceinline__ void tape_pilot(PilotTape& t, const DevPayloadState& pay, const AdjointPilot& ap,
                                           const float4* x, const float4* v) {
    t.com[0] = pay.com.x; t.com[1] = pay.com.y; t.com[2] = pay.com.z;
    t.q[0] = pay.q.x; t.q[1] = pay.q.y; t.q[2] = pay.q.z; t.q[3] = pay.q.w;
    for (int k = 0; k < 8; ++k) t.lambda[k] = pay.lambda[k];
    for (int s = 0; s < ap.slots; ++s) {
        t.xs[s] = x[ap.slot_node[s]];
        if (v) t.vs[s] = v[ap.slot_node[s]];
    }
}

// The ground plane (swb_structure_set_ground) on this CTA's nodes: a free
// node below the plane is moved back onto it along the normal; with
// friction its motion along the plane since the step start (`start`) is
// then stopped while it is at most friction x the correction, else
// shortened by that length.  `tape` (taping launches) records which nodes
// the plane moved.
__device__ __forceinline__ void ground_pass(float4* x, uint32_t n, float3 nrm, float off, float mu,
                                            const float4* start, uint8_t* tape) {
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        float4 X = x[i];
        const float c = X.w != 0.0f ? dot(nrm, f3(X)) - off : 0.0f;
        const bool active = c < 0.0f;
        if (active) {
            X.x -= c * nrm.x;
            X.y -= c * nrm.y;
            X.z -= c * nrm.z;
            if (mu > 0.0f) {
                const float4 P = __ldg(start + i);
                float3 d = make_float3(X.x - P.x, X.y - P.y, X.z - P.z);
                d = d - nrm * dot(nrm, d);
                const float len = length(d), lim = -mu * c;
                const float k = len <= lim ? 1.0f : lim / len;
                X.x -= d.x * k;
                X.y -= d.y * k;
                X.z -= d.z * k;
            }
            x[i] = X;
        }
        if (tape) tape[i] = active ? 1u : 0u;
    }
}

// kPacked = false: one structure per cluster (cluster index = structure).
// One load-path cable pair (soft_body.cpp:1265-1286): the levels of the
// reverse and the forward pass over this CTA's cable and tie records, a
// cluster barrier after each level.  Out of line: only runs with pairs.
__device__ __noinline__ void run_cable_pair(const ClusterInstance& I, uint32_t me, uint32_t rank_base,
                                            uint32_t x_base, float* lam0, uint32_t first0, float inv_dt2) {
    cooperative_groups::cluster_group cluster = cooperative_groups::this_cluster();
    const uint32_t* off = I.pair_offsets + static_cast<size_t>(me) * (I.pair_stages + 1);
    for (int l = 0; l < I.pair_stages; ++l) {
        const uint32_t hi = __ldg(off + l + 1);
        for (uint32_t i = __ldg(off + l) + threadIdx.x; i < hi; i += blockDim.x) {
            const uint32_t r = __ldg(I.pair_rec + i);
            apply_record<false>(load_record(I.kind[0].rec, r, r + 1), 0, me, rank_base, x_base, lam0, first0,
                                inv_dt2);
        }
        cluster.sync();
    }
}

// kPacked = true: a cluster carries several structures, each on its own
// contiguous range of ranks, all in lockstep over the cluster's stage count;
// the structure's buffers follow the launch role and its committed-buffer
// rotation (see ClusterParams).
// kTape = true: one structure per cluster; the step also records the inputs
// of every projection, line iteration and the pilot finish into p.tape for
// the reverse sweep of the adjoint.
// kMembrane = true: the launch's structures may carry membrane elements
// (a third record kind); without it their stage count is taken as zero.
template <bool kPacked, bool kTape = false, bool kMembrane = false, bool kContact = false>
__global__ void __launch_bounds__(kClusterMaxThreads) xpbd_cluster_kernel_t(const __grid_constant__ ClusterParams p) {
    static_assert(!(kContact && (kPacked || kTape)), "contact runs in single-structure forward launches only");
    namespace cg = cooperative_groups;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint64_t bar;
    __shared__ DevPayloadState pay;
    __shared__ DevPayloadDef pdef;  // suspension CTA: the payload definition, read on every line iteration
    __shared__ float4* peers[16];
    __shared__ float3 shift_s;
    __shared__ uint32_t pbeg_s[kClusterMaxCtasDev + 1];  // the structure's patch starts
    __shared__ double mom_scratch[kMaxWarps * kMomentumFields];
    __shared__ double mom_pred[kMomentumFields], mom_cur[kMomentumFields];
    __shared__ double mom_ptot[kMomentumFields], mom_tot[kMomentumFields];
    cg::cluster_group cluster = cg::this_cluster();
    if constexpr (kContact) {
        // a helper cluster of a contact launch: only the detection phases
        if (blockIdx.x >= static_cast<unsigned>(p.ctas)) {
            const ClusterInstance& I0 = p.instances[0];
            ContactCtx h{};
            h.C = I0.contact;
            h.me = cluster.block_rank();
            h.ctas = p.ctas;
            h.pos_in = I0.pos_in;
            for (int k = 0; k < 3; ++k) h.o[k] = I0.origin_in[k];
            h.dt = p.dt64;
            h.status = I0.status;
            h.grank = blockIdx.x;
            h.gctas = gridDim.x;
            h.helpers = p.helper_clusters;
            h.grid = p.grid;
            h.grid.status = I0.status;
            h.grid.blocks = gridDim.x;
            contact_helper(h, cluster, p.iterations);
            return;
        }
    }
    ClusterSlot slot{};
    if constexpr (kPacked) {
        slot = p.slots[blockIdx.x];
        if (slot.instance < 0) {
            // idle rank: take every cluster barrier the busy ranks take
            const int barriers = 3 + p.iterations * (slot.stages + slot.suspension + (p.ground ? 1 : 0)) +
                                 (p.iterations > 0 ? slot.seam_stages : 0) + (slot.guard && !p.ground ? 3 : 0);
            for (int b = 0; b < barriers; ++b) cluster.sync();
            return;
        }
    }
    const uint32_t rank_base = kPacked ? static_cast<uint32_t>(slot.rank_base) : 0u;
    const uint32_t me = cluster.block_rank() - rank_base;
    const ClusterInstance& I =
        kPacked ? p.instances[(static_cast<size_t>(slot.instance) * 3 + p.rotation[slot.instance]) * 3 + p.role]
                : p.instances[blockIdx.x / p.ctas];
    const int tid = threadIdx.x;
    float4* x = reinterpret_cast<float4*>(smem + p.smem_x);
    float4* v = reinterpret_cast<float4*>(smem + p.smem_v);
    float* lam0 = reinterpret_cast<float*>(smem + I.kind[0].smem_lambda);
    float* lam1 = reinterpret_cast<float*>(smem + I.kind[1].smem_lambda);
    float* lam2 = reinterpret_cast<float*>(smem + I.kind[2].smem_lambda);  // three per membrane record
    const uint32_t base = __ldg(I.patch_begin + me);
    const uint32_t n = __ldg(I.patch_begin + me + 1) - base;
    const bool owner = static_cast<int>(me) == I.susp_cta;
    const uint32_t x_base = smem_addr(x);
    // momentum guard: `guard` = this structure runs it; `guard_c` = the
    // cluster takes its barriers (a packed cluster when any of its
    // structures runs it); `sctas` = the structure's ranks
    // a ground plane is an external load, as the pilot's lines and contact
    // are: the momentum guard stands down while one is set
    const bool guard = I.momentum_guard != 0 && !p.ground;
    const bool guard_c = kPacked ? slot.guard != 0 && !p.ground : guard;
    // line-line contact: the substep's candidate pairs are counted afresh
    const LineContactDev* lines = kPacked ? nullptr : I.lines;
    auto line_addr = [&](uint32_t ref) { return node_addr(ref, me, rank_base, x_base); };
    if (lines && me == 0 && tid == 0) *lines->count = 0;
    const float ground_off =
        p.ground ? static_cast<float>(p.ground_offset - (p.ground_normal.x * I.origin_in[0] +
                                                         p.ground_normal.y * I.origin_in[1] +
                                                         p.ground_normal.z * I.origin_in[2]))
                 : 0.0f;
    const int sctas = kPacked ? slot.ctas : p.ctas;

    if (tid < p.ctas) peers[tid] = cluster.map_shared_rank(x, tid);
    if (tid == 0) {
        mbar_init(&bar, 1);
        mbar_expect_tx(&bar, n * 16u);
        if (n) bulk_load(x, I.pos_in + base, n * 16u, &bar);
    }
    // multipliers restart every substep (soft_body.cpp:1207-1218)
    for (int k = 0; k < (kMembrane ? 3 : 2); ++k) {
        const uint32_t* off = I.kind[k].offsets + static_cast<size_t>(me) * (I.kind[k].stages + 1);
        const uint32_t cnt = (__ldg(off + I.kind[k].stages) - __ldg(off)) * (k == 2 ? 3u : 1u);
        float* lam = k == 0 ? lam0 : (k == 1 ? lam1 : lam2);
        for (uint32_t i = tid; i < cnt; i += blockDim.x) lam[i] = 0.0f;
    }
    if (tid <= sctas) pbeg_s[tid] = __ldg(I.patch_begin + tid);
    ContactCtx cctx{};
    if constexpr (kContact) {
        cctx.C = I.contact;
        cctx.me = me;
        cctx.ctas = p.ctas;
        cctx.x = x;
        cctx.v = v;
        cctx.base = base;
        cctx.n = n;
        cctx.pbeg = pbeg_s;
        cctx.pos_in = I.pos_in;
        for (int k = 0; k < 3; ++k) cctx.o[k] = I.origin_in[k];
        cctx.dt = p.dt64;
        cctx.status = I.status;
        cctx.x_base = smem_addr(x);
        cctx.v_delta = smem_addr(v) - smem_addr(x);
        cctx.grank = me;
        cctx.gctas = gridDim.x;
        cctx.helpers = p.helper_clusters;
        cctx.grid = p.grid;
        cctx.grid.status = I.status;
        cctx.grid.blocks = gridDim.x;
        // multipliers and records restart every substep (beginContactSubstep,
        // contact.cpp:1043-1055)
        if (me == 0 && tid == 0) {
            I.contact->table_meta[0] = 0;
            I.contact->table_meta[1] = 0;
        }
    }
    // pressure gather (ascending triangle order) into v
    for (uint32_t i = tid; i < n; i += blockDim.x) {
        const uint32_t slot = base + i;
        float3 f = f3(__ldg(I.force + slot));
        const uint32_t lo = __ldg(I.tri_offsets + slot), hi = __ldg(I.tri_offsets + slot + 1);
        for (uint32_t q = lo; q < hi; ++q) {
            const uint4 t = __ldg(I.tri + __ldg(I.tri_list + q));
            const float3 pa = f3(__ldg(I.pos_in + t.x));
            const float3 pb = f3(__ldg(I.pos_in + t.y));
            const float3 pc = f3(__ldg(I.pos_in + t.z));
            const float3 area = 0.5f * cross(pb - pa, pc - pa);
            f = f + (__uint_as_float(t.w) * area) / 3.0f;
        }
        v[i] = make_float4(f.x, f.y, f.z, 0.0f);
    }
    if (owner && tid == 0) pay = *I.payload_in;
    if (owner)
        for (uint32_t i = tid; i < sizeof(DevPayloadDef) / 4; i += blockDim.x)
            reinterpret_cast<uint32_t*>(&pdef)[i] = __ldg(reinterpret_cast<const uint32_t*>(I.payload_def) + i);
    __syncthreads();  // mbarrier initialised before any thread waits on it
    if (!mbar_wait(&bar, 0, p.copy_budget)) {
        atomicOr(I.status, kStatusCopyTimeout);
        mbar_wait(&bar, 0, p.copy_budget);
    }
    // predict (soft_body.cpp:1536-1566)
    for (uint32_t i = tid; i < n; i += blockDim.x) {
        float4 X = x[i];
        if (X.w == 0.0f) continue;
        const float4 V0 = __ldg(I.vel_in + base + i);
        const float4 F = v[i];
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
        x[i] = X;
        if (guard) v[i] = make_float4(vx, vy, vz, 0.0f);  // the predicted velocity, for the momentum guard
    }
    if (owner && tid == 0) {
        for (int k = 0; k < 8; ++k) pay.lambda[k] = 0.0f;
        if (!payload_predict(pdef, pay, p.dt, p.gravity)) susp_fail(I.status, kSuspPredict);
    }
    if (guard) {
        // momentum of the predicted state (the guard's target)
        __syncthreads();
        cta_momentum_sums(x, v, n, mom_pred, mom_scratch);
    }
    cluster.sync();
    if (lines) {
        line_broadphase(*lines, me, static_cast<uint32_t>(sctas), cluster, line_addr, I.status);
        cluster.sync();
        if (me == 0) line_sort(*lines, lines->sort);
        if constexpr (kTape) {
            if (me == 0 && !line_tape_step(*lines, p.tape) && tid == 0) contact_fail(I.status, kContactLineTape);
        }
    }

    // ---- constraint iterations ------------------------------------------------
    // Stages of one iteration: distance colours, membrane colours, then
    // dihedral colours.  Each thread prefetches its first record of the next
    // stage before it works on the current one, so the record fetch from L2
    // overlaps the current stage and its cluster barrier.
    const int S0 = I.kind[0].stages, S1 = I.kind[1].stages, S2 = kMembrane ? I.kind[2].stages : 0,
              S = S0 + S1 + S2;
    const int stages_c = kPacked ? slot.stages : S;                       // cluster-wide
    const bool susp_c = kPacked ? slot.suspension != 0 : I.susp_cta >= 0;  // cluster-wide
    const int seam_c = kPacked ? slot.seam_stages : I.seam_stages;         // cluster-wide
    // this CTA's stage offsets, kind by kind: [S0 + 1] distance, [S1 + 1]
    // dihedral, [S2 + 1] membrane
    uint32_t* soff = reinterpret_cast<uint32_t*>(smem + p.smem_offsets);
    for (int k = 0; k < (kMembrane ? 3 : 2); ++k) {
        const int at = k == 0 ? 0 : (k == 1 ? S0 + 1 : S0 + S1 + 2);
        for (int i = tid; i <= I.kind[k].stages; i += blockDim.x)
            soff[at + i] = __ldg(I.kind[k].offsets + static_cast<size_t>(me) * (I.kind[k].stages + 1) + i);
    }
    __syncthreads();
    // global stage g -> kind, its stage within the kind, and its offsets
    // (plain arithmetic: without membranes S2 is the constant 0 and these
    // reduce to the two-kind forms)
    auto kind_of = [&](int g) { return g < S0 ? 0 : (g < S0 + S2 ? 2 : 1); };
    auto local_of = [&](int g) { return g < S0 ? g : (g < S0 + S2 ? g - S0 : g - S0 - S2); };
    auto stage_at = [&](int g) {
        return g < S0 ? g : (g < S0 + S2 ? S0 + S1 + 2 + (g - S0) : S0 + 1 + (g - S0 - S2));
    };
    auto stage_lo = [&](int g) { return soff[stage_at(g)]; };
    auto stage_hi = [&](int g) { return soff[stage_at(g) + 1]; };
    const uint32_t first0 = soff[0], first1 = soff[S0 + 1], first2 = kMembrane ? soff[S0 + S1 + 2] : 0u;
    // record arrays held in registers (the instance record lives in global memory)
    const uint4* rec0 = I.kind[0].rec;
    const uint4* rec1 = I.kind[1].rec;
    const uint4* rec2 = I.kind[2].rec;
    auto recs = [&](int k) { return k == 0 ? rec0 : (k == 1 ? rec1 : rec2); };
    auto apply = [&](const ClusterRecord& r, int kind, float* lam, uint32_t first, float4* tape, uint32_t rtotal) {
        if constexpr (kMembrane) {
            if (kind == 2) {
                if (!apply_membrane(r, me, rank_base, x_base, lam, first, I.kind[2].aux, I.pos_in, pbeg_s, p.inv_dt,
                                    p.inv_dt2))
                    atomicOr(I.status, kStatusMembrane);
                return;
            }
        }
        apply_record<kTape>(r, kind, me, rank_base, x_base, lam, first, p.inv_dt2, tape, rtotal);
    };
    ClusterRecord next;
    next.index = ~0u;
    if (p.iterations > 0 && S > 0) next = load_record(recs(kind_of(0)), stage_lo(0) + tid, stage_hi(0));
    const uint64_t sync0 = I.kind[0].sync_mask, sync1 = I.kind[1].sync_mask;
    // line iteration beside the last two stages: neither touches a
    // suspension endpoint node, so running it there gives the same result as
    // running it after them.  The last warp of the suspension CTA (no record
    // in either stage) arrives at the first stage's barrier, runs the line
    // iteration, then waits; its writes are released at its arrival on the
    // second stage's barrier, before the next iteration reads them.
    const int line_stage = !kPacked && susp_c ? I.line_stage : -1;
    const bool line_warp = line_stage >= 0 && owner && (tid >> 5) == static_cast<int>(blockDim.x >> 5) - 1;
    // load-path cable sweeps (soft_body.cpp:1288-1317): a quarter of the
    // pairs runs before the general sweeps of the first iterations, the rest
    // closes the substep (all of them without iterations)
    const int pairs = (kPacked || kTape) ? 0 : p.cable_pairs;
    const int closing_pairs = pairs > 0 ? pairs - pairs / 4 : 0;
    const int interleaved_pairs = pairs - closing_pairs;
    const int pair_iters = p.iterations > 1 ? p.iterations : 1;
    for (int it = 0; it < p.iterations; ++it) {
        if (pairs > 0) {
            const int n_pairs = interleaved_pairs / pair_iters + (it < interleaved_pairs % pair_iters ? 1 : 0);
            for (int q = 0; q < n_pairs; ++q) run_cable_pair(I, me, rank_base, x_base, lam0, first0, p.inv_dt2);
        }
        for (int g = 0; g < stages_c; ++g) {
            if (!kPacked || g < S) {
                const int kind = kind_of(g);
                const ClusterRecord cur = next;
                // prefetch the next stage (wrapping to the next iteration)
                const int gn = g + 1 < S ? g + 1 : 0;
                next = load_record(recs(kind_of(gn)), stage_lo(gn) + tid, stage_hi(gn));
                const uint32_t first = kind == 0 ? first0 : (kind == 1 ? first1 : first2);
                float* lam = kind == 0 ? lam0 : (kind == 1 ? lam1 : lam2);
                float4* tape = nullptr;
                uint32_t rtotal = 0;
                if constexpr (kTape) {
                    rtotal = kind ? p.tape.r1 : p.tape.r0;
                    tape = (kind ? p.tape.dih : p.tape.dist) + static_cast<size_t>(it) * (kind ? 4 : 2) * rtotal;
                }
                if (cur.index != ~0u) apply(cur, kind, lam, first, tape, rtotal);
                for (uint32_t i = stage_lo(g) + tid + blockDim.x; i < stage_hi(g); i += blockDim.x)
                    apply(load_record(recs(kind), i, stage_hi(g)), kind, lam, first, tape, rtotal);
            }
            if (g == line_stage) {
                if (line_warp) {
                    cluster_arrive();
                    if ((tid & 31) == 0) {
                        if constexpr (kTape) tape_pilot(p.tape.line[it], pay, *p.tape.pilot, x, nullptr);
                        line_iteration(pdef, pay, x, p.dt, I.status);
                    }
                    __syncwarp();
                    cluster_wait();
                } else {
                    cluster.sync();
                }
            } else if constexpr (kPacked) {
                cluster.sync();
            } else {
                // split stages: a CTA barrier between two stages of records
                // that touch only the CTA's own patch, else a cluster barrier;
                // membrane stages are classic
                const int kind = kind_of(g);
                const int gl = local_of(g);
                const uint64_t mask = kind == 0 ? sync0 : sync1;
                if (kind == 2 || gl >= 64 || ((mask >> gl) & 1ull))
                    cluster.sync();
                else
                    __syncthreads();
            }
        }
        if (susp_c && line_stage < 0) {
            if (owner && tid == 0) {
                if constexpr (kTape) tape_pilot(p.tape.line[it], pay, *p.tape.pilot, x, nullptr);
                line_iteration(pdef, pay, x, p.dt, I.status);
            }
            cluster.sync();
        }
        if constexpr (kContact) contact_iteration(cctx, cluster);
        if (lines) {
            float4* line_tape = nullptr;
            if constexpr (kTape) {
                if (lines->count[0] <= p.tape.line_cap)
                    line_tape = p.tape.line_in + static_cast<size_t>(it) * p.tape.line_cap * 4;
            }
            if (me == 0) line_project(*lines, line_addr, line_tape);
            cluster.sync();
        }
        if (p.ground) {
            uint8_t* gt = nullptr;
            if constexpr (kTape) gt = p.tape.ground + static_cast<size_t>(it) * pbeg_s[sctas] + base;
            ground_pass(x, n, p.ground_normal, ground_off, p.ground_friction, I.pos_in + base, gt);
            cluster.sync();
        }
    }
    // closing cable pairs
    for (int q = 0; q < (p.iterations > 0 ? closing_pairs : pairs); ++q)
        run_cable_pair(I, me, rank_base, x_base, lam0, first0, p.inv_dt2);
    // ---- final seam-stitch projections (soft_body.cpp:1389-1405) ----------
    if (p.iterations > 0) {
        for (int s = 0; s < seam_c; ++s) {
            const uint32_t* off = I.seam_offsets + static_cast<size_t>(me) * (I.seam_stages + 1);
            const uint32_t lo = s < I.seam_stages ? __ldg(off + s) : 0u;
            const uint32_t hi = s < I.seam_stages ? __ldg(off + s + 1) : 0u;
            for (uint32_t i = lo + tid; i < hi; i += blockDim.x) {
                const uint32_t r = __ldg(I.seam_ab + i);
                float4* pa = node_at(r & 0xffffu, me, rank_base, x, peers);
                float4* pb = node_at(r >> 16, me, rank_base, x, peers);
                float4 A = *pa, B = *pb;
                if constexpr (kTape) {
                    p.tape.seam[i] = A;
                    p.tape.seam[p.tape.rs + i] = B;
                }
                float l = 0.0f;  // rigid stitch: alpha = 0
                project_distance(A, B, 0.0f, 0.0f, l, p.inv_dt2);
                *pa = A;
                *pb = B;
            }
            cluster.sync();
        }
    }
    // ---- contact certification of the final state (soft_body.cpp:1411-1418) --
    if constexpr (kContact) contact_certify(cctx, cluster, I.contact_diag);
    // ---- membrane residuals after the iterations (soft_body.cpp:2366-2404) ---
    if (kMembrane && S2 > 0) {
        const uint32_t lo = soff[S0 + S1 + 2], hi = soff[S0 + S1 + 2 + S2];
        for (uint32_t i = lo + tid; i < hi; i += blockDim.x) {
            const uint4 q = __ldg(rec2 + i);
            const uint32_t ra = q.x & 0xffffu, rb = q.x >> 16, rc = q.y & 0xffffu;
            const float4 A = ld_node(node_addr(ra, me, rank_base, x_base));
            const float4 B = ld_node(node_addr(rb, me, rank_base, x_base));
            const float4 C = ld_node(node_addr(rc, me, rank_base, x_base));
            const MembraneConst m = load_membrane(I.kind[2].aux, i);
            float3 PA = make_float3(0.0f, 0.0f, 0.0f), PB = PA, PC = PA;
            if (m.damping_time != 0.0f) {
                PA = f3(__ldg(I.pos_in + pbeg_s[ra >> 12] + (ra & 0xfffu)));
                PB = f3(__ldg(I.pos_in + pbeg_s[rb >> 12] + (rb & 0xfffu)));
                PC = f3(__ldg(I.pos_in + pbeg_s[rc >> 12] + (rc & 0xfffu)));
            }
            I.membrane_residual[i] = membrane_residual(f3(A), f3(B), f3(C), PA, PB, PC, m, lam2 + 3 * (i - first2),
                                                       p.inv_dt, p.inv_dt2);
        }
    }
    // ---- finalize (soft_body.cpp:1568-1585) --------------------------------
    for (uint32_t i = tid; i < n; i += blockDim.x) {
        const float4 X = x[i];
        float4 V = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (X.w != 0.0f) {
            const float4 P = __ldg(I.pos_in + base + i);
            V = make_float4((X.x - P.x) * p.inv_dt, (X.y - P.y) * p.inv_dt, (X.z - P.z) * p.inv_dt, 0.0f);
        }
        v[i] = V;
    }
    __syncthreads();
    if (guard_c) {
        // restoreMomentum (soft_body.cpp:152-190): the linear momentum of the
        // predicted state by a uniform velocity change, then its angular
        // momentum about the centre of mass by a rigid rotation rate.  Three
        // cluster barriers whatever the structure (packed clusters take them
        // on every rank).
        if (guard) cta_momentum_sums(x, v, n, mom_cur, mom_scratch);
        cluster.sync();
        bool go = false;
        MomentumTotals target{};
        if (guard) {
            cluster_momentum_totals(cluster, mom_pred, sctas, rank_base, mom_ptot);
            cluster_momentum_totals(cluster, mom_cur, sctas, rank_base, mom_tot);
            target = momentum_of(mom_ptot);
            const MomentumTotals now = momentum_of(mom_tot);
            go = target.mass > 0.0;
            if (go) {
                const float dvx = static_cast<float>((target.p[0] - now.p[0]) / target.mass);
                const float dvy = static_cast<float>((target.p[1] - now.p[1]) / target.mass);
                const float dvz = static_cast<float>((target.p[2] - now.p[2]) / target.mass);
                for (uint32_t i = tid; i < n; i += blockDim.x)
                    if (x[i].w > 0.0f) {
                        float4 V = v[i];
                        V.x += dvx; V.y += dvy; V.z += dvz;
                        v[i] = V;
                    }
            }
            __syncthreads();
        }
        cluster.sync();  // every CTA has read the sums before they are replaced
        if (go) cta_momentum_sums(x, v, n, mom_cur, mom_scratch);
        cluster.sync();
        if (go) {
            cluster_momentum_totals(cluster, mom_cur, sctas, rank_base, mom_tot);
            const double* t = mom_tot;
            const MomentumTotals c = momentum_of(t);
            // inertia about the centre of mass from the second moments
            const double M = t[0];
            const double sxx = t[10] - M * c.com[0] * c.com[0], syy = t[11] - M * c.com[1] * c.com[1],
                         szz = t[12] - M * c.com[2] * c.com[2], sxy = t[13] - M * c.com[0] * c.com[1],
                         sxz = t[14] - M * c.com[0] * c.com[2], syz = t[15] - M * c.com[1] * c.com[2];
            const double inertia[6] = {syy + szz, sxx + szz, sxx + syy, -sxy, -sxz, -syz};
            const double dL[3] = {target.L[0] - c.L[0], target.L[1] - c.L[1], target.L[2] - c.L[2]};
            double w[3];
            if (guard_solve(inertia, dL, w))
                for (uint32_t i = tid; i < n; i += blockDim.x) {
                    const float4 X = x[i];
                    if (!(X.w > 0.0f)) continue;
                    const double rx = X.x - c.com[0], ry = X.y - c.com[1], rz = X.z - c.com[2];
                    float4 V = v[i];
                    V.x += static_cast<float>(w[1] * rz - w[2] * ry);
                    V.y += static_cast<float>(w[2] * rx - w[0] * rz);
                    V.z += static_cast<float>(w[0] * ry - w[1] * rx);
                    v[i] = V;
                }
            __syncthreads();
        }
    }
    // ---- the payload's velocity and line damping, contact friction on the
    // finalized velocities, the payload's certification (soft_body.cpp:
    // 1447-1457)
    bool finish_ok = true;
    if constexpr (kContact) {
        if (owner && tid == 0) finish_ok = payload_reconstruct_damp(pdef, pay, *I.payload_in, x, v, p.dt, I.status);
        contact_friction(cctx, cluster, I.contact_diag);
    }
    if (owner && tid == 0) {
        if constexpr (kTape) tape_pilot(*p.tape.finish, pay, *p.tape.pilot, x, v);
        if constexpr (kContact) {
            if (finish_ok) payload_certify_finish(pdef, pay, x, v, p.dt, I.status);
        } else {
            payload_finish(pdef, pay, *I.payload_in, x, v, p.dt, I.status);
        }
        float3 s = make_float3(0.0f, 0.0f, 0.0f);
        if (I.recentre && finite3(pay.com) &&
            fmaxf(fabsf(pay.com.x), fmaxf(fabsf(pay.com.y), fabsf(pay.com.z))) > 0.25f)
            s = make_float3(rintf(pay.com.x * 256.0f) / 256.0f, rintf(pay.com.y * 256.0f) / 256.0f,
                            rintf(pay.com.z * 256.0f) / 256.0f);
        shift_s = s;
    }
    if (I.susp_cta < 0 && tid == 0) shift_s = make_float3(0.0f, 0.0f, 0.0f);
    cluster.sync();
    float3 shift = shift_s;
    if (I.susp_cta >= 0) shift = *cluster.map_shared_rank(&shift_s, I.susp_cta + static_cast<int>(rank_base));
    // ---- write the trial state --------------------------------------------
    int bad = 0;
    for (uint32_t i = tid; i < n; i += blockDim.x) {
        float4 X = x[i];
        float4 P = __ldg(I.pos_in + base + i);
        const float4 V = v[i];
        X.x -= shift.x; X.y -= shift.y; X.z -= shift.z;
        P.x -= shift.x; P.y -= shift.y; P.z -= shift.z;
        bad |= !(isfinite(X.x) && isfinite(X.y) && isfinite(X.z) && isfinite(V.x) && isfinite(V.y) && isfinite(V.z));
        I.pos_out[base + i] = X;
        I.prev_out[base + i] = P;
        I.vel_out[base + i] = V;
    }
    if (__syncthreads_or(bad) && tid == 0) atomicOr(I.status, kStatusNonFinite);
    if (owner && tid == 0) {
        pay.com = pay.com - shift;
        *I.payload_out = pay;
    }
    if (me == 0 && tid == 0) {
        I.origin_out[0] = I.origin_in[0] + static_cast<double>(shift.x);
        I.origin_out[1] = I.origin_in[1] + static_cast<double>(shift.y);
        I.origin_out[2] = I.origin_in[2] + static_cast<double>(shift.z);
    }
    cluster.sync();  // no CTA leaves while a peer may still read its memory
}

// One structure per cluster (the plain step) and several structures per
// cluster (the batched step).
inline constexpr auto xpbd_cluster_kernel = &xpbd_cluster_kernel_t<false>;
inline constexpr auto xpbd_cluster_packed_kernel = &xpbd_cluster_kernel_t<true>;
// The same with membrane elements.
inline constexpr auto xpbd_cluster_membrane_kernel = &xpbd_cluster_kernel_t<false, false, true>;
inline constexpr auto xpbd_cluster_packed_membrane_kernel = &xpbd_cluster_kernel_t<true, false, true>;
// One structure per cluster with fabric self-contact.
inline constexpr auto xpbd_cluster_contact_kernel = &xpbd_cluster_kernel_t<false, false, false, true>;
inline constexpr auto xpbd_cluster_contact_membrane_kernel = &xpbd_cluster_kernel_t<false, false, true, true>;
// One structure per cluster, recording the adjoint's tape.
inline constexpr auto xpbd_cluster_tape_kernel = &xpbd_cluster_kernel_t<false, true>;

}  // namespace dev
}  // namespace swb
