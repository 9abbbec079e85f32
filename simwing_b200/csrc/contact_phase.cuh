// Fabric self-contact inside the cluster step kernel: the contact iteration
// after each iteration's constraint stages (SoftBody::solveContactIteration,
// contact.cpp:1057-1582), the certification after the seam pass
// (certifyContactState, contact.cpp:1583-2080) and the friction pass after
// finalize (applyContactFriction, contact.cpp:2081-2209).
//
// Each runs as phases over the whole cluster, a cluster barrier after each:
//   snapshot  every CTA writes its nodes' positions to global memory;
//   boxes     swept boxes of every proxy (step start -> snapshot);
//   count     one warp per candidate row counts its overlapping features;
//   scan      rank 0 turns the counts into row offsets;
//   write     the rows write their feature codes, in key order;
//   queries   per candidate, the swept query and the snapshot's closest
//             features (both read only the snapshot, as the reference's
//             candidates carry the positions of their emission);
//   serial    one thread walks the candidates in key order: the multiplier
//             warm starts, the projection on the live nodes (distributed
//             shared memory), the record book.
// Contact math is FP64 on the FP32-resident state.
#pragma once

#include "cluster_params.h"
#include "contact_geometry.cuh"
#include "device_common.cuh"

#include <cooperative_groups.h>

namespace swb {
namespace dev {

// Detail codes of kStatusContact (status[1]), one per ContactStepError
// the reference raises on the path, plus the device's capacities.
enum : int {
    kContactCcd = 1,             // "Contact CCD could not certify a supported feature"
    kContactGeometry = 2,        // "Contact endpoint geometry is not certifiable"
    kContactNormal = 3,          // "Contact normal is not finite/unit"
    kContactNoResponse = 4,      // "Penetrating contact has no movable/compliant response"
    kContactProjection = 5,      // "Non-finite contact projection"
    kContactSolved = 6,          // "Non-finite solved contact geometry"
    kContactFinalCcd = 7,        // "Final contact geometry could not be certified"
    kContactFinalGeometry = 8,   // "Final contact closest geometry is not certifiable"
    kContactFinalNonFinite = 9,  // "Final contact geometry is non-finite"
    kContactPenetration = 10,    // "Final contact penetration exceeds the certified gate"
    kContactLost = 11,           // "Applied contact impulse lost its supported feature"
    kContactCleared = 12,        // "Cleared contact final geometry is not certifiable"
    kContactClearedGate = 13,    // "Cleared contact failed final geometry certification"
    kContactFriction = 14,       // "Non-finite/positive contact friction work"
    kContactInput = 15,          // "Contact broadphase input failed" (non-finite positions)
    kContactCandidates = 16,     // more candidates than the device list holds
    kContactTable = 17,          // more warm-started features than the device table holds
    kContactRecords = 18,        // more records than the device book holds
    kContactLinePairs = 19,      // more line-line candidate pairs than the device list holds
    kContactLineTape = 20,       // more line-line candidates than a rollout's tape holds
};

__device__ __forceinline__ void contact_fail(int* status, int code) {
    if ((atomicOr(status, kStatusContact) & kStatusContact) == 0) status[1] = code;
}

// A failure that belongs to a candidate feature also records the feature.
// The reference's sweeps are key-ordered and throw at their first failing
// feature, so the device keeps the failing feature first in key order: the
// candidate code (row << 32 | col) packed with the detail code as
// row << 37 | col << 5 | detail (rows stay below 2^27), kept by atomicMin
// in C.fail, which is reset before every step.
__device__ __forceinline__ void contact_fail_at(const ContactDev& C, int* status, int detail,
                                                unsigned long long code) {
    const unsigned long long packed =
        ((code >> 32) << 37) | ((code & 0xffffffffull) << 5) | static_cast<unsigned long long>(detail);
    atomicMin(C.fail, packed);
    contact_fail(status, detail);
}

__device__ __forceinline__ bool contact_failed(const int* status) {
    return (*reinterpret_cast<const volatile int*>(status) & kStatusContact) != 0;
}

struct ContactCtx {
    const ContactDev* C;
    uint32_t me;               // this CTA's rank
    int ctas;
    float4* x;                 // this CTA's nodes (shared memory)
    float4* v;                 // this CTA's velocities (shared memory)
    uint32_t base, n;          // this CTA's slots
    const uint32_t* pbeg;      // patch starts (shared memory, ctas + 1)
    const float4* pos_in;      // step-start positions by slot
    double o[3];               // coordinate origin of the state
    double dt;
    int* status;
    uint32_t x_base;           // shared address of this CTA's node array
    uint32_t v_delta;          // offset from the node array to the velocity array
    // the detection phases run over every CTA of the launch: the structure's
    // cluster and `helpers` helper clusters (grank = this CTA's rank among
    // gctas), with the grid barrier between phases when there are helpers
    uint32_t grank, gctas;
    int helpers;
    GridBarrier grid;
};

// The barrier between two detection phases.
__device__ __forceinline__ void detect_sync(const ContactCtx& c, cooperative_groups::cluster_group& cluster) {
    if (c.helpers)
        grid_sync(c.grid);
    else
        cluster.sync();
}

using contact::D3;

__device__ __forceinline__ D3 world_of(const ContactCtx& c, float4 X) {
    return {c.o[0] + static_cast<double>(X.x), c.o[1] + static_cast<double>(X.y), c.o[2] + static_cast<double>(X.z)};
}

struct FeatureSlots {
    uint32_t kind;
    uint32_t f[3], s[3];
    int fc, sc;
};

__device__ __forceinline__ FeatureSlots feature_slots(const ContactDev& C, unsigned long long code) {
    const uint32_t row = static_cast<uint32_t>(code >> 32), col = static_cast<uint32_t>(code & 0xffffffffu);
    FeatureSlots q;
    if (row < C.nv) {
        q.kind = SWB_FEATURE_VERTEX_TRIANGLE;
        q.f[0] = C.vid[row];
        q.fc = 1;
        const uint3 t = C.tid[col];
        q.s[0] = t.x; q.s[1] = t.y; q.s[2] = t.z;
        q.sc = 3;
    } else {
        q.kind = SWB_FEATURE_EDGE_EDGE;
        const uint2 e = C.eid[row - C.nv], g = C.eid[col];
        q.f[0] = e.x; q.f[1] = e.y;
        q.s[0] = g.x; q.s[1] = g.y;
        q.fc = q.sc = 2;
    }
    return q;
}

// Order key of a double, monotone for every non-NaN value, so that
// unsigned 64-bit atomics take minima and maxima of doubles.
__device__ __forceinline__ unsigned long long order_key(double d) {
    const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(d));
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double from_order_key(unsigned long long k) {
    const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double(static_cast<long long>(b));
}

// Warp-reduced atomic minimum / maximum of order keys (every lane calls,
// `valid` marks the lanes that contribute).
__device__ __forceinline__ void warp_atomic_range(unsigned long long* lo_min, unsigned long long* lo_max,
                                                  unsigned long long* ext_max, bool valid, unsigned long long lo,
                                                  unsigned long long ext) {
    unsigned long long mn = valid ? lo : ~0ull, mx = valid ? lo : 0ull, ex = valid ? ext : 0ull;
    for (int d = 16; d > 0; d >>= 1) {
        mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, d));
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, d));
        ex = max(ex, __shfl_xor_sync(0xffffffffu, ex, d));
    }
    const bool any = __any_sync(0xffffffffu, valid);  // every lane takes part
    if ((threadIdx.x & 31) == 0 && any) {
        atomicMin(lo_min, mn);
        atomicMax(lo_max, mx);
        atomicMax(ext_max, ex);
    }
}

// One axis of a column set's grid: cell width at least the widest column
// box on that axis, so that the columns a row's box can overlap have their
// low ends in the cells from of(lo - widest) to of(hi).
struct Axis {
    double lo, width, widest;
    uint32_t count;
    __device__ uint32_t of(double x) const {
        if (!(x > lo)) return 0u;
        const double q = floor((x - lo) / width);
        return q >= static_cast<double>(count - 1) ? count - 1 : static_cast<uint32_t>(q);
    }
};

__device__ __forceinline__ Axis make_axis(const unsigned long long* range, uint32_t cap) {
    Axis b;
    b.lo = from_order_key(range[0]);
    const double hi = from_order_key(range[1]);
    b.widest = from_order_key(range[2]);
    if (!isfinite(b.lo) || !isfinite(hi) || !isfinite(b.widest) || hi < b.lo) {
        // no column contributed (an empty set): one cell
        b.lo = 0.0;
        b.width = 1.0;
        b.widest = 0.0;
        b.count = 1;
        return b;
    }
    const double span = hi - b.lo;
    b.width = fmax(b.widest, span / static_cast<double>(cap));
    if (!(b.width > 0.0)) b.width = 1.0;
    const double n = floor(span / b.width) + 1.0;
    b.count = n >= static_cast<double>(cap) ? cap : static_cast<uint32_t>(n);
    if (b.count == 0) b.count = 1;
    return b;
}

// A column set's grid on the two broadphase axes; cells numbered a-major,
// so the cells of one a-index form a contiguous run of bucketed columns.
struct Bins {
    Axis a, b;
    __device__ uint32_t count() const { return a.count * b.count; }
    __device__ uint32_t of(double xa, double xb) const { return a.of(xa) * b.count + b.of(xb); }
};

// range: the set's six keys (axis a: lo min, lo max, widest; axis b: the same)
__device__ __forceinline__ Bins make_bins(const unsigned long long* range, uint32_t cap) {
    uint32_t side = 1;
    while ((side + 1) * (side + 1) <= cap) ++side;
    Bins g;
    g.a = make_axis(range, side);
    g.b = make_axis(range + 3, side);
    return g;
}

// ---- parallel phases (every thread of the cluster; a barrier after each) ----

__device__ __forceinline__ void contact_snapshot(const ContactCtx& c) {
    const ContactDev& C = *c.C;
    for (uint32_t i = threadIdx.x; i < c.n; i += blockDim.x) C.snapshot[c.base + i] = c.x[i];
    const uint32_t gt = c.grank * blockDim.x + threadIdx.x, stride = c.gctas * blockDim.x;
    for (uint32_t i = gt; i <= C.bins_cap; i += stride) {
        C.tbin[i] = 0u;
        C.tbin_fill[i] = 0u;
        C.ebin[i] = 0u;
        C.ebin_fill[i] = 0u;
    }
    if (gt < 12) C.range[gt] = (gt % 3 == 0) ? ~0ull : 0ull;
}

static __device__ __noinline__ void contact_boxes(const ContactCtx& c) {
    const ContactDev& C = *c.C;
    const uint32_t total = C.nv + C.ne + C.nt;
    const uint32_t stride = c.gctas * blockDim.x;
    const int a = C.axis, a2 = C.axis2;
    // warp-uniform trip count: every lane takes part in the warp reductions
    for (uint32_t base = c.grank * blockDim.x + (threadIdx.x & ~31u); base < total; base += stride) {
        const uint32_t i = base + (threadIdx.x & 31);
        bool tri = false, edge = false;
        unsigned long long lo_key = 0, ext_key = 0, lo_key2 = 0, ext_key2 = 0;
        if (i < total) {
            uint32_t s[3];
            int count;
            double* out;
            if (i < C.nv) {
                s[0] = C.vid[i];
                count = 1;
                out = C.vbox + 6 * static_cast<size_t>(i);
            } else if (i < C.nv + C.ne) {
                const uint2 e = C.eid[i - C.nv];
                s[0] = e.x; s[1] = e.y;
                count = 2;
                out = C.ebox + 6 * static_cast<size_t>(i - C.nv);
                edge = true;
            } else {
                const uint3 t = C.tid[i - C.nv - C.ne];
                s[0] = t.x; s[1] = t.y; s[2] = t.z;
                count = 3;
                out = C.tbox + 6 * static_cast<size_t>(i - C.nv - C.ne);
                tri = true;
            }
            D3 prev[3], cur[3];
            bool finite = true;
            for (int k = 0; k < count; ++k) {
                prev[k] = world_of(c, c.pos_in[s[k]]);
                cur[k] = world_of(c, C.snapshot[s[k]]);
                finite = finite && contact::finite3(prev[k]) && contact::finite3(cur[k]);
            }
            if (!finite) contact_fail(c.status, kContactInput);
            const contact::Box b = contact::swept_box(prev, cur, count, C.separation);
            for (int k = 0; k < 3; ++k) {
                out[k] = b.lo[k];
                out[3 + k] = b.hi[k];
            }
            lo_key = order_key(b.lo[a]);
            ext_key = order_key(b.hi[a] - b.lo[a]);
            lo_key2 = order_key(b.lo[a2]);
            ext_key2 = order_key(b.hi[a2] - b.lo[a2]);
            if (!finite) tri = edge = false;
        }
        warp_atomic_range(C.range + 0, C.range + 1, C.range + 2, tri, lo_key, ext_key);
        warp_atomic_range(C.range + 3, C.range + 4, C.range + 5, tri, lo_key2, ext_key2);
        warp_atomic_range(C.range + 6, C.range + 7, C.range + 8, edge, lo_key, ext_key);
        warp_atomic_range(C.range + 9, C.range + 10, C.range + 11, edge, lo_key2, ext_key2);
    }
}

// Bucket counts of the columns by the grid cell of their box's low corner
// (every thread of the cluster).
__device__ __noinline__ void contact_bin_counts(const ContactCtx& c) {
    const ContactDev& C = *c.C;
    const uint32_t gt = c.grank * blockDim.x + threadIdx.x, stride = c.gctas * blockDim.x;
    const int a = C.axis, a2 = C.axis2;
    const Bins bt = make_bins(C.range, C.bins_cap), be = make_bins(C.range + 6, C.bins_cap);
    for (uint32_t t = gt; t < C.nt; t += stride) {
        const double* q = C.tbox + 6 * static_cast<size_t>(t);
        atomicAdd(&C.tbin[bt.of(q[a], q[a2])], 1u);
    }
    for (uint32_t e = gt; e < C.ne; e += stride) {
        const double* q = C.ebox + 6 * static_cast<size_t>(e);
        atomicAdd(&C.ebin[be.of(q[a], q[a2])], 1u);
    }
}

// Columns into their buckets (every thread of the cluster).
__device__ __noinline__ void contact_bin_scatter(const ContactCtx& c) {
    const ContactDev& C = *c.C;
    const uint32_t gt = c.grank * blockDim.x + threadIdx.x, stride = c.gctas * blockDim.x;
    const int a = C.axis, a2 = C.axis2;
    const Bins bt = make_bins(C.range, C.bins_cap), be = make_bins(C.range + 6, C.bins_cap);
    for (uint32_t t = gt; t < C.nt; t += stride) {
        const double* q = C.tbox + 6 * static_cast<size_t>(t);
        const uint32_t b = bt.of(q[a], q[a2]);
        C.tbin_items[C.tbin[b] + atomicAdd(&C.tbin_fill[b], 1u)] = t;
    }
    for (uint32_t e = gt; e < C.ne; e += stride) {
        const double* q = C.ebox + 6 * static_cast<size_t>(e);
        const uint32_t b = be.of(q[a], q[a2]);
        C.ebin_items[C.ebin[b] + atomicAdd(&C.ebin_fill[b], 1u)] = e;
    }
}

// Count (write == false) or write the candidate rows, one warp per row.  A
// row tests only the columns of the grid cells its box can reach on the two
// broadphase axes: every column whose box can overlap the row's.  The
// write pass collects the row's hits, then orders them by column (a rank
// sort of the row's segment), so the list is the exhaustive one in key
// order.
__device__ __noinline__ void contact_rows(const ContactCtx& c, bool write) {
    const ContactDev& C = *c.C;
    const uint32_t rows = C.nv + C.ne;
    const uint32_t warps = (c.gctas * blockDim.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    const int a = C.axis;
    const contact::Box* vb = reinterpret_cast<const contact::Box*>(C.vbox);
    const contact::Box* eb = reinterpret_cast<const contact::Box*>(C.ebox);
    const contact::Box* tb = reinterpret_cast<const contact::Box*>(C.tbox);
    const int a2 = C.axis2;
    const Bins bt = make_bins(C.range, C.bins_cap), be = make_bins(C.range + 6, C.bins_cap);
    for (uint32_t row = (c.grank * blockDim.x + threadIdx.x) >> 5; row < rows; row += warps) {
        const bool vertex_row = row < C.nv;
        const contact::Box b = vertex_row ? vb[row] : eb[row - C.nv];
        const Bins& g = vertex_row ? bt : be;
        const uint32_t* cell_start = vertex_row ? C.tbin : C.ebin;
        const uint32_t* items = vertex_row ? C.tbin_items : C.ebin_items;
        // the window's low ends, widened by a relative margin against the
        // rounding of the columns' extents (the overlap test decides)
        const double reach_a = b.lo[a] - g.a.widest - 1.0e-9 * (fabs(b.lo[a]) + g.a.widest);
        const double reach_b = b.lo[a2] - g.b.widest - 1.0e-9 * (fabs(b.lo[a2]) + g.b.widest);
        const uint32_t ia0 = g.a.of(reach_a), ia1 = g.a.of(b.hi[a]);
        const uint32_t ib0 = g.b.of(reach_b), ib1 = g.b.of(b.hi[a2]);
        uint32_t v = 0;
        uint2 e = make_uint2(0, 0);
        if (vertex_row) v = C.vid[row];
        else e = C.eid[row - C.nv];
        const uint32_t i = row - C.nv;
        const unsigned long long base = write ? C.offsets[row] : 0ull;
        uint32_t hits = 0;
        for (uint32_t ia = ia0; ia <= ia1; ++ia) {
            const uint32_t lo = cell_start[ia * g.b.count + ib0];
            const uint32_t hi = cell_start[ia * g.b.count + ib1 + 1];
            for (uint32_t k0 = lo; k0 < hi; k0 += 32) {
                const uint32_t k = k0 + lane;
                bool hit = false;
                uint32_t col = 0;
                if (k < hi) {
                    col = items[k];
                    if (vertex_row) {
                        const uint3 t = C.tid[col];
                        hit = t.x != v && t.y != v && t.z != v && contact::boxes_overlap(b, tb[col]);
                    } else {
                        const uint2 f = C.eid[col];
                        hit = col > i && e.x != f.x && e.x != f.y && e.y != f.x && e.y != f.y &&
                              contact::boxes_overlap(b, eb[col]);
                    }
                }
                const unsigned mask = __ballot_sync(0xffffffffu, hit);
                if (write && hit) C.cand_tmp[base + hits + __popc(mask & ((1u << lane) - 1u))] = col;
                hits += __popc(mask);
            }
        }
        if (!write) {
            if (lane == 0) C.counts[row] = hits;
            continue;
        }
        __syncwarp();
        // rank sort of the row's hits (columns are distinct)
        const unsigned long long code_hi = static_cast<unsigned long long>(row) << 32;
        for (uint32_t p = lane; p < hits; p += 32) {
            const uint32_t mine = C.cand_tmp[base + p];
            uint32_t rank = 0;
            for (uint32_t q = 0; q < hits; ++q) rank += C.cand_tmp[base + q] < mine ? 1u : 0u;
            C.cand[base + rank] = code_hi | mine;
        }
    }
}

// Exclusive scan of the row counts into offsets (rank 0's block).
static __device__ __noinline__ void contact_scan(const ContactCtx& c) {
    __shared__ unsigned long long warp_total[32];
    const ContactDev& C = *c.C;
    const uint32_t n = C.nv + C.ne, t = threadIdx.x, threads = blockDim.x;
    const uint32_t chunk = (n + threads - 1) / threads;
    const uint32_t lo = min(n, t * chunk), hi = min(n, lo + chunk);
    unsigned long long own = 0;
    for (uint32_t i = lo; i < hi; ++i) own += C.counts[i];
    unsigned long long incl = own;
    const uint32_t lane = t & 31, warp = t >> 5;
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= static_cast<uint32_t>(d)) incl += y;
    }
    if (lane == 31) warp_total[warp] = incl;
    __syncthreads();
    if (t == 0) {
        unsigned long long run = 0;
        for (uint32_t w = 0; w < (threads + 31) / 32; ++w) {
            const unsigned long long y = warp_total[w];
            warp_total[w] = run;
            run += y;
        }
    }
    __syncthreads();
    unsigned long long at = warp_total[warp] + incl - own;
    for (uint32_t i = lo; i < hi; ++i) {
        C.offsets[i] = at;
        at += C.counts[i];
    }
    if (t == threads - 1) {
        C.offsets[n] = at;
        if (at > C.cand_cap) contact_fail(c.status, kContactCandidates);
    }
}

// Cluster-window address of the node in `slot` (valid from every CTA).
__device__ __forceinline__ uint32_t slot_addr(const ContactCtx& c, uint32_t slot) {
    int r = c.ctas - 1;
    while (r > 0 && c.pbeg[r] > slot) --r;
    const uint32_t local = c.x_base + (slot - c.pbeg[r]) * 16u;
    uint32_t addr;
    asm("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(addr) : "r"(local), "r"(r));
    return addr;
}

// Per candidate: the swept query, the snapshot's closest features, and what
// the serial pass needs of the feature's nodes (slots, inverse masses,
// effective inverse mass; the structure's cluster turns the slots of the
// candidates in contact into cluster addresses).
__device__ __noinline__ void contact_queries(const ContactCtx& c) {
    const ContactDev& C = *c.C;
    const unsigned long long count = C.offsets[C.nv + C.ne];
    const uint32_t stride = c.gctas * blockDim.x;
    const uint32_t gt = c.grank * blockDim.x + threadIdx.x;
    contact::Interval* queue =
        reinterpret_cast<contact::Interval*>(C.queues) + static_cast<size_t>(gt) * C.queue_stride;
    for (unsigned long long i = gt; i < count; i += stride) {
        const FeatureSlots q = feature_slots(C, C.cand[i]);
        contact::Linear f, s;
        f.count = q.fc;
        s.count = q.sc;
        ContactQuery& out = C.query[i];
        double eff = 0.0;
        const contact::Closest g = [&] {
            for (int k = 0; k < q.fc; ++k) {
                f.prev[k] = world_of(c, c.pos_in[q.f[k]]);
                f.cur[k] = world_of(c, C.snapshot[q.f[k]]);
            }
            for (int k = 0; k < q.sc; ++k) {
                s.prev[k] = world_of(c, c.pos_in[q.s[k]]);
                s.cur[k] = world_of(c, C.snapshot[q.s[k]]);
            }
            return contact::evaluate_current(q.kind, f, s, C.separation);
        }();
        for (int k = 0; k < q.fc; ++k) {
            const float w = C.snapshot[q.f[k]].w;
            out.slot[k] = q.f[k];
            out.inv[k] = w;
            eff += static_cast<double>(w) * g.fw[k] * g.fw[k];
        }
        for (int k = 0; k < q.sc; ++k) {
            const float w = C.snapshot[q.s[k]].w;
            out.slot[q.fc + k] = q.s[k];
            out.inv[q.fc + k] = w;
            eff += static_cast<double>(w) * g.sw[k] * g.sw[k];
        }
        out.eff = eff;
        out.fc = static_cast<uint32_t>(q.fc);
        out.sc = static_cast<uint32_t>(q.sc);
        for (int k = 0; k < 3; ++k) {
            out.fw[k] = g.fw[k];
            out.sw[k] = g.sw[k];
        }
        out.normal[0] = g.normal.x; out.normal[1] = g.normal.y; out.normal[2] = g.normal.z;
        out.certified = g.certified() ? 1u : 0u;
        const contact::Ccd ccd = contact::swept_contact(q.kind, f, s, C.separation, C.ccd, queue);
        out.ccd_normal[0] = ccd.geometry.normal.x;
        out.ccd_normal[1] = ccd.geometry.normal.y;
        out.ccd_normal[2] = ccd.geometry.normal.z;
        out.ccd_state = ccd.state;
    }
}

// ---- key-ordered passes, in rounds of node-disjoint items ----------------------

__device__ __forceinline__ uint32_t cluster_tid(const ContactCtx& c) { return c.me * blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint32_t cluster_threads(const ContactCtx& c) {
    return static_cast<uint32_t>(c.ctas) * blockDim.x;
}

// Weighted point of a primitive's live nodes (weightedPoint,
// contact.cpp:1010-1019), streaming the nodes from distributed shared memory.
__device__ __forceinline__ D3 weighted_live(const ContactCtx& c, const uint32_t* addr, uint32_t n, const double* w) {
    D3 r{0.0, 0.0, 0.0};
    for (uint32_t k = 0; k < 3; ++k)
        if (k < n) r = r + w[k] * world_of(c, ld_node(addr[k]));
    return r;
}

__device__ __forceinline__ D3 d3_of(const double* v) { return {v[0], v[1], v[2]}; }

// First index in the sorted codes[0..n) whose code is not below `code`.
template <class Code>
__device__ __forceinline__ uint32_t lower_bound_code(Code code_at, uint32_t n, unsigned long long code) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (code_at(mid) < code) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Exclusive scan of in[0..n) into out[0..n] (in place allowed) by the
// calling block.
__device__ __noinline__ void block_scan(const uint32_t* in, uint32_t n, uint32_t* out) {
    __shared__ uint32_t warp_total[32];
    const uint32_t t = threadIdx.x, threads = blockDim.x;
    const uint32_t chunk = (n + threads - 1) / threads;
    const uint32_t lo = min(n, t * chunk), hi = min(n, lo + chunk);
    uint32_t own = 0;
    for (uint32_t i = lo; i < hi; ++i) own += in[i];
    uint32_t incl = own;
    const uint32_t lane = t & 31, warp = t >> 5;
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= static_cast<uint32_t>(d)) incl += y;
    }
    if (lane == 31) warp_total[warp] = incl;
    __syncthreads();
    if (t == 0) {
        uint32_t run = 0;
        for (uint32_t w = 0; w < (threads + 31) / 32; ++w) {
            const uint32_t y = warp_total[w];
            warp_total[w] = run;
            run += y;
        }
    }
    __syncthreads();
    uint32_t at = warp_total[warp] + incl - own;
    for (uint32_t i = lo; i < hi; ++i) {
        const uint32_t v = in[i];
        out[i] = at;
        at += v;
    }
    if (t == threads - 1) out[n] = at;
    __syncthreads();
}

// The order links of `items` taken in order (every thread of every CTA
// calls it): get(i, slots) returns item i's nodes (0: the item touches no
// node).  Item j must follow item i when i < j and they share a node; it is
// enough that each item follows the item just before it in each of its
// nodes' lists.  The (node, item) pairs are bucketed by node with a counting
// sort, each bucket is put in item order, and each item gets, per node, a
// link to the next item of the bucket (lv_succ, lv_nsucc) and the count of
// items it follows (lv_npred).  Items that follow none of the others can run
// first, together: they share no node.
template <class Get>
__device__ __noinline__ void cluster_order(const ContactCtx& c, cooperative_groups::cluster_group& cluster,
                                           uint32_t items, uint32_t slots, Get get) {
    const ContactDev& C = *c.C;
    const uint32_t gt = cluster_tid(c), stride = cluster_threads(c);
    uint32_t* count = C.lv_node_start;  // counts, then (scanned in place) bucket starts
    for (uint32_t i = gt; i <= slots; i += stride) count[i] = 0;
    for (uint32_t i = gt; i < slots; i += stride) C.lv_node_fill[i] = 0;
    for (uint32_t i = gt; i < items; i += stride) {
        C.lv_npred[i] = 0;
        C.lv_nsucc[i] = 0;
    }
    cluster.sync();
    uint32_t s6[6];
    for (uint32_t i = gt; i < items; i += stride) {
        const uint32_t n = get(i, s6);
        for (uint32_t q = 0; q < n; ++q) atomicAdd(&count[s6[q]], 1u);
    }
    cluster.sync();
    if (c.me == 0) block_scan(count, slots, count);
    cluster.sync();
    for (uint32_t i = gt; i < items; i += stride) {
        const uint32_t n = get(i, s6);
        for (uint32_t q = 0; q < n; ++q) C.lv_pairs[count[s6[q]] + atomicAdd(&C.lv_node_fill[s6[q]], 1u)] = i;
    }
    cluster.sync();
    for (uint32_t v = gt; v < slots; v += stride) {
        const uint32_t lo = count[v], hi = count[v + 1];
        for (uint32_t a = lo + 1; a < hi; ++a) {
            const uint32_t x = C.lv_pairs[a];
            uint32_t b = a;
            while (b > lo && C.lv_pairs[b - 1] > x) {
                C.lv_pairs[b] = C.lv_pairs[b - 1];
                --b;
            }
            C.lv_pairs[b] = x;
        }
        for (uint32_t a = lo + 1; a < hi; ++a) {
            const uint32_t i = C.lv_pairs[a - 1], j = C.lv_pairs[a];
            C.lv_succ[static_cast<size_t>(i) * 6 + atomicAdd(&C.lv_nsucc[i], 1u)] = j;
            atomicAdd(&C.lv_npred[j], 1u);
        }
    }
    cluster.sync();
}

// Runs work(id[item]) (work(item) without `id`) for `items` items in an
// order that keeps, for every node, the items touching it in item order
// (the calling block, after cluster_order): rounds, each running together
// the items whose earlier neighbours have all run (they share no node), a
// block barrier after each.  The nodes may live in any CTA of the cluster,
// but only this block's threads touch them until the cluster barrier that
// follows, so the block barrier orders one round's writes before the next
// round's reads.  Every item ends a round with all its links released, so a
// round runs at least one item and there are at most `items` rounds.
template <class Work>
__device__ __forceinline__ void run_order(const ContactDev& C, uint32_t items, const uint32_t* id, Work work) {
    __shared__ uint32_t front_n[2];
    uint32_t* front[2] = {C.lv_front, C.lv_front + C.cand_cap};
    if (threadIdx.x < 2) front_n[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < items; i += blockDim.x)
        if (__ldcg(C.lv_npred + i) == 0u) front[0][atomicAdd(&front_n[0], 1u)] = i;
    __syncthreads();
    uint32_t done = 0;
    for (uint32_t r = 0; r < items && done < items; ++r) {
        const uint32_t cur = r & 1u, n = front_n[cur];
        for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
            const uint32_t i = front[cur][k];
            work(id ? id[i] : i);
            const uint32_t m = C.lv_nsucc[i];
            for (uint32_t q = 0; q < m; ++q) {
                const uint32_t j = C.lv_succ[static_cast<size_t>(i) * 6 + q];
                if (atomicSub(&C.lv_npred[j], 1u) == 1u) front[cur ^ 1u][atomicAdd(&front_n[cur ^ 1u], 1u)] = j;
            }
        }
        done += n;
        __syncthreads();
        if (threadIdx.x == 0) front_n[cur] = 0;
        // read by every thread before the reset above takes effect two
        // rounds later: the next round's barrier separates them
    }
    __syncthreads();
}

__device__ __forceinline__ bool impact_state(uint32_t s) {
    return s == SWB_CCD_IMPACT || s == SWB_CCD_INITIALLY_PROXIMATE;
}

// The record book's flags after an iteration in which the entry was not
// visited: it stays a record only when it applied an impulse
// (contact.cpp:1462-1495).
__device__ __forceinline__ uint32_t carried_flags(uint32_t f) {
    return ((f & kEntryRecord) && (f & kEntryApplied)) ? (kEntryRecord | kEntryApplied) : 0u;
}

// One candidate's projection (contact.cpp:1318-1457): warm start from its
// entry of the previous table (copied into cand_entry beforehand), the XPBD
// normal projection on the live nodes, its entry for the next table.
static __device__ __noinline__ void project_one(const ContactCtx& c, uint32_t i) {
    const ContactDev& C = *c.C;
    const ContactQuery& Q = C.query[i];
    ContactEntry& out = C.cand_entry[i];
    ContactEntry e = out;  // the warm start
    if (!Q.certified) {
        contact_fail_at(C, c.status, kContactGeometry, C.cand[i]);
        return;
    }
    D3 normal = d3_of(Q.normal);
    if (contact::dot(normal, d3_of(Q.ccd_normal)) < 0.0) normal = -normal;
    if (!contact::finite3(normal) || fabs(contact::norm2(normal) - 1.0) > 1.0e-8) {
        contact_fail_at(C, c.status, kContactNormal, C.cand[i]);
        return;
    }
    const double dt = c.dt;
    const double alpha = C.compliance / (dt * dt);
    const double margin = contact::dmax(0.1 * C.separation, 8.0 * C.ccd.distance_tolerance);
    const uint32_t fc = Q.fc, sc = Q.sc;
    // the first primitive's nodes in A, the second's in B (constant indices)
    float4 A[3], B[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (k < static_cast<int>(fc)) A[k] = ld_node(Q.addr[k]);
        if (k < static_cast<int>(sc)) B[k] = ld_node(Q.addr[fc + k]);
    }
    auto point = [&](const float4* P, uint32_t count, const double* w) {
        D3 r{0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (k < static_cast<int>(count)) r = r + w[k] * world_of(c, P[k]);
        return r;
    };
    const double gap = contact::dot(point(A, fc, Q.fw) - point(B, sc, Q.sw), normal) - C.separation;
    const double eff = Q.eff;
    if ((gap > margin && e.lambda == 0.0) || !(eff + alpha > 0.0)) {
        if (!(eff + alpha > 0.0) && gap < 0.0 && !(gap > margin && e.lambda == 0.0)) {
            contact_fail_at(C, c.status, kContactNoResponse, C.cand[i]);
            return;
        }
        e.flags = carried_flags(e.flags);
        out = e;
        return;
    }
    const double delta = (-gap - alpha * e.lambda) / (eff + alpha);
    const double next = contact::dmax(0.0, e.lambda + delta);
    const double applied = next - e.lambda;
    if (!isfinite(next) || !isfinite(applied)) {
        contact_fail_at(C, c.status, kContactProjection, C.cand[i]);
        return;
    }
    // impulse w (applied / dt) n on the first primitive, the opposite on the
    // second; positions move by m^-1 dt impulse (contact.cpp:1404-1417)
    auto move = [&](float4& X, double w, float inv, uint32_t addr) {
        const D3 impulse = (w * (applied / dt)) * normal;
        const D3 p = world_of(c, X) + impulse * (static_cast<double>(inv) * dt);
        X.x = static_cast<float>(p.x - c.o[0]);
        X.y = static_cast<float>(p.y - c.o[1]);
        X.z = static_cast<float>(p.z - c.o[2]);
        st_node(addr, X);
    };
#pragma unroll
    for (int k = 0; k < 3; ++k)
        if (k < static_cast<int>(fc)) move(A[k], Q.fw[k], Q.inv[k], Q.addr[k]);
#pragma unroll
    for (int k = 0; k < 3; ++k)
        if (k < static_cast<int>(sc)) move(B[k], -Q.sw[k], Q.inv[fc + k], Q.addr[fc + k]);
    const D3 fp = point(A, fc, Q.fw), sp = point(B, sc, Q.sw);
    const double solved = contact::dot(fp - sp, normal) - C.separation;
    if (!contact::finite3(fp) || !contact::finite3(sp) || !isfinite(solved)) {
        contact_fail_at(C, c.status, kContactSolved, C.cand[i]);
        return;
    }
    // a record continuing from the previous iteration keeps its impulse
    // ledger; a new one starts it (contact.cpp:1391-1401); visited, it is a
    // record of this iteration
    const bool ledger = (e.flags & kEntryRecord) && (e.flags & kEntryApplied);
    e.lambda = next;
    e.flags = kEntryRecord | ((ledger || applied != 0.0) ? kEntryApplied : 0u);
    e.normal[0] = normal.x; e.normal[1] = normal.y; e.normal[2] = normal.z;
    out = e;
}

// The contact iteration's projections in key order (rounds of candidates
// that share no node), and the next multiplier table (the merge of this iteration's candidates in
// contact with the previous table's other entries).
__device__ __noinline__ void contact_project(const ContactCtx& c, cooperative_groups::cluster_group& cluster) {
    const ContactDev& C = *c.C;
    const bool skip = contact_failed(c.status);
    const uint32_t count = skip ? 0u : static_cast<uint32_t>(C.offsets[C.nv + C.ne]);
    const uint32_t sel = C.table_meta[0], old_n = C.table_meta[1];
    const ContactEntry* old = C.table[sel];
    ContactEntry* nw = C.table[sel ^ 1u];
    const uint32_t gt = cluster_tid(c), stride = cluster_threads(c);
    const uint32_t slots = c.pbeg[c.ctas];
    // reset
    for (uint32_t k = gt; k < old_n; k += stride) C.mark_b[k] = 1u;
    cluster.sync();
    // in contact or not; warm-start entry; previous entries taken over
    for (uint32_t i = gt; i < count; i += stride) {
        const uint32_t s = C.query[i].ccd_state;
        if (s == SWB_CCD_INDETERMINATE) contact_fail_at(C, c.status, kContactCcd, C.cand[i]);
        const bool hit = impact_state(s);
        C.mark_a[i] = hit ? 1u : 0u;
        if (hit) {
            const unsigned long long code = C.cand[i];
            const uint32_t k = lower_bound_code([&](uint32_t m) { return old[m].code; }, old_n, code);
            ContactEntry e;
            if (k < old_n && old[k].code == code) {
                e = old[k];
                C.mark_b[k] = 0u;
            } else {
                e.code = code;
                e.lambda = 0.0;
                e.normal[0] = e.normal[1] = e.normal[2] = 0.0;
                e.flags = 0;
                e.pad = 0;
            }
            C.cand_entry[i] = e;  // the warm start, replaced by the projection's result
        }
    }
    cluster.sync();
    // ranks of the two merged lists and the candidates in contact (rank 0's
    // block); their order links (the cluster); their projections, round by
    // round (rank 0's block)
    if (c.me == 0) {
        block_scan(C.mark_a, count, C.mark_a);
        block_scan(C.mark_b, old_n, C.mark_b);
        if (!contact_failed(c.status))
            for (uint32_t i = threadIdx.x; i < count; i += blockDim.x)
                if (C.mark_a[i + 1] != C.mark_a[i]) C.hit[C.mark_a[i]] = i;
    }
    cluster.sync();
    if (!contact_failed(c.status)) {  // uniform: read after the barrier
        const uint32_t hits = C.mark_a[count];
        // cluster addresses of the nodes of the candidates in contact (read
        // by rank 0's rounds after cluster_order's barriers)
        for (uint32_t h = gt; h < hits; h += stride) {
            ContactQuery& Q = C.query[C.hit[h]];
            for (uint32_t j = 0; j < Q.fc + Q.sc; ++j) Q.addr[j] = slot_addr(c, Q.slot[j]);
        }
        cluster_order(c, cluster, hits, slots, [&](uint32_t h, uint32_t* s) -> uint32_t {
            const ContactQuery& Q = C.query[C.hit[h]];
            const uint32_t n = Q.fc + Q.sc;
#pragma unroll
            for (int j = 0; j < 6; ++j) s[j] = j < static_cast<int>(n) ? Q.slot[j] : 0u;
            return n;
        });
        if (c.me == 0) run_order(C, hits, C.hit, [&](uint32_t i) { project_one(c, i); });
    }
    cluster.sync();
    if (contact_failed(c.status)) return;  // uniform: read after the barrier
    // the next table: sorted union of the candidates in contact and the
    // previous entries they did not take over (codes are disjoint)
    const uint32_t hits = C.mark_a[count], kept = C.mark_b[old_n];
    if (hits + kept > C.table_cap) {
        if (gt == 0) contact_fail(c.status, kContactTable);
        return;
    }
    for (uint32_t i = gt; i < count; i += stride) {
        if (C.mark_a[i + 1] == C.mark_a[i]) continue;
        const unsigned long long code = C.cand[i];
        const uint32_t k = lower_bound_code([&](uint32_t m) { return old[m].code; }, old_n, code);
        nw[C.mark_a[i] + C.mark_b[k]] = C.cand_entry[i];
    }
    for (uint32_t k = gt; k < old_n; k += stride) {
        if (C.mark_b[k + 1] == C.mark_b[k]) continue;
        ContactEntry e = old[k];
        e.flags = carried_flags(e.flags);
        const uint32_t i = lower_bound_code([&](uint32_t m) { return C.cand[m]; }, count, e.code);
        nw[C.mark_b[k] + C.mark_a[i]] = e;
    }
    cluster.sync();
    if (c.me == 0 && threadIdx.x == 0) {
        C.table_meta[0] = sel ^ 1u;
        C.table_meta[1] = hits + kept;
    }
}

// The certification of the final state (contact.cpp:1800-2078): the
// certified records of the candidates the swept query finds in contact and
// the retained records of earlier solver visits, in key order.
__device__ __noinline__ void contact_certify_all(const ContactCtx& c, cooperative_groups::cluster_group& cluster,
                                                 ContactDiagDev* diag) {
    const ContactDev& C = *c.C;
    const bool skip = contact_failed(c.status);
    const uint32_t count = skip ? 0u : static_cast<uint32_t>(C.offsets[C.nv + C.ne]);
    const uint32_t sel = C.table_meta[0], tn = C.table_meta[1];
    const ContactEntry* tab = C.table[sel];
    const uint32_t gt = cluster_tid(c), stride = cluster_threads(c);
    const double limit = contact::dmax(0.02 * C.separation, 1.0e-8);
    for (uint32_t i = gt; i < count; i += stride) {
        C.mark_a[i] = 0u;
        const ContactQuery& Q = C.query[i];
        const unsigned long long code = C.cand[i];
        if (Q.ccd_state == SWB_CCD_INDETERMINATE) {
            contact_fail_at(C, c.status, kContactFinalCcd, code);
            continue;
        }
        const uint32_t k = lower_bound_code([&](uint32_t m) { return tab[m].code; }, tn, code);
        const ContactEntry* e = (k < tn && tab[k].code == code) ? &tab[k] : nullptr;
        const bool impact = Q.ccd_state != SWB_CCD_NO_IMPACT;
        if (!impact && !(e && (e->flags & kEntryRecord))) continue;
        if (!Q.certified) {
            contact_fail_at(C, c.status, impact ? kContactFinalGeometry : kContactCleared, code);
            continue;
        }
        D3 normal = d3_of(Q.normal);
        if (contact::dot(normal, impact ? d3_of(Q.ccd_normal) : d3_of(e->normal)) < 0.0) normal = -normal;
        const uint32_t fc = Q.fc, sc = Q.sc;
        const D3 fp = weighted_live(c, Q.addr, fc, Q.fw), sp = weighted_live(c, Q.addr + fc, sc, Q.sw);
        const double gap = contact::dot(fp - sp, normal) - C.separation;
        if (impact && (!contact::finite3(fp) || !contact::finite3(sp) || !contact::finite3(normal) || !isfinite(gap))) {
            contact_fail_at(C, c.status, kContactFinalNonFinite, code);
            continue;
        }
        const double pen = contact::dmax(0.0, -gap);
        if ((!impact && !isfinite(gap)) || pen > limit) {
            contact_fail_at(C, c.status, impact ? kContactPenetration : kContactClearedGate, code);
            continue;
        }
        ContactRecordDev& r = C.cand_rec[i];
        r.code = code;
        for (int j = 0; j < 3; ++j) {
            r.fw[j] = Q.fw[j];
            r.sw[j] = Q.sw[j];
        }
        for (int j = 0; j < 6; ++j) {
            r.addr[j] = j < static_cast<int>(fc + sc) ? slot_addr(c, Q.slot[j]) : 0u;
            r.slot[j] = Q.slot[j];
            r.inv[j] = Q.inv[j];
        }
        r.fc = fc;
        r.sc = sc;
        r.eff = Q.eff;
        r.normal[0] = normal.x; r.normal[1] = normal.y; r.normal[2] = normal.z;
        r.lambda = e ? e->lambda : 0.0;
        r.active = impact && r.lambda > 0.0 ? 1u : 0u;
        r.pad = 0;
        C.mark_a[i] = 1u;
        if (r.active) atomicAdd(&C.reduce[0], 1ull);
        atomicMax(&C.reduce[1], static_cast<unsigned long long>(__double_as_longlong(pen)));  // pen >= 0
    }
    // every record of the solver must still be a supported feature
    for (uint32_t k = gt; k < tn; k += stride) {
        if (!(tab[k].flags & kEntryRecord)) continue;
        const uint32_t i = lower_bound_code([&](uint32_t m) { return C.cand[m]; }, count, tab[k].code);
        if (!(i < count && C.cand[i] == tab[k].code)) contact_fail_at(C, c.status, kContactLost, tab[k].code);
    }
    cluster.sync();
    if (c.me == 0) {
        block_scan(C.mark_a, count, C.mark_a);
        if (threadIdx.x == 0) {
            diag->candidates = count;
            diag->active = C.reduce[0];
            diag->records = C.mark_a[count];
            diag->max_penetration = __longlong_as_double(static_cast<long long>(C.reduce[1]));
        }
    }
    cluster.sync();
    for (uint32_t i = gt; i < count; i += stride)
        if (C.mark_a[i + 1] != C.mark_a[i]) C.records[C.mark_a[i]] = C.cand_rec[i];
}

// Coulomb friction of one certified record on the finalized velocities
// (contact.cpp:2081-2147).
static __device__ __noinline__ void friction_one(const ContactCtx& c, const ContactRecordDev& r) {
    const ContactDev& C = *c.C;
    const uint32_t fc = r.fc, sc = r.sc;
    float4 A[3], B[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (k < static_cast<int>(fc)) A[k] = ld_node(r.addr[k] + c.v_delta);
        if (k < static_cast<int>(sc)) B[k] = ld_node(r.addr[fc + k] + c.v_delta);
    }
    D3 vf{0.0, 0.0, 0.0}, vs{0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (k < static_cast<int>(fc)) vf = vf + r.fw[k] * D3{A[k].x, A[k].y, A[k].z};
        if (k < static_cast<int>(sc)) vs = vs + r.sw[k] * D3{B[k].x, B[k].y, B[k].z};
    }
    const contact::Friction fr = contact::coulomb_friction(vf - vs, d3_of(r.normal), r.eff, r.lambda / c.dt,
                                                           C.static_mu, C.dynamic_mu, r.active != 0);
    if (!contact::finite3(fr.impulse) || !isfinite(fr.work) ||
        fr.work > 1.0e-12 * contact::dmax(1.0, contact::norm2(fr.initial_tangent))) {
        contact_fail_at(C, c.status, kContactFriction, r.code);
        return;
    }
    if (fr.state == contact::kFrictionInactive) return;  // no impulse
    auto kick = [&](float4& V, double w, float inv, uint32_t addr) {
        const D3 dv = (w * fr.impulse) * static_cast<double>(inv);
        V.x = static_cast<float>(V.x + dv.x);
        V.y = static_cast<float>(V.y + dv.y);
        V.z = static_cast<float>(V.z + dv.z);
        st_node(addr + c.v_delta, V);
    };
#pragma unroll
    for (int k = 0; k < 3; ++k)
        if (k < static_cast<int>(fc)) kick(A[k], r.fw[k], r.inv[k], r.addr[k]);
#pragma unroll
    for (int k = 0; k < 3; ++k)
        if (k < static_cast<int>(sc)) kick(B[k], -r.sw[k], r.inv[fc + k], r.addr[fc + k]);
}

// ---- the three contact steps of a substep ------------------------------------

__device__ __forceinline__ uint32_t* C_bins_t(const ContactCtx& c) { return c.C->tbin; }
__device__ __forceinline__ uint32_t* C_bins_e(const ContactCtx& c) { return c.C->ebin; }

// Broadphase and queries of the current state (phases snapshot .. queries),
// over every CTA of the launch (the structure's cluster and its helpers).
__device__ __forceinline__ void contact_detect(const ContactCtx& c, cooperative_groups::cluster_group& cluster) {
    cluster.sync();  // every CTA's projections (local and remote) are done
    contact_snapshot(c);
    detect_sync(c, cluster);
    contact_boxes(c);
    detect_sync(c, cluster);
    if (!contact_failed(c.status)) contact_bin_counts(c);
    detect_sync(c, cluster);
    if (c.grank == 0 && !contact_failed(c.status)) {
        block_scan(C_bins_t(c), make_bins(c.C->range, c.C->bins_cap).count(), C_bins_t(c));
        block_scan(C_bins_e(c), make_bins(c.C->range + 6, c.C->bins_cap).count(), C_bins_e(c));
    }
    detect_sync(c, cluster);
    if (!contact_failed(c.status)) contact_bin_scatter(c);
    detect_sync(c, cluster);
    if (!contact_failed(c.status)) contact_rows(c, false);
    detect_sync(c, cluster);
    if (c.grank == 0 && !contact_failed(c.status)) contact_scan(c);
    detect_sync(c, cluster);
    if (!contact_failed(c.status)) contact_rows(c, true);
    detect_sync(c, cluster);
    if (!contact_failed(c.status)) contact_queries(c);
    detect_sync(c, cluster);
}

// A helper cluster's part of a launch: the detection phases of every
// contact iteration and of the certification, in the order the structure's
// cluster runs them.
__device__ __forceinline__ void contact_helper(const ContactCtx& c, cooperative_groups::cluster_group& cluster,
                                               int iterations) {
    for (int it = 0; it < iterations; ++it) contact_detect(c, cluster);
    contact_detect(c, cluster);
}

__device__ __forceinline__ void contact_iteration(const ContactCtx& c, cooperative_groups::cluster_group& cluster) {
    contact_detect(c, cluster);
    contact_project(c, cluster);
    cluster.sync();
}

__device__ __forceinline__ void contact_certify(const ContactCtx& c, cooperative_groups::cluster_group& cluster,
                                                ContactDiagDev* diag) {
    if (c.me == 0 && threadIdx.x == 0) {
        c.C->reduce[0] = 0ull;
        c.C->reduce[1] = 0ull;
    }
    contact_detect(c, cluster);
    contact_certify_all(c, cluster, diag);
    cluster.sync();
}

__device__ __forceinline__ void contact_friction(const ContactCtx& c, cooperative_groups::cluster_group& cluster,
                                                 const ContactDiagDev* diag) {
    const ContactDev& C = *c.C;
    cluster.sync();  // every CTA has finalized its velocities
    const bool skip = contact_failed(c.status);
    const uint32_t records = skip ? 0u : static_cast<uint32_t>(diag->records);
    cluster_order(c, cluster, records, c.pbeg[c.ctas], [&](uint32_t i, uint32_t* s) -> uint32_t {
        const ContactRecordDev& r = C.records[i];
        const uint32_t n = r.fc + r.sc;
#pragma unroll
        for (int j = 0; j < 6; ++j) s[j] = j < static_cast<int>(n) ? r.slot[j] : 0u;
        return n;
    });
    if (c.me == 0) run_order(C, records, nullptr, [&](uint32_t i) { friction_one(c, C.records[i]); });
    cluster.sync();
}

}  // namespace dev
}  // namespace swb
