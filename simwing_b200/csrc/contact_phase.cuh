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
};

__device__ __forceinline__ void contact_fail(int* status, int code) {
    if ((atomicOr(status, kStatusContact) & kStatusContact) == 0) status[1] = code;
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
};

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

// ---- parallel phases (every thread of the cluster; a barrier after each) ----

__device__ __forceinline__ void contact_snapshot(const ContactCtx& c) {
    for (uint32_t i = threadIdx.x; i < c.n; i += blockDim.x) c.C->snapshot[c.base + i] = c.x[i];
}

static __device__ __noinline__ void contact_boxes(const ContactCtx& c) {
    const ContactDev& C = *c.C;
    const uint32_t total = C.nv + C.ne + C.nt;
    const uint32_t stride = static_cast<uint32_t>(c.ctas) * blockDim.x;
    for (uint32_t i = c.me * blockDim.x + threadIdx.x; i < total; i += stride) {
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
        } else {
            const uint3 t = C.tid[i - C.nv - C.ne];
            s[0] = t.x; s[1] = t.y; s[2] = t.z;
            count = 3;
            out = C.tbox + 6 * static_cast<size_t>(i - C.nv - C.ne);
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
    }
}

// Count (write == false) or write the candidate rows, one warp per row.
static __device__ __noinline__ void contact_rows(const ContactCtx& c, bool write) {
    const ContactDev& C = *c.C;
    const uint32_t rows = C.nv + C.ne;
    const uint32_t warps = (static_cast<uint32_t>(c.ctas) * blockDim.x) >> 5;
    const contact::Box* vb = reinterpret_cast<const contact::Box*>(C.vbox);
    const contact::Box* eb = reinterpret_cast<const contact::Box*>(C.ebox);
    const contact::Box* tb = reinterpret_cast<const contact::Box*>(C.tbox);
    for (uint32_t row = (c.me * blockDim.x + threadIdx.x) >> 5; row < rows; row += warps) {
        const unsigned long long base = write ? C.offsets[row] : 0ull;
        const unsigned long long hi = static_cast<unsigned long long>(row) << 32;
        const uint32_t hits =
            contact::scan_candidate_row(row, C.nv, C.ne, C.nt, C.vid, C.eid, C.tid, vb, eb, tb,
                                        [&](uint32_t col, uint32_t k) {
                                            if (write) C.cand[base + k] = hi | col;
                                        });
        if (!write && (threadIdx.x & 31) == 0) C.counts[row] = hits;
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
// the serial pass needs of the feature's nodes (cluster addresses, inverse
// masses, effective inverse mass).
__device__ __noinline__ void contact_queries(const ContactCtx& c) {
    const ContactDev& C = *c.C;
    const unsigned long long count = C.offsets[C.nv + C.ne];
    const uint32_t stride = static_cast<uint32_t>(c.ctas) * blockDim.x;
    const uint32_t gt = c.me * blockDim.x + threadIdx.x;
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
            out.addr[k] = slot_addr(c, q.f[k]);
            out.inv[k] = w;
            eff += static_cast<double>(w) * g.fw[k] * g.fw[k];
        }
        for (int k = 0; k < q.sc; ++k) {
            const float w = C.snapshot[q.s[k]].w;
            out.addr[q.fc + k] = slot_addr(c, q.s[k]);
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

// ---- serial passes (rank 0, thread 0) ---------------------------------------

__device__ __forceinline__ void prefetch_l1(const void* p) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
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

__device__ __forceinline__ bool push_entry(const ContactDev& C, ContactEntry* out, uint32_t& m, const ContactEntry& e,
                                           int* status) {
    if (m >= C.table_cap) {
        contact_fail(status, kContactTable);
        return false;
    }
    out[m++] = e;
    return true;
}

constexpr int kContactPrefetch = 4;  // candidates fetched ahead by the serial passes

// One contact iteration's projections in key order (contact.cpp:1281-1457):
// warm-started multipliers merged into the other table buffer.
static __device__ __noinline__ void contact_project_serial(const ContactCtx& c) {
    const ContactDev& C = *c.C;
    if (contact_failed(c.status)) return;
    const unsigned long long count = C.offsets[C.nv + C.ne];
    const uint32_t sel = C.table_meta[0], old_n = C.table_meta[1];
    const ContactEntry* old = C.table[sel];
    ContactEntry* nw = C.table[sel ^ 1u];
    uint32_t k = 0, m = 0;
    const double dt = c.dt;
    const double alpha = C.compliance / (dt * dt);
    const double margin = contact::dmax(0.1 * C.separation, 8.0 * C.ccd.distance_tolerance);
    for (unsigned long long i = 0; i < count; ++i) {
        if (i + kContactPrefetch < count) {
            prefetch_l1(C.query + i + kContactPrefetch);
            prefetch_l1(reinterpret_cast<const char*>(C.query + i + kContactPrefetch) + 128);
            prefetch_l1(C.cand + i + kContactPrefetch);
        }
        const ContactQuery& Q = C.query[i];
        const uint32_t state = Q.ccd_state;
        if (state == SWB_CCD_INDETERMINATE) {
            contact_fail(c.status, kContactCcd);
            return;
        }
        if (state == SWB_CCD_NO_IMPACT) continue;
        const unsigned long long code = C.cand[i];
        while (k < old_n && old[k].code < code)
            if (!push_entry(C, nw, m, old[k++], c.status)) return;
        ContactEntry e;
        if (k < old_n && old[k].code == code) {
            e = old[k++];
        } else {
            e.code = code;
            e.lambda = 0.0;
            e.normal[0] = e.normal[1] = e.normal[2] = 0.0;
            e.flags = 0;
            e.pad = 0;
        }
        if (k < old_n) prefetch_l1(old + k);
        if (!Q.certified) {
            contact_fail(c.status, kContactGeometry);
            return;
        }
        D3 normal = d3_of(Q.normal);
        if (contact::dot(normal, d3_of(Q.ccd_normal)) < 0.0) normal = -normal;
        if (!contact::finite3(normal) || fabs(contact::norm2(normal) - 1.0) > 1.0e-8) {
            contact_fail(c.status, kContactNormal);
            return;
        }
        const uint32_t fc = Q.fc, sc = Q.sc, n = fc + sc;
        const double gap =
            contact::dot(weighted_live(c, Q.addr, fc, Q.fw) - weighted_live(c, Q.addr + fc, sc, Q.sw), normal) -
            C.separation;
        if (gap > margin && e.lambda == 0.0) {
            if (!push_entry(C, nw, m, e, c.status)) return;
            continue;
        }
        const double eff = Q.eff;
        if (!(eff + alpha > 0.0)) {
            if (gap < 0.0) {
                contact_fail(c.status, kContactNoResponse);
                return;
            }
            if (!push_entry(C, nw, m, e, c.status)) return;
            continue;
        }
        const double delta = (-gap - alpha * e.lambda) / (eff + alpha);
        const double next = contact::dmax(0.0, e.lambda + delta);
        const double applied = next - e.lambda;
        if (!isfinite(next) || !isfinite(applied)) {
            contact_fail(c.status, kContactProjection);
            return;
        }
        e.lambda = next;
        // impulse w (applied / dt) n on the first primitive, the opposite on
        // the second; positions move by m^-1 dt impulse (contact.cpp:1404-1417)
        for (uint32_t j = 0; j < n; ++j) {
            const double w = j < fc ? Q.fw[j] : -Q.sw[j - fc];
            const D3 impulse = (w * (applied / dt)) * normal;
            float4 X = ld_node(Q.addr[j]);
            const D3 p = world_of(c, X) + impulse * (static_cast<double>(Q.inv[j]) * dt);
            X.x = static_cast<float>(p.x - c.o[0]);
            X.y = static_cast<float>(p.y - c.o[1]);
            X.z = static_cast<float>(p.z - c.o[2]);
            st_node(Q.addr[j], X);
        }
        const D3 fp = weighted_live(c, Q.addr, fc, Q.fw), sp = weighted_live(c, Q.addr + fc, sc, Q.sw);
        const double solved = contact::dot(fp - sp, normal) - C.separation;
        if (!contact::finite3(fp) || !contact::finite3(sp) || !isfinite(solved)) {
            contact_fail(c.status, kContactSolved);
            return;
        }
        // a record continuing from the previous iteration keeps its impulse
        // ledger; a new one starts it (contact.cpp:1391-1401)
        const bool ledger = (e.flags & kEntryRecord) && (e.flags & kEntryApplied);
        e.flags = (e.flags & kEntryRecord) | kEntryVisited | ((ledger || applied != 0.0) ? kEntryApplied : 0u);
        e.normal[0] = normal.x; e.normal[1] = normal.y; e.normal[2] = normal.z;
        if (!push_entry(C, nw, m, e, c.status)) return;
    }
    while (k < old_n)
        if (!push_entry(C, nw, m, old[k++], c.status)) return;
    // the record book after the iteration: this iteration's visits plus the
    // earlier records that applied an impulse (contact.cpp:1462-1495)
    for (uint32_t j = 0; j < m; ++j) {
        uint32_t f = nw[j].flags;
        const bool record = (f & kEntryVisited) || ((f & kEntryRecord) && (f & kEntryApplied));
        f = record ? ((f & kEntryApplied) | kEntryRecord) : 0u;
        nw[j].flags = f;
    }
    C.table_meta[0] = sel ^ 1u;
    C.table_meta[1] = m;
}

// The certification of the final state (contact.cpp:1800-2078): certified
// records of the candidates the swept query finds in contact, retained
// records of earlier solver visits, in key order.
static __device__ __noinline__ void contact_certify_serial(const ContactCtx& c, ContactDiagDev* diag) {
    const ContactDev& C = *c.C;
    if (contact_failed(c.status)) return;
    const unsigned long long count = C.offsets[C.nv + C.ne];
    const uint32_t sel = C.table_meta[0], tn = C.table_meta[1];
    const ContactEntry* tab = C.table[sel];
    const double limit = contact::dmax(0.02 * C.separation, 1.0e-8);
    uint32_t k = 0;
    unsigned long long records = 0, active = 0;
    double max_pen = 0.0;
    for (unsigned long long i = 0; i < count; ++i) {
        if (i + kContactPrefetch < count) {
            prefetch_l1(C.query + i + kContactPrefetch);
            prefetch_l1(C.cand + i + kContactPrefetch);
        }
        const unsigned long long code = C.cand[i];
        while (k < tn && tab[k].code < code) {
            if (tab[k].flags & kEntryRecord) {
                contact_fail(c.status, kContactLost);
                return;
            }
            ++k;
        }
        const ContactEntry* e = (k < tn && tab[k].code == code) ? &tab[k] : nullptr;
        if (e) ++k;
        const ContactQuery& Q = C.query[i];
        if (Q.ccd_state == SWB_CCD_INDETERMINATE) {
            contact_fail(c.status, kContactFinalCcd);
            return;
        }
        const bool impact = Q.ccd_state != SWB_CCD_NO_IMPACT;
        if (!impact && !(e && (e->flags & kEntryRecord))) continue;
        if (!Q.certified) {
            contact_fail(c.status, impact ? kContactFinalGeometry : kContactCleared);
            return;
        }
        D3 normal = d3_of(Q.normal);
        if (contact::dot(normal, impact ? d3_of(Q.ccd_normal) : d3_of(e->normal)) < 0.0) normal = -normal;
        const uint32_t fc = Q.fc, sc = Q.sc;
        const D3 fp = weighted_live(c, Q.addr, fc, Q.fw), sp = weighted_live(c, Q.addr + fc, sc, Q.sw);
        const double gap = contact::dot(fp - sp, normal) - C.separation;
        if (impact && (!contact::finite3(fp) || !contact::finite3(sp) || !contact::finite3(normal) || !isfinite(gap))) {
            contact_fail(c.status, kContactFinalNonFinite);
            return;
        }
        const double pen = contact::dmax(0.0, -gap);
        if ((!impact && !isfinite(gap)) || pen > limit) {
            contact_fail(c.status, impact ? kContactPenetration : kContactClearedGate);
            return;
        }
        if (records >= C.record_cap) {
            contact_fail(c.status, kContactRecords);
            return;
        }
        ContactRecordDev& r = C.records[records++];
        r.code = code;
        for (int j = 0; j < 3; ++j) {
            r.fw[j] = Q.fw[j];
            r.sw[j] = Q.sw[j];
        }
        for (int j = 0; j < 6; ++j) {
            r.addr[j] = Q.addr[j];
            r.inv[j] = Q.inv[j];
        }
        r.fc = fc;
        r.sc = sc;
        r.eff = Q.eff;
        r.normal[0] = normal.x; r.normal[1] = normal.y; r.normal[2] = normal.z;
        r.lambda = e ? e->lambda : 0.0;
        r.active = impact && r.lambda > 0.0 ? 1u : 0u;
        r.pad = 0;
        active += r.active;
        max_pen = contact::dmax(max_pen, pen);
    }
    for (; k < tn; ++k)
        if (tab[k].flags & kEntryRecord) {
            contact_fail(c.status, kContactLost);
            return;
        }
    diag->candidates = count;
    diag->active = active;
    diag->records = records;
    diag->max_penetration = max_pen;
}

// Coulomb friction of the certified records on the finalized velocities,
// in key order (contact.cpp:2081-2147).
static __device__ __noinline__ void contact_friction_serial(const ContactCtx& c, const ContactDiagDev* diag) {
    const ContactDev& C = *c.C;
    if (contact_failed(c.status)) return;
    const double dt = c.dt;
    const unsigned long long records = diag->records;
    for (unsigned long long i = 0; i < records; ++i) {
        if (i + kContactPrefetch < records) {
            prefetch_l1(C.records + i + kContactPrefetch);
            prefetch_l1(reinterpret_cast<const char*>(C.records + i + kContactPrefetch) + 128);
        }
        const ContactRecordDev& r = C.records[i];
        const uint32_t fc = r.fc, sc = r.sc, n = fc + sc;
        float4 V[6];
        for (uint32_t j = 0; j < 6; ++j)
            if (j < n) V[j] = ld_node(r.addr[j] + c.v_delta);
        D3 vf{0.0, 0.0, 0.0}, vs{0.0, 0.0, 0.0};
        for (uint32_t j = 0; j < 3; ++j) {
            if (j < fc) vf = vf + r.fw[j] * D3{V[j].x, V[j].y, V[j].z};
            if (j < sc) vs = vs + r.sw[j] * D3{V[fc + j].x, V[fc + j].y, V[fc + j].z};
        }
        const contact::Friction fr = contact::coulomb_friction(vf - vs, d3_of(r.normal), r.eff, r.lambda / dt,
                                                               C.static_mu, C.dynamic_mu, r.active != 0);
        if (!contact::finite3(fr.impulse) || !isfinite(fr.work) ||
            fr.work > 1.0e-12 * contact::dmax(1.0, contact::norm2(fr.initial_tangent))) {
            contact_fail(c.status, kContactFriction);
            return;
        }
        if (fr.state == contact::kFrictionInactive) continue;  // no impulse
        for (uint32_t j = 0; j < 6; ++j) {
            if (j >= n) break;
            const double w = j < fc ? r.fw[j] : -r.sw[j - fc];
            const D3 dv = (w * fr.impulse) * static_cast<double>(r.inv[j]);
            float4 W = V[j];
            W.x = static_cast<float>(W.x + dv.x);
            W.y = static_cast<float>(W.y + dv.y);
            W.z = static_cast<float>(W.z + dv.z);
            st_node(r.addr[j] + c.v_delta, W);
        }
    }
}

// ---- the three contact steps of a substep ------------------------------------

// Broadphase and queries of the current state (phases snapshot .. queries).
__device__ __forceinline__ void contact_detect(const ContactCtx& c, cooperative_groups::cluster_group& cluster) {
    cluster.sync();  // every CTA's projections (local and remote) are done
    contact_snapshot(c);
    cluster.sync();
    contact_boxes(c);
    cluster.sync();
    if (!contact_failed(c.status)) contact_rows(c, false);
    cluster.sync();
    if (c.me == 0 && !contact_failed(c.status)) contact_scan(c);
    cluster.sync();
    if (!contact_failed(c.status)) contact_rows(c, true);
    cluster.sync();
    if (!contact_failed(c.status)) contact_queries(c);
    cluster.sync();
}

__device__ __forceinline__ void contact_iteration(const ContactCtx& c, cooperative_groups::cluster_group& cluster) {
    contact_detect(c, cluster);
    if (c.me == 0 && threadIdx.x == 0) contact_project_serial(c);
    cluster.sync();
}

__device__ __forceinline__ void contact_certify(const ContactCtx& c, cooperative_groups::cluster_group& cluster,
                                                ContactDiagDev* diag) {
    contact_detect(c, cluster);
    if (c.me == 0 && threadIdx.x == 0) contact_certify_serial(c, diag);
    cluster.sync();
}

__device__ __forceinline__ void contact_friction(const ContactCtx& c, cooperative_groups::cluster_group& cluster,
                                                 const ContactDiagDev* diag) {
    cluster.sync();  // every CTA has finalized its velocities
    if (c.me == 0 && threadIdx.x == 0) contact_friction_serial(c, diag);
    cluster.sync();
}

}  // namespace dev
}  // namespace swb
