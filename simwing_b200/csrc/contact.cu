// Contact building blocks on the device (FP64): the candidate features of a
// fabric self-contact pair (exhaustive swept-AABB overlap in key order),
// closest features and the swept contact query.  This translation unit is
// compiled without FMA contraction, so its FP64 results equal softwing's
// (src/softwing/contact.cpp, built with FP contraction off) bit for bit.
#include "common.h"
#include "contact_geometry.cuh"
#include "contact_surface.h"
#include "structure_impl.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace swb {
namespace {

using contact::Box;
using contact::D3;

// Owned device allocation of `count` elements of T.
template <class T>
struct DeviceArray {
    T* ptr = nullptr;
    size_t count = 0;
    explicit DeviceArray(size_t n) : count(n) {
        if (n) cuda_check(cudaMalloc(&ptr, n * sizeof(T)), "cudaMalloc (contact)");
    }
    DeviceArray(const T* host, size_t n) : DeviceArray(n) {
        if (n) cuda_check(cudaMemcpy(ptr, host, n * sizeof(T), cudaMemcpyHostToDevice), "contact upload");
    }
    ~DeviceArray() {
        if (ptr) cudaFree(ptr);
    }
    DeviceArray(const DeviceArray&) = delete;
    DeviceArray& operator=(const DeviceArray&) = delete;
    void download(T* host, size_t n) const {
        if (n) cuda_check(cudaMemcpy(host, ptr, n * sizeof(T), cudaMemcpyDeviceToHost), "contact download");
    }
};

__device__ __forceinline__ D3 load3(const double* p) { return {p[0], p[1], p[2]}; }

// Swept boxes of every proxy: surface vertices, then edges, then triangles.
__global__ void proxy_boxes_kernel(const double* __restrict__ prev, const double* __restrict__ cur,
                                   const uint32_t* __restrict__ vertices, uint32_t nv,
                                   const uint2* __restrict__ edges, uint32_t ne,
                                   const uint3* __restrict__ triangles, uint32_t nt, double expansion,
                                   Box* __restrict__ vbox, Box* __restrict__ ebox, Box* __restrict__ tbox) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t nodes[3];
    int count;
    Box* out;
    if (i < nv) {
        nodes[0] = vertices[i];
        count = 1;
        out = vbox + i;
    } else if (i < nv + ne) {
        const uint2 e = edges[i - nv];
        nodes[0] = e.x; nodes[1] = e.y;
        count = 2;
        out = ebox + (i - nv);
    } else if (i < nv + ne + nt) {
        const uint3 t = triangles[i - nv - ne];
        nodes[0] = t.x; nodes[1] = t.y; nodes[2] = t.z;
        count = 3;
        out = tbox + (i - nv - ne);
    } else {
        return;
    }
    D3 p[3], c[3];
    for (int k = 0; k < count; ++k) {
        p[k] = load3(prev + 3 * static_cast<size_t>(nodes[k]));
        c[k] = load3(cur + 3 * static_cast<size_t>(nodes[k]));
    }
    *out = contact::swept_box(p, c, count, expansion);
}

// One warp per candidate row (contact::scan_candidate_row); with `cols` ==
// nullptr the warp counts its row's hits, else it writes their column
// indices from offsets[row] on, in column order.
__global__ void candidate_rows_kernel(uint32_t nv, uint32_t ne, uint32_t nt, const uint32_t* __restrict__ vertices,
                                      const uint2* __restrict__ edges, const uint3* __restrict__ triangles,
                                      const Box* __restrict__ vbox, const Box* __restrict__ ebox,
                                      const Box* __restrict__ tbox, uint32_t* __restrict__ counts,
                                      const unsigned long long* __restrict__ offsets, uint32_t* __restrict__ cols) {
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t rows = nv + ne;
    for (uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < rows; row += warps) {
        const unsigned long long base = cols ? offsets[row] : 0;
        const uint32_t hits = contact::scan_candidate_row(row, nv, ne, nt, vertices, edges, triangles, vbox, ebox, tbox,
                                                          [&](uint32_t col, uint32_t k) {
                                                              if (cols) cols[base + k] = col;
                                                          });
        if (!cols && (threadIdx.x & 31) == 0) counts[row] = hits;
    }
}

// Exclusive prefix sum of `n` counts into offsets[0..n] (one block).
__global__ void exclusive_scan_kernel(const uint32_t* __restrict__ counts, uint32_t n,
                                      unsigned long long* __restrict__ offsets) {
    __shared__ unsigned long long partial[1024];
    const uint32_t t = threadIdx.x, threads = blockDim.x;
    const uint32_t chunk = (n + threads - 1) / threads;
    const uint32_t begin = min(n, t * chunk), end = min(n, begin + chunk);
    unsigned long long sum = 0;
    for (uint32_t i = begin; i < end; ++i) sum += counts[i];
    partial[t] = sum;
    __syncthreads();
    if (t == 0) {
        unsigned long long run = 0;
        for (uint32_t k = 0; k < threads; ++k) {
            const unsigned long long v = partial[k];
            partial[k] = run;
            run += v;
        }
        offsets[n] = run;
    }
    __syncthreads();
    unsigned long long run = partial[t];
    for (uint32_t i = begin; i < end; ++i) {
        offsets[i] = run;
        run += counts[i];
    }
}

__device__ __forceinline__ void load_side(contact::Linear& l, const double* prev, const double* cur, size_t feature,
                                          int count) {
    l.count = count;
    for (int k = 0; k < count; ++k) {
        l.prev[k] = load3(prev + 9 * feature + 3 * k);
        l.cur[k] = load3(cur + 9 * feature + 3 * k);
    }
}

__device__ __forceinline__ void store3(double* out, D3 v) {
    out[0] = v.x; out[1] = v.y; out[2] = v.z;
}

__device__ __forceinline__ void store_closest(swb_closest_result& o, const contact::Closest& r) {
    o.status = r.status;
    o.first_feature = r.first_feature;
    o.second_feature = r.second_feature;
    o.reserved = 0;
    store3(o.first_point, r.first_point);
    store3(o.second_point, r.second_point);
    for (int k = 0; k < 3; ++k) {
        o.first_weights[k] = r.fw[k];
        o.second_weights[k] = r.sw[k];
    }
    store3(o.normal, r.normal);
    o.distance = r.distance;
    o.gap = r.gap;
}

__global__ void closest_kernel(uint32_t kind, size_t count, const double* __restrict__ first,
                               const double* __restrict__ second, double separation,
                               swb_closest_result* __restrict__ out) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= count) return;
    const double* f = first + 9 * i;
    const double* s = second + 9 * i;
    const contact::Closest r =
        kind == SWB_FEATURE_VERTEX_TRIANGLE
            ? contact::closest_vertex_triangle(load3(f), load3(s), load3(s + 3), load3(s + 6), separation)
            : contact::closest_edge_edge(load3(f), load3(f + 3), load3(s), load3(s + 3), separation);
    store_closest(out[i], r);
}

__global__ void sweep_kernel(uint32_t kind, size_t count, const double* __restrict__ fp,
                             const double* __restrict__ fc, const double* __restrict__ sp,
                             const double* __restrict__ sc, double separation, swb_ccd_settings cs,
                             contact::Interval* __restrict__ queues, size_t queue_stride,
                             swb_ccd_result* __restrict__ out) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= count) return;
    contact::Linear f, s;
    const bool vt = kind == SWB_FEATURE_VERTEX_TRIANGLE;
    load_side(f, fp, fc, i, vt ? 1 : 2);
    load_side(s, sp, sc, i, vt ? 3 : 2);
    const contact::Ccd r =
        contact::swept_contact(kind, f, s, separation, cs, queues + i * queue_stride);
    swb_ccd_result& o = out[i];
    o.state = r.state;
    o.conservative_iterations = r.iterations;
    o.interval_subdivisions = r.subdivisions;
    o.used_interval_fallback = r.fallback ? 1u : 0u;
    o.time_of_impact = r.toi;
    o.bracket_lower = r.lower;
    o.bracket_upper = r.upper;
    store_closest(o.geometry, r.geometry);
}

void require_device() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
        raise(SWB_CUDA_ERROR, "no CUDA device: the contact kernels need a GPU");
}

void check_kind(uint32_t kind) {
    if (kind == SWB_FEATURE_SEGMENT_TRIANGLE)
        raise(SWB_UNSUPPORTED, "segment-triangle contact (suspension lines) is not available in this build");
    if (kind != SWB_FEATURE_VERTEX_TRIANGLE && kind != SWB_FEATURE_EDGE_EDGE)
        raise(SWB_INVALID_ARGUMENT, "unknown contact feature kind");
}

}  // namespace

// Candidate features of one self pair on the device; `cols` of row r hold
// the matches in column order (see candidate_rows_kernel).
CandidateRows contact_candidate_rows(const ContactSurface& surface, const double* prev, const double* cur,
                                     uint64_t node_count, double separation) {
    require_device();
    const uint32_t nv = static_cast<uint32_t>(surface.vertices.size());
    const uint32_t ne = static_cast<uint32_t>(surface.edges.size());
    const uint32_t nt = static_cast<uint32_t>(surface.triangles.size());
    CandidateRows rows;
    rows.offsets.assign(static_cast<size_t>(nv) + ne + 1, 0);
    if (nv + ne == 0) return rows;
    DeviceArray<double> d_prev(prev, node_count * 3), d_cur(cur, node_count * 3);
    DeviceArray<uint32_t> d_vertices(surface.vertices.data(), nv);
    DeviceArray<uint2> d_edges(reinterpret_cast<const uint2*>(surface.edges.data()), ne);
    DeviceArray<uint3> d_tri(reinterpret_cast<const uint3*>(surface.triangles.data()), nt);
    DeviceArray<Box> vbox(nv), ebox(ne), tbox(nt);
    const uint32_t proxies = nv + ne + nt;
    proxy_boxes_kernel<<<(proxies + 255) / 256, 256>>>(d_prev.ptr, d_cur.ptr, d_vertices.ptr, nv, d_edges.ptr, ne,
                                                       d_tri.ptr, nt, separation, vbox.ptr, ebox.ptr, tbox.ptr);
    cuda_check(cudaGetLastError(), "proxy_boxes_kernel");
    const uint32_t row_count = nv + ne;
    DeviceArray<uint32_t> counts(row_count);
    DeviceArray<unsigned long long> offsets(static_cast<size_t>(row_count) + 1);
    const int threads = 256;
    const uint32_t blocks = std::min<uint32_t>((row_count + threads / 32 - 1) / (threads / 32), 148u * 8u);
    candidate_rows_kernel<<<blocks, threads>>>(nv, ne, nt, d_vertices.ptr, d_edges.ptr, d_tri.ptr, vbox.ptr,
                                               ebox.ptr, tbox.ptr, counts.ptr, nullptr, nullptr);
    cuda_check(cudaGetLastError(), "candidate_rows_kernel (count)");
    exclusive_scan_kernel<<<1, 1024>>>(counts.ptr, row_count, offsets.ptr);
    cuda_check(cudaGetLastError(), "exclusive_scan_kernel");
    std::vector<unsigned long long> host_offsets(static_cast<size_t>(row_count) + 1);
    offsets.download(host_offsets.data(), host_offsets.size());
    const uint64_t total = host_offsets.back();
    DeviceArray<uint32_t> cols(total);
    if (total) {
        candidate_rows_kernel<<<blocks, threads>>>(nv, ne, nt, d_vertices.ptr, d_edges.ptr, d_tri.ptr, vbox.ptr,
                                                   ebox.ptr, tbox.ptr, nullptr, offsets.ptr, cols.ptr);
        cuda_check(cudaGetLastError(), "candidate_rows_kernel (write)");
    }
    rows.cols.resize(total);
    cols.download(rows.cols.data(), total);
    std::copy(host_offsets.begin(), host_offsets.end(), rows.offsets.begin());
    return rows;
}

}  // namespace swb

using namespace swb;

void swb_default_ccd_settings(swb_ccd_settings* out) {
    if (!out) return;
    out->conservative_iterations = 32;
    out->interval_subdivisions = 256;
    out->time_tolerance = 1.0e-8;
    out->distance_tolerance = 1.0e-10;
}

swb_status swb_contact_candidates(const swb_structure_definition* definition, double half_thickness,
                                  const double* previous, const double* current, swb_contact_key* keys,
                                  uint64_t capacity, uint64_t* candidate_count, uint64_t* possible_count,
                                  uint64_t* excluded_count) {
    return guarded([&] {
        if (!definition || !previous || !current || !candidate_count || (capacity && !keys))
            raise(SWB_INVALID_ARGUMENT, "null argument");
        const ContactSurface surface = build_contact_surface(*definition, half_thickness);
        for (uint64_t i = 0; i < 3 * definition->node_count; ++i)
            if (!std::isfinite(previous[i]) || !std::isfinite(current[i]))
                raise(SWB_CONTACT_ERROR, "Contact broadphase input failed: Swept AABB positions must be finite");
        const CandidateRows rows =
            contact_candidate_rows(surface, previous, current, definition->node_count, 2.0 * half_thickness);
        const uint64_t total = rows.cols.size();
        *candidate_count = total;
        if (possible_count) *possible_count = surface.possible;
        if (excluded_count) *excluded_count = surface.excluded;
        if (total > capacity) raise(SWB_OUT_OF_RANGE, "candidate capacity too small");
        const size_t nv = surface.vertices.size();
        uint64_t k = 0;
        for (size_t row = 0; row + 1 < rows.offsets.size(); ++row) {
            for (uint64_t c = rows.offsets[row]; c < rows.offsets[row + 1]; ++c, ++k) {
                swb_contact_key& key = keys[k];
                std::memset(&key, 0, sizeof key);
                if (row < nv) {
                    key.kind = SWB_FEATURE_VERTEX_TRIANGLE;
                    key.first[0] = surface.vertices[row];
                    key.second[0] = rows.cols[c];
                } else {
                    const auto& e = surface.edges[row - nv];
                    const auto& f = surface.edges[rows.cols[c]];
                    key.kind = SWB_FEATURE_EDGE_EDGE;
                    key.first[0] = e[0];
                    key.first[1] = e[1];
                    key.second[0] = f[0];
                    key.second[1] = f[1];
                }
            }
        }
    });
}

swb_status swb_contact_closest(uint32_t kind, uint64_t count, const double* first, const double* second,
                               double separation, swb_closest_result* results) {
    return guarded([&] {
        check_kind(kind);
        if (count && (!first || !second || !results)) raise(SWB_INVALID_ARGUMENT, "null argument");
        if (!count) return;
        require_device();
        DeviceArray<double> f(first, 9 * count), s(second, 9 * count);
        DeviceArray<swb_closest_result> out(count);
        closest_kernel<<<static_cast<unsigned>((count + 127) / 128), 128>>>(kind, count, f.ptr, s.ptr, separation,
                                                                            out.ptr);
        cuda_check(cudaGetLastError(), "closest_kernel");
        out.download(results, count);
    });
}

swb_status swb_contact_sweep(uint32_t kind, uint64_t count, const double* first_previous,
                             const double* first_current, const double* second_previous,
                             const double* second_current, double separation, const swb_ccd_settings* settings,
                             swb_ccd_result* results) {
    return guarded([&] {
        check_kind(kind);
        if (!settings) raise(SWB_INVALID_ARGUMENT, "null settings");
        if (count && (!first_previous || !first_current || !second_previous || !second_current || !results))
            raise(SWB_INVALID_ARGUMENT, "null argument");
        if (settings->interval_subdivisions > SWB_CCD_MAX_SUBDIVISIONS)
            raise(SWB_INVALID_ARGUMENT, "interval_subdivisions above SWB_CCD_MAX_SUBDIVISIONS");
        if (!count) return;
        require_device();
        const swb_ccd_settings cs = *settings;
        // Invalid settings are the query's to report (state Indeterminate,
        // before any scratch is touched); the scratch is sized from a
        // non-negative budget.
        const size_t per_query = static_cast<size_t>(std::max(cs.interval_subdivisions, 0)) + 1;
        const size_t batch = std::max<size_t>(1, std::min<size_t>(count, (size_t(1) << 28) / (per_query * sizeof(contact::Interval))));
        DeviceArray<contact::Interval> queues(batch * per_query);
        for (uint64_t begin = 0; begin < count; begin += batch) {
            const size_t n = std::min<size_t>(batch, count - begin);
            DeviceArray<double> fp(first_previous + 9 * begin, 9 * n), fc(first_current + 9 * begin, 9 * n);
            DeviceArray<double> sp(second_previous + 9 * begin, 9 * n), sc(second_current + 9 * begin, 9 * n);
            DeviceArray<swb_ccd_result> out(n);
            sweep_kernel<<<static_cast<unsigned>((n + 63) / 64), 64>>>(kind, n, fp.ptr, fc.ptr, sp.ptr, sc.ptr,
                                                                        separation, cs, queues.ptr, per_query,
                                                                        out.ptr);
            cuda_check(cudaGetLastError(), "sweep_kernel");
            out.download(results + begin, n);
        }
    });
}
