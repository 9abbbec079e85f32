// Closed cell (bay) volumes on the device in FP64: softwing's
// estimateClosedCellVolume (src/softwing/cell_volume.cpp:161-306) for many
// cells at once.  The topology of a cell (which skin edges are used once or
// more than twice, which rib-loop edges close the skin, the orientation
// votes of the two caps) does not depend on the positions and is computed
// once on the host; one device thread per cell then runs the geometric part
// in the reference's order of operations (origin, orientation score, the
// geometric cap-orientation fallback, the tetrahedron sums).  This
// translation unit is compiled without FMA contraction, so its results equal
// the reference build's bit for bit.
#include "common.h"
#include "contact_geometry.cuh"
#include "structure_impl.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <set>
#include <vector>

namespace swb {
namespace {

using contact::D3;

constexpr double kEpsilon = 2.220446049250313e-16;  // DBL_EPSILON

// Position-independent facts of one cell.
struct CellTopology {
    uint32_t face_begin, face_count, low_begin, low_count, high_begin, high_count;
    uint32_t fail_at;       // first face position whose index, uniqueness or nodes fail (face_count: none)
    uint32_t loops_ok;      // both loops have >= 3 distinct, known nodes
    uint32_t boundary, non_manifold, cap_matched, watertight;
    int32_t low_forward, low_reverse, high_forward, high_reverse;  // cap-orientation votes
};

__device__ __forceinline__ D3 pos(const double* p, uint32_t n) { return {p[3 * n], p[3 * n + 1], p[3 * n + 2]}; }

__device__ __forceinline__ double tetra(D3 a, D3 b, D3 c, D3 o) {
    return contact::dot(a - o, contact::cross(b - o, c - o)) / 6.0;
}

__device__ D3 centroid(const double* p, const uint32_t* loop, uint32_t n) {
    D3 r{0.0, 0.0, 0.0};
    for (uint32_t i = 0; i < n; ++i) r = r + pos(p, loop[i]);
    return r / static_cast<double>(n);
}

// capOrientation's geometric fallback (cell_volume.cpp:116-126): the cap's
// area vector against the desired outward normal.
__device__ void cap_fallback(const double* p, const uint32_t* loop, uint32_t n, D3 desired, bool& forward,
                             bool& valid) {
    const D3 center = centroid(p, loop, n);
    D3 area{0.0, 0.0, 0.0};
    for (uint32_t i = 0; i < n; ++i)
        area = area + contact::cross(pos(p, loop[i]) - center, pos(p, loop[(i + 1) % n]) - center);
    area = area * 0.5;
    const double alignment = contact::dot(area, desired);
    const double scale = contact::norm(area) * contact::norm(desired);
    if (!isfinite(alignment) || !isfinite(scale) || scale <= kEpsilon || fabs(alignment) <= scale * 1.0e-10) {
        forward = true;
        valid = false;
        return;
    }
    forward = alignment > 0.0;
    valid = true;
}

__device__ double cap_volume(const double* p, const uint32_t* loop, uint32_t n, bool forward, D3 origin) {
    const D3 center = centroid(p, loop, n);
    double r = 0.0;
    for (uint32_t i = 0; i < n; ++i) {
        const D3 a = pos(p, loop[i]), b = pos(p, loop[(i + 1) % n]);
        r += forward ? tetra(center, a, b, origin) : tetra(center, b, a, origin);
    }
    return r;
}

__global__ void cell_volume_kernel(uint32_t cells, const CellTopology* __restrict__ topo,
                                   const uint3* __restrict__ tri, const uint32_t* __restrict__ faces,
                                   const uint32_t* __restrict__ loops, const double* __restrict__ p,
                                   swb_cell_volume* __restrict__ out) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= cells) return;
    const CellTopology t = topo[k];
    swb_cell_volume r{};
    const uint32_t* low = loops + t.low_begin;
    const uint32_t* high = loops + t.high_begin;
    bool loops_finite = true;
    for (uint32_t i = 0; i < t.low_count; ++i) loops_finite = loops_finite && contact::finite3(pos(p, low[i]));
    for (uint32_t i = 0; i < t.high_count; ++i) loops_finite = loops_finite && contact::finite3(pos(p, high[i]));
    if (t.face_count == 0 || !t.loops_ok || !loops_finite) {
        out[k] = r;
        return;
    }
    const uint32_t* f = faces + t.face_begin;
    D3 origin{0.0, 0.0, 0.0};
    uint64_t samples = 0;
    for (uint32_t i = 0; i < t.face_count; ++i) {
        if (i == t.fail_at) {
            out[k] = r;
            return;
        }
        const uint3 q = tri[f[i]];
        const D3 a = pos(p, q.x), b = pos(p, q.y), c = pos(p, q.z);
        if (!contact::finite3(a) || !contact::finite3(b) || !contact::finite3(c)) {
            out[k] = r;
            return;
        }
        origin = origin + ((a + b) + c);
        samples += 3;
        if (contact::norm2(contact::cross(b - a, c - a)) <= kEpsilon) ++r.degenerate_skin_faces;
    }
    for (uint32_t i = 0; i < t.low_count; ++i) origin = origin + pos(p, low[i]);
    for (uint32_t i = 0; i < t.high_count; ++i) origin = origin + pos(p, high[i]);
    samples += t.low_count + t.high_count;
    origin = origin / static_cast<double>(samples);
    r.skin_boundary_edges = t.boundary;
    r.non_manifold_skin_edges = t.non_manifold;
    r.cap_boundary_edges_matched = t.cap_matched;
    r.watertight_after_capping = t.watertight;
    const D3 span = centroid(p, high, t.high_count) - centroid(p, low, t.low_count);
    if (!contact::finite3(span) || contact::norm2(span) <= kEpsilon) {
        out[k] = r;
        return;
    }
    double score = 0.0, scale = 0.0;
    for (uint32_t i = 0; i < t.face_count; ++i) {
        const uint3 q = tri[f[i]];
        const D3 a = pos(p, q.x), b = pos(p, q.y), c = pos(p, q.z);
        const D3 area = contact::cross(b - a, c - a);
        const D3 center = ((a + b) + c) / 3.0;
        score += contact::dot(area, center - origin);
        scale += contact::norm(area) * contact::norm(center - origin);
    }
    const bool ambiguous = scale <= kEpsilon || fabs(score) <= scale * 1.0e-10;
    r.ambiguous_skin_orientation = ambiguous ? 1u : 0u;
    const double sign = score < 0.0 ? -1.0 : 1.0;
    bool low_forward, low_valid = true, low_fallback = false;
    bool high_forward, high_valid = true, high_fallback = false;
    if (t.low_forward != t.low_reverse) {
        low_forward = t.low_forward > t.low_reverse;
    } else {
        low_fallback = true;
        cap_fallback(p, low, t.low_count, span * -sign, low_forward, low_valid);
    }
    if (t.high_forward != t.high_reverse) {
        high_forward = t.high_forward > t.high_reverse;
    } else {
        high_fallback = true;
        cap_fallback(p, high, t.high_count, span * sign, high_forward, high_valid);
    }
    r.used_geometric_orientation_fallback = (low_fallback || high_fallback) ? 1u : 0u;
    if (!low_valid || !high_valid || ((low_fallback || high_fallback) && ambiguous)) {
        out[k] = r;
        return;
    }
    double signed_volume = 0.0;
    for (uint32_t i = 0; i < t.face_count; ++i) {
        const uint3 q = tri[f[i]];
        signed_volume += tetra(pos(p, q.x), pos(p, q.y), pos(p, q.z), origin);
    }
    signed_volume += cap_volume(p, low, t.low_count, low_forward, origin);
    signed_volume += cap_volume(p, high, t.high_count, high_forward, origin);
    r.signed_volume = signed_volume;
    r.volume = fabs(signed_volume);
    r.valid = isfinite(r.volume) && r.volume > kEpsilon ? 1u : 0u;
    if (!r.valid) {
        r.signed_volume = 0.0;
        r.volume = 0.0;
    }
    out[k] = r;
}

// The position-independent part of estimateClosedCellVolume
// (cell_volume.cpp:168-240, 88-114).
CellTopology cell_topology(const swb_structure_definition& d, const uint64_t* faces, const uint64_t* loops,
                           const swb_cell_def& cell) {
    CellTopology t{};
    t.face_begin = static_cast<uint32_t>(cell.face_begin);
    t.face_count = static_cast<uint32_t>(cell.face_count);
    t.low_begin = static_cast<uint32_t>(cell.low_begin);
    t.low_count = static_cast<uint32_t>(cell.low_count);
    t.high_begin = static_cast<uint32_t>(cell.high_begin);
    t.high_count = static_cast<uint32_t>(cell.high_count);
    const auto loop_ok = [&](uint64_t begin, uint64_t count) {
        if (count < 3) return false;
        std::set<uint64_t> seen;
        for (uint64_t i = 0; i < count; ++i)
            if (loops[begin + i] >= d.node_count || !seen.insert(loops[begin + i]).second) return false;
        return true;
    };
    t.loops_ok = loop_ok(cell.low_begin, cell.low_count) && loop_ok(cell.high_begin, cell.high_count) ? 1u : 0u;
    t.fail_at = t.face_count;
    std::set<uint64_t> unique;
    struct Use {
        uint32_t count = 0;
        bool low_to_high = false;
    };
    std::map<std::pair<uint64_t, uint64_t>, Use> edges;
    const auto add_edge = [&](uint64_t a, uint64_t b) {
        const auto key = std::minmax(a, b);
        Use& u = edges[{key.first, key.second}];
        if (++u.count == 1) u.low_to_high = a == key.first;
    };
    for (uint64_t i = 0; i < cell.face_count; ++i) {
        const uint64_t fi = faces[cell.face_begin + i];
        if (fi >= d.triangle_count || !unique.insert(fi).second) {
            t.fail_at = static_cast<uint32_t>(i);
            return t;
        }
        const uint64_t* n = d.triangles[fi].nodes;
        if (n[0] >= d.node_count || n[1] >= d.node_count || n[2] >= d.node_count) {
            t.fail_at = static_cast<uint32_t>(i);
            return t;
        }
        add_edge(n[0], n[1]);
        add_edge(n[1], n[2]);
        add_edge(n[2], n[0]);
    }
    for (const auto& e : edges) {
        if (e.second.count == 1) ++t.boundary;
        else if (e.second.count > 2) ++t.non_manifold;
    }
    std::set<std::pair<uint64_t, uint64_t>> cap_edges;
    bool unique_caps = true;
    const auto cap_loop = [&](uint64_t begin, uint64_t count, int32_t& forward, int32_t& reverse) {
        for (uint64_t i = 0; i < count; ++i) {
            const uint64_t a = loops[begin + i], b = loops[begin + (i + 1) % count];
            const auto key = std::minmax(a, b);
            const std::pair<uint64_t, uint64_t> edge{key.first, key.second};
            unique_caps = cap_edges.insert(edge).second && unique_caps;
            const auto found = edges.find(edge);
            if (found != edges.end() && found->second.count == 1) {
                ++t.cap_matched;
                // a cap closes the skin when its edge runs opposite to the
                // skin's sole use of it
                if ((a == key.first) != found->second.low_to_high) ++forward;
                else ++reverse;
            }
        }
    };
    if (t.loops_ok) {
        cap_loop(cell.low_begin, cell.low_count, t.low_forward, t.low_reverse);
        cap_loop(cell.high_begin, cell.high_count, t.high_forward, t.high_reverse);
    }
    const uint64_t cap_edge_count = cell.low_count + cell.high_count;
    t.watertight = unique_caps && t.non_manifold == 0 && t.boundary == cap_edge_count &&
                           t.cap_matched == cap_edge_count
                       ? 1u
                       : 0u;
    return t;
}

template <class T>
struct DeviceBuffer {
    T* ptr = nullptr;
    explicit DeviceBuffer(const std::vector<T>& host) {
        cuda_check(cudaMalloc(&ptr, std::max<size_t>(host.size(), 1) * sizeof(T)), "cudaMalloc (cell volumes)");
        if (!host.empty())
            cuda_check(cudaMemcpy(ptr, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
    }
    ~DeviceBuffer() { cudaFree(ptr); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
};

}  // namespace
}  // namespace swb

namespace swb {
namespace {

// The position-independent tables of a set of cells, ready for upload: the
// per-cell topology, the triangles' node triples, the face and loop index
// lists (indices clamped into range: out-of-range ones only reach the
// device in faces or loops the topology rejects).
struct CellTables {
    std::vector<CellTopology> topo;
    std::vector<uint3> tri;
    std::vector<uint32_t> faces, loops;
};

CellTables cell_tables(const swb_structure_definition* definition, const uint64_t* face_indices,
                       const uint64_t* loop_nodes, const swb_cell_def* cells, uint64_t cell_count) {
    if (definition->node_count > 0xffffffffu || definition->triangle_count > 0xffffffffu)
        raise(SWB_INVALID_ARGUMENT, "definition too large for 32-bit indices");
    uint64_t faces_total = 0, loops_total = 0;
    for (uint64_t k = 0; k < cell_count; ++k) {
        faces_total = std::max(faces_total, cells[k].face_begin + cells[k].face_count);
        loops_total = std::max({loops_total, cells[k].low_begin + cells[k].low_count,
                                cells[k].high_begin + cells[k].high_count});
    }
    if ((faces_total && !face_indices) || (loops_total && !loop_nodes)) raise(SWB_INVALID_ARGUMENT, "null argument");
    if (faces_total > 0xffffffffu || loops_total > 0xffffffffu)
        raise(SWB_INVALID_ARGUMENT, "cell tables too large for 32-bit indices");
    CellTables t;
    t.topo.resize(cell_count);
    for (uint64_t k = 0; k < cell_count; ++k) t.topo[k] = cell_topology(*definition, face_indices, loop_nodes, cells[k]);
    t.tri.resize(definition->triangle_count);
    for (uint64_t i = 0; i < t.tri.size(); ++i) {
        const uint64_t* n = definition->triangles[i].nodes;
        t.tri[i] = make_uint3(static_cast<uint32_t>(std::min<uint64_t>(n[0], definition->node_count - 1)),
                              static_cast<uint32_t>(std::min<uint64_t>(n[1], definition->node_count - 1)),
                              static_cast<uint32_t>(std::min<uint64_t>(n[2], definition->node_count - 1)));
    }
    t.faces.resize(faces_total);
    t.loops.resize(loops_total);
    for (uint64_t i = 0; i < faces_total; ++i)
        t.faces[i] = static_cast<uint32_t>(std::min<uint64_t>(face_indices[i], std::max<uint64_t>(t.tri.size(), 1) - 1));
    for (uint64_t i = 0; i < loops_total; ++i)
        t.loops[i] = static_cast<uint32_t>(std::min<uint64_t>(loop_nodes[i], definition->node_count - 1));
    return t;
}

void require_gpu() {
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0)
        raise(SWB_CUDA_ERROR, "no CUDA device: the cell volume kernel needs a GPU");
}

template <class T>
T* upload_owned(std::vector<void*>& owned, const std::vector<T>& host) {
    T* p = nullptr;
    cuda_check(cudaMalloc(&p, std::max<size_t>(host.size(), 1) * sizeof(T)), "cudaMalloc (cell volume plan)");
    owned.push_back(p);
    if (!host.empty()) cuda_check(cudaMemcpy(p, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
    return p;
}

// World positions in FP64 from a structure's device state: node n is slot
// slot_of_node[n], stored as an FP32 offset from the state's FP64 origin.
__global__ void gather_world_positions(const float4* __restrict__ pos, const double* __restrict__ origin,
                                       const uint32_t* __restrict__ slot_of_node, uint32_t n, double* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 x = pos[slot_of_node[i]];
    out[3 * i] = origin[0] + static_cast<double>(x.x);
    out[3 * i + 1] = origin[1] + static_cast<double>(x.y);
    out[3 * i + 2] = origin[2] + static_cast<double>(x.z);
}

}  // namespace
}  // namespace swb

// A set of cells whose tables live on one device.
struct swb_cell_volume_plan {
    int device = 0;
    uint32_t cells = 0;
    uint64_t node_count = 0;
    swb::CellTopology* topo = nullptr;
    uint3* tri = nullptr;
    uint32_t* faces = nullptr;
    uint32_t* loops = nullptr;
    // the structure form's world positions, node-major
    double* world = nullptr;
    uint32_t* slot_of_node = nullptr;
    const void* structure = nullptr;  // the structure `slot_of_node` belongs to
    std::vector<void*> owned;
    ~swb_cell_volume_plan() {
        for (void* p : owned) cudaFree(p);
    }
};

using namespace swb;

swb_status swb_cell_volumes(const swb_structure_definition* definition, const uint64_t* face_indices,
                            const uint64_t* loop_nodes, const swb_cell_def* cells, uint64_t cell_count,
                            const double* positions, swb_cell_volume* out) {
    return guarded([&] {
        if (!definition || !positions || (cell_count && (!cells || !out))) raise(SWB_INVALID_ARGUMENT, "null argument");
        if (!cell_count) return;
        if (definition->node_count == 0) {  // no node: no valid loop, no valid face
            for (uint64_t k = 0; k < cell_count; ++k) out[k] = swb_cell_volume{};
            return;
        }
        require_gpu();
        const CellTables t = cell_tables(definition, face_indices, loop_nodes, cells, cell_count);
        std::vector<double> p(positions, positions + 3 * definition->node_count);
        DeviceBuffer<CellTopology> d_topo(t.topo);
        DeviceBuffer<uint3> d_tri(t.tri);
        DeviceBuffer<uint32_t> d_faces(t.faces), d_loops(t.loops);
        DeviceBuffer<double> d_p(p);
        std::vector<swb_cell_volume> result(cell_count);
        DeviceBuffer<swb_cell_volume> d_out(result);
        cell_volume_kernel<<<static_cast<unsigned>((cell_count + 63) / 64), 64>>>(
            static_cast<uint32_t>(cell_count), d_topo.ptr, d_tri.ptr, d_faces.ptr, d_loops.ptr, d_p.ptr, d_out.ptr);
        cuda_check(cudaGetLastError(), "cell_volume_kernel");
        cuda_check(cudaMemcpy(out, d_out.ptr, cell_count * sizeof(swb_cell_volume), cudaMemcpyDeviceToHost), "download");
    });
}

swb_status swb_cell_volume_plan_create(const swb_structure_definition* definition, const uint64_t* face_indices,
                                       const uint64_t* loop_nodes, const swb_cell_def* cells, uint64_t cell_count,
                                       int device, swb_cell_volume_plan** out) {
    return guarded([&] {
        if (!definition || !out || (cell_count && !cells)) raise(SWB_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        if (cell_count > 0xffffffffu) raise(SWB_INVALID_ARGUMENT, "too many cells");
        if (definition->node_count == 0) raise(SWB_INVALID_ARGUMENT, "definition has no node");
        require_gpu();
        const CellTables t = cell_tables(definition, face_indices, loop_nodes, cells, cell_count);
        cuda_check(cudaSetDevice(device), "cudaSetDevice");
        auto plan = std::make_unique<swb_cell_volume_plan>();
        plan->device = device;
        plan->cells = static_cast<uint32_t>(cell_count);
        plan->node_count = definition->node_count;
        plan->topo = upload_owned(plan->owned, t.topo);
        plan->tri = upload_owned(plan->owned, t.tri);
        plan->faces = upload_owned(plan->owned, t.faces);
        plan->loops = upload_owned(plan->owned, t.loops);
        plan->world = upload_owned(plan->owned, std::vector<double>(3 * definition->node_count));
        plan->slot_of_node = upload_owned(plan->owned, std::vector<uint32_t>(definition->node_count));
        *out = plan.release();
    });
}

void swb_cell_volume_plan_destroy(swb_cell_volume_plan* plan) {
    if (!plan) return;
    cudaSetDevice(plan->device);
    delete plan;
}

swb_status swb_cell_volumes_device(const swb_cell_volume_plan* plan, const double* positions, swb_cell_volume* out,
                                   void* stream) {
    return guarded([&] {
        if (!plan || !positions || (plan->cells && !out)) raise(SWB_INVALID_ARGUMENT, "null argument");
        if (!plan->cells) return;
        cuda_check(cudaSetDevice(plan->device), "cudaSetDevice");
        cell_volume_kernel<<<(plan->cells + 63) / 64, 64, 0, static_cast<cudaStream_t>(stream)>>>(
            plan->cells, plan->topo, plan->tri, plan->faces, plan->loops, positions, out);
        cuda_check(cudaGetLastError(), "cell_volume_kernel");
    });
}

swb_status swb_structure_cell_volumes(const swb_structure* s, swb_cell_volume_plan* plan, swb_cell_volume* out) {
    return guarded([&] {
        if (!s || !plan || (plan->cells && !out)) raise(SWB_INVALID_ARGUMENT, "null argument");
        const StructureImpl& m = s->s;
        if (m.def.nodes.size() != plan->node_count) raise(SWB_INVALID_ARGUMENT, "plan belongs to another definition");
        if (m.device != plan->device) raise(SWB_INVALID_ARGUMENT, "plan and structure are on different devices");
        cuda_check(cudaSetDevice(plan->device), "cudaSetDevice");
        if (plan->structure != s) {
            // first use with this structure: its node -> slot table
            cuda_check(cudaMemcpy(plan->slot_of_node, m.slot_of_node.data(), plan->node_count * sizeof(uint32_t),
                                  cudaMemcpyHostToDevice), "upload");
            plan->structure = s;
        }
        const uint32_t n = static_cast<uint32_t>(plan->node_count);
        gather_world_positions<<<(n + 255) / 256, 256, 0, m.stream>>>(m.d_pos[m.cur], m.d_origin[m.cur],
                                                                       plan->slot_of_node, n, plan->world);
        cuda_check(cudaGetLastError(), "gather_world_positions");
        if (!plan->cells) return;
        cell_volume_kernel<<<(plan->cells + 63) / 64, 64, 0, m.stream>>>(plan->cells, plan->topo, plan->tri,
                                                                          plan->faces, plan->loops, plan->world, out);
        cuda_check(cudaGetLastError(), "cell_volume_kernel");
    });
}
