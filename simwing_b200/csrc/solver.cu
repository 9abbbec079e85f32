// Single-structure device solver: the swb_structure_* entry points.
// Replaces simwing::fsi::Structure (src/fsi/structure.h:273-309).
#include "common.h"
#include "schedule.h"
#include "adjoint_kernel.cuh"
#include "cluster_kernel.cuh"
#include "step_kernel.cuh"
#include "structure_impl.h"

#include <algorithm>
#include <limits>
#include <bit>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>

namespace swb {

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess)
        raise(e == cudaErrorMemoryAllocation ? SWB_OUT_OF_MEMORY : SWB_CUDA_ERROR,
              std::string(what) + ": " + cudaGetErrorString(e));
}

namespace {

// A point on the origin grid (1/256 m) nearest to x.
double origin_grid(double x) { return std::nearbyint(x * 256.0) / 256.0; }

void initial_origin(const OwnedDefinition& def, double o[3]) {
    o[0] = o[1] = o[2] = 0.0;
    if (def.has_suspension) {
        const swb_vec3& c = def.suspension.pilot_initial_com_world;
        o[0] = origin_grid(c.x);
        o[1] = origin_grid(c.y);
        o[2] = origin_grid(c.z);
        return;
    }
    if (def.nodes.empty()) return;
    double lo[3], hi[3];
    for (int k = 0; k < 3; ++k) lo[k] = hi[k] = (&def.nodes[0].position.x)[k];
    for (const auto& n : def.nodes)
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], (&n.position.x)[k]);
            hi[k] = std::max(hi[k], (&n.position.x)[k]);
        }
    for (int k = 0; k < 3; ++k) o[k] = origin_grid(0.5 * (lo[k] + hi[k]));
}

template <class T>
T* dalloc(std::vector<void*>& owned, size_t count) {
    void* p = nullptr;
    cuda_check(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)), "cudaMalloc");
    owned.push_back(p);
    return static_cast<T*>(p);
}

template <class T>
T* dupload(std::vector<void*>& owned, const std::vector<T>& host, cudaStream_t s) {
    T* p = dalloc<T>(owned, host.size());
    if (!host.empty())
        cuda_check(cudaMemcpyAsync(p, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice, s),
                   "cudaMemcpyAsync");
    return p;
}

uint32_t align16(uint32_t v) { return (v + 15u) & ~15u; }

// Sort key of the reference's suspension normalisation: records are sorted
// by their string ids "segment:<id>" / "harness:<id>"
// (suspension.cpp:1000-1006), i.e. by the decimal spelling of the id.
bool id_string_less(uint64_t a, uint64_t b) { return std::to_string(a) < std::to_string(b); }

// The fabric self-contact multiplier table is part of the step transaction,
// as the reference's contactMultipliers_ / contactRecords_ are
// (soft_body.cpp:1090-1112): the step's contact iterations ping-pong the
// table, so the committed table is copied aside before a step and put back
// when the step fails.  Both kernels read the entry count on the device.
__global__ void contact_table_save(const ContactDev* c, ContactEntry* out, uint32_t* meta_out) {
    const uint32_t sel = c->table_meta[0], n = c->table_meta[1];
    const ContactEntry* src = c->table[sel];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = src[i];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        meta_out[0] = 0u;
        meta_out[1] = n;
        *c->fail = ~0ull;  // no failing feature yet
    }
}

__global__ void contact_table_restore(const ContactDev* c, const ContactEntry* in, const uint32_t* meta_in) {
    const uint32_t n = meta_in[1];
    ContactEntry* dst = c->table[0];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = in[i];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        c->table_meta[0] = 0u;
        c->table_meta[1] = n;
    }
}

// Diagnostics partial sums per CTA (double).
constexpr int kDiagFields = 16;

__global__ void diagnostics_kernel(const float4* pos, const float4* prev, const float4* vel, uint32_t n,
                                   const uint32_t* ca, const uint32_t* cb, const float* rest, const uint8_t* kind,
                                   uint32_t m, const uint4* mem, const float4* maux, const float* mres, uint32_t nm,
                                   double* partials) {
    // fields: 0 dyn count, 1 mass, 2-4 sum m x, 5-7 sum m v, 8 KE, 9 finite(min),
    //         10 max |distance error|, 11 max cable extension,
    //         12 max |membrane strain component|, 13 max |membrane residual|
    constexpr int F = 14;
    double acc[F] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0};
    const uint32_t stride = blockDim.x * gridDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float4 X = pos[i], P = prev[i], V = vel[i];
        const bool fin = isfinite(X.x) && isfinite(X.y) && isfinite(X.z) && isfinite(P.x) && isfinite(P.y) &&
                         isfinite(P.z) && isfinite(V.x) && isfinite(V.y) && isfinite(V.z) && isfinite(X.w) &&
                         X.w >= 0.0f;
        if (!fin) acc[9] = 0.0;
        if (X.w > 0.0f) {
            const double mass = 1.0 / static_cast<double>(X.w);
            acc[0] += 1.0;
            acc[1] += mass;
            acc[2] += mass * X.x; acc[3] += mass * X.y; acc[4] += mass * X.z;
            acc[5] += mass * V.x; acc[6] += mass * V.y; acc[7] += mass * V.z;
            acc[8] += 0.5 * mass * (double(V.x) * V.x + double(V.y) * V.y + double(V.z) * V.z);
        }
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        const float4 A = pos[ca[i]], B = pos[cb[i]];
        const double dx = double(B.x) - A.x, dy = double(B.y) - A.y, dz = double(B.z) - A.z;
        const double e = sqrt(dx * dx + dy * dy + dz * dz) - rest[i];
        if (kind[i] == SWB_CONSTRAINT_CABLE) acc[11] = fmax(acc[11], fmax(0.0, e));
        else acc[10] = fmax(acc[10], fabs(e));
    }
    // membrane Green strain at the current positions (evaluateMembraneElement,
    // soft_body.cpp:204-225) and the last substep's residual
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nm; i += stride) {
        const uint4 e = mem[i];
        const float4 q0 = maux[static_cast<size_t>(e.w) * kMembraneAux];
        const float4 q1 = maux[static_cast<size_t>(e.w) * kMembraneAux + 1];
        const float4 q2 = maux[static_cast<size_t>(e.w) * kMembraneAux + 2];
        const float4 A = pos[e.x], B = pos[e.y], C = pos[e.z];
        const double e1[3] = {double(B.x) - A.x, double(B.y) - A.y, double(B.z) - A.z};
        const double e2[3] = {double(C.x) - A.x, double(C.y) - A.y, double(C.z) - A.z};
        double wa[3], wf[3];
        for (int k = 0; k < 3; ++k) {
            wa[k] = q0.x * e1[k] + q0.z * e2[k];
            wf[k] = q0.y * e1[k] + q0.w * e2[k];
        }
        const double sx = 0.5 * (wa[0] * wa[0] + wa[1] * wa[1] + wa[2] * wa[2] - 1.0) + q1.w;
        const double sy = 0.5 * (wf[0] * wf[0] + wf[1] * wf[1] + wf[2] * wf[2] - 1.0) + q2.x;
        const double sz = wa[0] * wf[0] + wa[1] * wf[1] + wa[2] * wf[2];
        const double r = mres[e.w];
        if (!isfinite(sx) || !isfinite(sy) || !isfinite(sz) || !isfinite(r)) acc[9] = 0.0;
        acc[12] = fmax(acc[12], fmax(fabs(sx), fmax(fabs(sy), fabs(sz))));
        acc[13] = fmax(acc[13], fabs(r));
    }
    __shared__ double red[32][F];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int f = 0; f < F; ++f) {
        double v = acc[f];
        for (int o = 16; o > 0; o >>= 1) {
            const double u = __shfl_down_sync(0xffffffffu, v, o);
            v = f == 9 ? fmin(v, u) : (f >= 10 ? fmax(v, u) : v + u);
        }
        if (lane == 0) red[warp][f] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int warps = (blockDim.x + 31) / 32;
        for (int f = 0; f < F; ++f) {
            double v = red[0][f];
            for (int w = 1; w < warps; ++w)
                v = f == 9 ? fmin(v, red[w][f]) : (f >= 10 ? fmax(v, red[w][f]) : v + red[w][f]);
            partials[blockIdx.x * kDiagFields + f] = v;
        }
    }
}

}  // namespace

// ---- Structure construction --------------------------------------------------

StructureImpl::~StructureImpl() {
    if (device >= 0) cudaSetDevice(device);
    for (void* p : owned) cudaFree(p);
    if (h_force) cudaFreeHost(h_force);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
}

void StructureImpl::build(const swb_structure_definition& definition, const swb_solver_options* options) {
    def.assign(definition);
    validate_definition(def.view);
    fingerprint = definition_fingerprint(def.view);
    if (def.has_contact) contact_surface = build_contact_surface(def.view, def.contact.half_thickness);
    // Solver-drift momentum restoration of isolated free structures: no
    // suspension, no contact, bending or membranes present, no fixed node.
    momentum_guard = !def.has_suspension && !def.has_contact && (!def.dihedrals.empty() || !def.membranes.empty()) &&
                     std::none_of(def.nodes.begin(), def.nodes.end(), [](const swb_node_def& n) { return n.fixed != 0; });
    swb_solver_options opt;
    swb_default_solver_options(&opt);
    if (options) opt = *options;
    device = opt.device;
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    cudaDeviceProp prop{};
    cuda_check(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
    if (!prop.cooperativeLaunch) raise(SWB_UNSUPPORTED, "device lacks cooperative launch");
    sm_count = prop.multiProcessorCount;
    cuda_check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
    cuda_check(cudaEventCreate(&ev0), "cudaEventCreate");
    cuda_check(cudaEventCreate(&ev1), "cudaEventCreate");

    const uint64_t N = def.nodes.size();
    if (N >= (1ull << 31)) raise(SWB_UNSUPPORTED, "too many nodes");
    pending.assign(N, swb_vec3{0, 0, 0});
    pressure.resize(def.triangles.size());
    for (size_t t = 0; t < def.triangles.size(); ++t) pressure[t] = def.triangles[t].pressure_difference;

    // Suspension: endpoint nodes must share one level-1 patch.
    if (def.has_suspension && (def.segments.size() > 8 || def.harness.size() > 8))
        raise(SWB_UNSUPPORTED, "more than 8 suspension segments or harness points");
    const std::vector<uint32_t> susp_nodes = suspension_endpoint_nodes(def);
    const size_t smem_limit = dynamic_smem_limit(prop);
    smem_cap = smem_limit;
    cluster_mode = false;
    if (!(opt.flags & (SWB_OPT_GRID | SWB_OPT_GLOBAL_ONLY))) {
        if (opt.cluster_ctas < 0 || opt.cluster_ctas > kClusterMaxCtas)
            raise(SWB_INVALID_ARGUMENT, "cluster_ctas must be in 0..16");
        std::vector<int> candidates;
        if (opt.cluster_ctas > 0) {
            candidates.push_back(opt.cluster_ctas);
        } else if (def.has_contact) {
            // the contact phases run over the whole cluster: the widest that fits
            for (int c = kClusterMaxCtas; c >= 1; c /= 2) candidates.push_back(c);
        } else {
            int c = 1;
            while (c < kClusterMaxCtas && static_cast<uint64_t>(c) * 2048 < N) c *= 2;
            for (; c <= kClusterMaxCtas; c *= 2) candidates.push_back(c);
        }
        for (int c : candidates) {
            if (!build_cluster_schedule(def, susp_nodes, c, csched, (opt.flags & SWB_OPT_SPLIT_STAGES) != 0)) continue;
            const size_t bytes = cluster_shared_bytes(csched);
            if (bytes > smem_limit) continue;
            cluster_mode = true;
            break;
        }
        if (!cluster_mode && opt.cluster_ctas > 0)
            raise(SWB_UNSUPPORTED, "the mesh does not fit a cluster of " + std::to_string(opt.cluster_ctas) + " CTAs");
    }
    if (!cluster_mode && momentum_guard)
        raise(SWB_UNSUPPORTED, "the momentum guard of a free structure needs the cluster schedule (the mesh does not fit one)");
    if (!cluster_mode && !def.membranes.empty())
        raise(SWB_UNSUPPORTED, "membrane elements need the cluster schedule (the mesh does not fit one)");
    if (!cluster_mode && def.has_contact)
        raise(SWB_UNSUPPORTED, "fabric self-contact needs the cluster schedule (the mesh does not fit one)");
    uint32_t widest = 32;
    if (cluster_mode) {
        verify_cluster_schedule(def, susp_nodes, csched);
        G = csched.ctas;
        slot_of_node = csched.slot_of_node;
        node_of_slot = csched.node_of_slot;
        susp_owner = csched.susp_cta;
        susp_base = susp_owner >= 0 ? csched.patch_begin[susp_owner] : 0;
        for (int k = 0; k < 2; ++k) {
            const ClusterKind& K = csched.kinds[k];
            for (int c = 0; c < G; ++c)
                for (int s = 0; s < K.stages; ++s) {
                    const size_t o = static_cast<size_t>(c) * (K.stages + 1) + s;
                    widest = std::max(widest, K.offsets[o + 1] - K.offsets[o]);
                }
        }
    } else {
        ScheduleOptions so;
        so.blocks = opt.blocks > 0 ? opt.blocks : sm_count;
        so.blocks = static_cast<int>(std::min<uint64_t>(so.blocks, std::max<uint64_t>(1, N)));
        so.levels = opt.partition_levels > 0 ? opt.partition_levels : 3;
        so.global_only = (opt.flags & SWB_OPT_GLOBAL_ONLY) != 0;
        sched = build_schedule(def, susp_nodes, so);
        verify_schedule(def, susp_nodes, sched);
        G = sched.blocks;
        slot_of_node = sched.slot_of_node;
        node_of_slot = sched.node_of_slot;
        susp_owner = sched.suspension_block;
        susp_base = susp_owner >= 0 ? sched.l1_begin[susp_owner] : 0;
        // Threads per CTA: enough for the widest local stage, in warps.
        for (int l = 0; l < sched.levels; ++l)
            for (int k = 0; k < kKinds; ++k) {
                const Table& t = sched.tables[l][k];
                for (int b = 0; b < G; ++b)
                    for (int s = 0; s < t.stages; ++s) {
                        const size_t o = static_cast<size_t>(b) * (t.stages + 1) + s;
                        widest = std::max(widest, t.stage_offsets[o + 1] - t.stage_offsets[o]);
                    }
            }
    }
    threads = opt.block_threads > 0
                  ? opt.block_threads
                  : static_cast<int>(std::clamp<uint32_t>((widest + 31) / 32 * 32, 64,
                                                          cluster_mode ? dev::kClusterMaxThreads : 512));
    if (opt.block_threads <= 0 && cluster_mode && def.has_contact) threads = dev::kClusterMaxThreads;
    if (threads % 32 != 0 || threads < 32 || threads > (cluster_mode ? dev::kClusterMaxThreads : 1024))
        raise(SWB_INVALID_ARGUMENT, "block_threads out of range for the chosen schedule");
    if (cluster_mode && csched.line_stage >= 0) {
        // the line iteration needs a warp of the suspension CTA that is idle
        // in its two stages
        const int need = static_cast<int>((csched.line_owner_records + 31) / 32 * 32 + 32);
        if (opt.block_threads <= 0 && need > threads && need <= dev::kClusterMaxThreads) threads = need;
        if (need > threads) csched.line_stage = -1;
    }

    // ---- device images -------------------------------------------------------
    // The node states are FP32 offsets from an FP64 origin on a 1/256 m grid
    // (a shift by a grid step is exact in both).  The origin starts at the
    // pilot's centre of mass when there is one (the step recentres there
    // whenever the pilot has moved a quarter metre), else at the centre of
    // the nodes' bounding box, so that the offsets are as small as the
    // structure allows from the first step on.
    initial_origin(def, origin0);
    // nodes (slot order)
    std::vector<float4> pos(N), vel(N, make_float4(0, 0, 0, 0));
    for (uint64_t s = 0; s < N; ++s) {
        const swb_node_def& n = def.nodes[node_of_slot[s]];
        const float w = n.fixed ? 0.0f : static_cast<float>(1.0 / n.mass);
        pos[s] = make_float4(static_cast<float>(n.position.x - origin0[0]), static_cast<float>(n.position.y - origin0[1]),
                             static_cast<float>(n.position.z - origin0[2]), w);
    }
    inv_mass.resize(N);
    for (uint64_t s = 0; s < N; ++s) inv_mass[s] = pos[s].w;
    for (int i = 0; i < 3; ++i) {
        d_pos[i] = dupload(owned, pos, stream);
        d_vel[i] = dupload(owned, vel, stream);
        d_prev[i] = dupload(owned, pos, stream);
    }
    d_force = dalloc<float4>(owned, N);
    cuda_check(cudaMemsetAsync(d_force, 0, N * sizeof(float4), stream), "memset");
    cuda_check(cudaMallocHost(&h_force, std::max<uint64_t>(N, 1) * sizeof(float4)), "cudaMallocHost");

    // schedule tables
    StepParams& p = params;
    std::memset(&p, 0, sizeof(p));
    upload_pressure();  // fills params.tri*, so after the reset above
    p.blocks = G;
    if (cluster_mode) {
        upload_cluster_tables();
    } else {
        upload_grid_tables();
    }
    finish_build(opt, prop);
}

// Device constants of one membrane element (kMembraneAux float4, layout in
// cluster_params.h): the chart's inverse edge matrix, sqrt(area) and the
// material's compliance, computed in FP64 as addMembraneElements does
// (soft_body.cpp:664-690, membrane.cpp:131-271), then rounded.
static void membrane_constants(const swb_membrane_def& m, float4 out[kMembraneAux]) {
    const double e1x = m.chart[1][0] - m.chart[0][0], e1y = m.chart[1][1] - m.chart[0][1];
    const double e2x = m.chart[2][0] - m.chart[0][0], e2y = m.chart[2][1] - m.chart[0][1];
    const double det = e1x * e2y - e2x * e1y;  // edge matrix [e1x e2x; e1y e2y]
    const double id = 1.0 / det;
    const double i00 = e2y * id, i01 = -e2x * id, i10 = -e1y * id, i11 = e1x * id;
    const swb_membrane_material& q = m.material;
    const double kxx = q.warp_stiffness, kyy = q.weft_stiffness, kzz = q.shear_stiffness, kxy = q.coupling_stiffness;
    // symmetric inverse of [kxx kxy 0; kxy kyy 0; 0 0 kzz]
    const double kdet = kxx * (kyy * kzz) - kxy * (kxy * kzz);
    const double kid = 1.0 / kdet;
    const double cxx = (kyy * kzz) * kid, cyy = (kxx * kzz) * kid, czz = (kxx * kyy - kxy * kxy) * kid;
    const double cxy = (-kxy * kzz) * kid;
    auto f = [](double v) { return static_cast<float>(v); };
    out[0] = make_float4(f(i00), f(i01), f(i10), f(i11));
    out[1] = make_float4(f(std::sqrt(0.5 * det)), f(q.damping_seconds), f(q.compression_stiffness_ratio),
                         f(q.warp_pretension));
    out[2] = make_float4(f(q.weft_pretension), f(cxx), f(cyy), f(czz));
    out[3] = make_float4(f(cxy), 0.0f, 0.0f, f(kxx));
    out[4] = make_float4(f(kyy), f(kzz), f(kxy), 0.0f);
}

// One instance record per (input, output) buffer pair, so that a launch only
// selects a pointer; uploaded again when a setting they carry changes.
void StructureImpl::upload_instances() {
    std::vector<ClusterInstance> inst(9);
    for (int in = 0; in < 3; ++in)
        for (int out = 0; out < 3; ++out) {
            ClusterInstance c = cluster_base;
            c.pos_in = d_pos[in]; c.vel_in = d_vel[in];
            c.pos_out = d_pos[out]; c.vel_out = d_vel[out]; c.prev_out = d_prev[out];
            c.force = d_force;
            c.tri_offsets = d_tri_off; c.tri_list = d_tri_list; c.tri = d_tri;
            c.susp_cta = def.has_suspension ? susp_owner : -1;
            c.payload_def = d_payload_def;
            c.payload_in = d_payload[in]; c.payload_out = d_payload[out];
            c.origin_in = d_origin[in]; c.origin_out = d_origin[out];
            c.membrane_residual = d_mres[out];
            c.contact = d_contact;
            c.contact_diag = d_cdiag[out];
            c.lines = line_contact ? d_lines : nullptr;
            c.status = d_control->status;
            c.recentre = def.has_suspension ? 1 : 0;
            inst[in * 3 + out] = c;
        }
    if (!d_instances) {
        d_instances = dupload(owned, inst, stream);
    } else {
        cuda_check(cudaMemcpyAsync(d_instances, inst.data(), inst.size() * sizeof(ClusterInstance),
                                   cudaMemcpyHostToDevice, stream), "instance upload");
        cuda_check(cudaStreamSynchronize(stream), "instance upload");
    }
}

// The cable segments of line-line contact and their step scratch (once).
void StructureImpl::setup_line_contact() {
    std::vector<std::pair<uint64_t, uint64_t>> segs;
    for (const auto& c : def.constraints)
        if (c.kind == SWB_CONSTRAINT_CABLE)
            segs.push_back({std::min(c.first_node, c.second_node), std::max(c.first_node, c.second_node)});
    std::sort(segs.begin(), segs.end());
    segs.erase(std::unique(segs.begin(), segs.end()), segs.end());
    if (segs.size() > 65535) raise(SWB_UNSUPPORTED, "line-line contact takes at most 65,535 cable segments");
    auto ref = [&](uint64_t node) {
        const uint32_t slot = slot_of_node[node];
        uint32_t cta = 0;
        while (cta + 1 < static_cast<uint32_t>(G) && csched.patch_begin[cta + 1] <= slot) ++cta;
        return (cta << 12) | (slot - csched.patch_begin[cta]);
    };
    std::vector<uint32_t> seg(segs.size());
    std::vector<uint2> nodes(segs.size());
    for (size_t i = 0; i < segs.size(); ++i) {
        seg[i] = ref(segs[i].first) | (ref(segs[i].second) << 16);
        nodes[i] = make_uint2(static_cast<uint32_t>(segs[i].first), static_cast<uint32_t>(segs[i].second));
    }
    LineContactDev L{};
    L.segments = static_cast<uint32_t>(segs.size());
    L.capacity = 1u << 16;
    L.seg = dupload(owned, seg, stream);
    L.seg_nodes = dupload(owned, nodes, stream);
    L.box = dalloc<float4>(owned, 2 * std::max<size_t>(segs.size(), 1));
    L.pair = dalloc<uint32_t>(owned, L.capacity);
    L.sort = dalloc<uint32_t>(owned, L.capacity);
    L.order = dalloc<uint32_t>(owned, L.capacity);
    L.pred = dalloc<uint32_t>(owned, 4 * static_cast<size_t>(L.capacity));
    L.level_off = dalloc<uint32_t>(owned, L.capacity + 1);
    L.count = dalloc<uint32_t>(owned, 2);
    lines_host = L;
    d_lines = dupload(owned, std::vector<LineContactDev>{L}, stream);
}

void (*StructureImpl::step_kernel() const)(ClusterParams) {
    if (def.has_contact)
        return def.membranes.empty() ? dev::xpbd_cluster_contact_kernel : dev::xpbd_cluster_contact_membrane_kernel;
    return def.membranes.empty() ? dev::xpbd_cluster_kernel : dev::xpbd_cluster_membrane_kernel;
}

// Device tables and scratch of the fabric self-contact phases: the surface
// by node slot, the candidate list of one phase, the per-thread queues of
// the swept queries, the ping-pong multiplier table and the record book.
// Capacities: up to kContactCapacity candidates per phase (and as many
// warm-started features and records); beyond that the step fails with
// SWB_CONTACT_ERROR.
void StructureImpl::setup_contact(const swb_solver_options& opt) {
    constexpr uint64_t kContactCapacity = uint64_t(1) << 20;
    const ContactSurface& S = contact_surface;
    ContactDev c{};
    c.nv = static_cast<uint32_t>(S.vertices.size());
    c.ne = static_cast<uint32_t>(S.edges.size());
    c.nt = static_cast<uint32_t>(S.triangles.size());
    std::vector<uint32_t> vid(c.nv);
    std::vector<uint2> eid(c.ne);
    std::vector<uint3> tid(c.nt);
    for (uint32_t i = 0; i < c.nv; ++i) vid[i] = slot_of_node[S.vertices[i]];
    for (uint32_t i = 0; i < c.ne; ++i) eid[i] = make_uint2(slot_of_node[S.edges[i][0]], slot_of_node[S.edges[i][1]]);
    for (uint32_t i = 0; i < c.nt; ++i)
        tid[i] = make_uint3(slot_of_node[S.triangles[i][0]], slot_of_node[S.triangles[i][1]],
                            slot_of_node[S.triangles[i][2]]);
    c.vid = dupload(owned, vid, stream);
    c.eid = dupload(owned, eid, stream);
    c.tid = dupload(owned, tid, stream);
    c.separation = 2.0 * def.contact.half_thickness;
    c.compliance = def.contact.normal_compliance;
    c.static_mu = def.contact.static_friction;
    c.dynamic_mu = def.contact.dynamic_friction;
    swb_default_ccd_settings(&c.ccd);  // Structure steps with the default CCD settings
    c.snapshot = dalloc<float4>(owned, def.nodes.size());
    c.vbox = dalloc<double>(owned, 6 * static_cast<size_t>(c.nv));
    c.ebox = dalloc<double>(owned, 6 * static_cast<size_t>(c.ne));
    c.tbox = dalloc<double>(owned, 6 * static_cast<size_t>(c.nt));
    c.counts = dalloc<uint32_t>(owned, static_cast<size_t>(c.nv) + c.ne);
    c.offsets = dalloc<unsigned long long>(owned, static_cast<size_t>(c.nv) + c.ne + 1);
    cuda_check(cudaMemsetAsync(c.offsets, 0, (static_cast<size_t>(c.nv) + c.ne + 1) * sizeof(unsigned long long),
                               stream), "memset");
    const uint64_t cap = std::max<uint64_t>(1, std::min<uint64_t>(S.possible, kContactCapacity));
    c.cand_cap = cap;
    c.cand = dalloc<unsigned long long>(owned, cap);
    c.query = dalloc<ContactQuery>(owned, cap);
    // helper clusters of the detection phases: as many as can be resident
    // beside the structure's cluster in one cooperative launch, at most
    // kMaxContactHelpers, for surfaces of kContactHelperRows candidate rows
    // or more (on smaller ones the grid barriers cost more than the spread
    // work saves: 16 x 16 sheets, 2,000 rows, step in 18.0 ms with helpers
    // against 14.1 ms without)
    contact_helpers = 0;
    if (!(opt.flags & SWB_OPT_CONTACT_ONE_CLUSTER) && c.nv + c.ne >= kContactHelperRows) {
        const auto kernel = step_kernel();
        cudaLaunchConfig_t cfg{};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = static_cast<unsigned>(G);
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(G);
        cfg.blockDim = dim3(threads);
        cfg.dynamicSmemBytes = cluster_smem;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int clusters = 0;
        if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem_cap)) == cudaSuccess &&
            (G <= 8 || cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) &&
            cudaOccupancyMaxActiveClusters(&clusters, kernel, &cfg) == cudaSuccess)
            contact_helpers = std::clamp(clusters - 1, 0, kMaxContactHelpers);
        (void)cudaGetLastError();
    }
    c.queue_stride = static_cast<uint32_t>(c.ccd.interval_subdivisions + 1);
    c.queues = dalloc<double>(owned, static_cast<size_t>(G) * (1 + contact_helpers) * threads * c.queue_stride * 4);
    for (int b = 0; b < 2; ++b) c.table[b] = dalloc<ContactEntry>(owned, cap);
    c.table_meta = dalloc<uint32_t>(owned, 2);
    cuda_check(cudaMemsetAsync(c.table_meta, 0, 2 * sizeof(uint32_t), stream), "memset");
    c.table_cap = cap;
    c.records = dalloc<ContactRecordDev>(owned, cap);
    c.record_cap = cap;
    c.hit = dalloc<uint32_t>(owned, cap);
    // binned broadphase along the longest extent of the initial geometry
    {
        double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
        for (size_t i = 0; i < def.nodes.size(); ++i) {
            const double q[3] = {def.nodes[i].position.x, def.nodes[i].position.y, def.nodes[i].position.z};
            for (int k = 0; k < 3; ++k) {
                lo[k] = i ? std::min(lo[k], q[k]) : q[k];
                hi[k] = i ? std::max(hi[k], q[k]) : q[k];
            }
        }
        int order[3] = {0, 1, 2};
        std::sort(order, order + 3, [&](int a, int b) { return hi[a] - lo[a] > hi[b] - lo[b]; });
        c.axis = order[0];
        c.axis2 = order[1];
    }
    c.bins_cap = 1u << 16;
    c.tbin = dalloc<uint32_t>(owned, c.bins_cap + 1);
    c.tbin_fill = dalloc<uint32_t>(owned, c.bins_cap + 1);
    c.tbin_items = dalloc<uint32_t>(owned, std::max<uint32_t>(c.nt, 1));
    c.ebin = dalloc<uint32_t>(owned, c.bins_cap + 1);
    c.ebin_fill = dalloc<uint32_t>(owned, c.bins_cap + 1);
    c.ebin_items = dalloc<uint32_t>(owned, std::max<uint32_t>(c.ne, 1));
    c.range = dalloc<unsigned long long>(owned, 12);
    c.cand_tmp = dalloc<uint32_t>(owned, cap);
    c.mark_a = dalloc<uint32_t>(owned, cap + 1);
    c.mark_b = dalloc<uint32_t>(owned, cap + 1);
    c.cand_entry = dalloc<ContactEntry>(owned, cap);
    c.cand_rec = dalloc<ContactRecordDev>(owned, cap);
    c.reduce = dalloc<unsigned long long>(owned, 2);
    // a failing feature is packed as row << 37 | col << 5 | detail
    if (static_cast<uint64_t>(c.nv) + c.ne >= (uint64_t(1) << 27))
        raise(SWB_UNSUPPORTED, "fabric self-contact surface too large for the device feature codes");
    c.lv_node_start = dalloc<uint32_t>(owned, def.nodes.size() + 1);
    c.lv_node_fill = dalloc<uint32_t>(owned, std::max<size_t>(def.nodes.size(), 1));
    c.lv_pairs = dalloc<uint32_t>(owned, 6 * cap);
    c.lv_succ = dalloc<uint32_t>(owned, 6 * cap);
    c.lv_nsucc = dalloc<uint32_t>(owned, cap);
    c.lv_npred = dalloc<uint32_t>(owned, cap);
    c.lv_front = dalloc<uint32_t>(owned, 2 * cap);
    c.fail = dalloc<unsigned long long>(owned, 1);
    cuda_check(cudaMemsetAsync(c.fail, 0xff, sizeof(unsigned long long), stream), "memset");
    d_contact = dupload(owned, std::vector<ContactDev>{c}, stream);
    contact_host = c;
    d_table_commit = dalloc<ContactEntry>(owned, cap);
    d_meta_commit = dalloc<uint32_t>(owned, 2);
    cuda_check(cudaMemsetAsync(d_meta_commit, 0, 2 * sizeof(uint32_t), stream), "memset");
    for (int b = 0; b < 3; ++b) {
        d_cdiag[b] = dalloc<ContactDiagDev>(owned, 1);
        cuda_check(cudaMemsetAsync(d_cdiag[b], 0, sizeof(ContactDiagDev), stream), "memset");
    }
}

void StructureImpl::upload_cluster_tables() {
    ClusterParams& cp = cparams;
    std::memset(&cp, 0, sizeof(cp));
    cp.ctas = G;
    uint32_t off = 0;
    cp.smem_x = off; off = align16(off + csched.max_patch * 16u);
    cp.smem_v = off; off = align16(off + csched.max_patch * 16u);
    ClusterInstance base{};
    base.patch_begin = dupload(owned, csched.patch_begin, stream);
    for (int k = 0; k < 3; ++k) {
        const ClusterKind& K = csched.kinds[k];
        ClusterKindDev& dk = base.kind[k];
        dk.offsets = dupload(owned, K.offsets, stream);
        std::vector<uint4> rec(K.ab.size());
        for (size_t r = 0; r < rec.size(); ++r)
            rec[r] = make_uint4(K.ab[r], k >= 1 ? K.cd[r] : 0u, std::bit_cast<uint32_t>(K.rest[r]),
                                std::bit_cast<uint32_t>(K.comp[r]));
        dk.rec = dupload(owned, rec, stream);
        if (k == 2) {
            std::vector<float4> aux(rec.size() * kMembraneAux);
            for (size_t r = 0; r < rec.size(); ++r) membrane_constants(def.membranes[K.def_index[r]], &aux[r * kMembraneAux]);
            dk.aux = dupload(owned, aux, stream);
            for (int b = 0; b < 3; ++b) {
                d_mres[b] = dalloc<float>(owned, rec.size());
                cuda_check(cudaMemsetAsync(d_mres[b], 0, std::max<size_t>(rec.size(), 1) * sizeof(float), stream),
                           "memset");
            }
        }
        dk.stages = K.stages;
        dk.smem_lambda = off;
        // stages from 64 on always take a cluster barrier (a superset of any CTA barrier)
        dk.sync_mask = 0;
        for (int g = 0; g < std::min(K.stages, 64); ++g)
            if (K.cluster_sync[g]) dk.sync_mask |= 1ull << g;
        dk.interior_stages = K.interior_stages;
        off = align16(off + K.max_cta_records * (k == 2 ? 12u : 4u));
    }
    cp.smem_offsets = off;
    off = align16(off + (total_stages(csched) + 3) * 4u);
    cluster_smem = off;
    base.seam_offsets = dupload(owned, csched.seam_offsets, stream);
    base.seam_ab = dupload(owned, csched.seam_ab, stream);
    base.seam_stages = csched.seam_stages;
    base.line_stage = csched.line_stage;
    base.pair_stages = csched.pair_stages;
    base.pair_offsets = dupload(owned, csched.pair_offsets, stream);
    base.pair_rec = dupload(owned, csched.pair_rec, stream);
    base.momentum_guard = momentum_guard ? 1 : 0;
    cluster_base = base;
}

void StructureImpl::upload_grid_tables() {
    StepParams& p = params;
    p.levels = sched.levels;
    p.l1_begin = dupload(owned, sched.l1_begin, stream);
    uint32_t off = 0;
    sched_n1_max = static_cast<uint32_t>(sched.max_patch_nodes);
    sched_n2_max = static_cast<uint32_t>(sched.max_gather_nodes);
    p.n1_max = sched_n1_max;
    p.n2_max = sched_n2_max;
    p.smem_x1 = off; off = align16(off + sched_n1_max * 16u);
    p.smem_prev1 = off; off = align16(off + sched_n1_max * 16u);
    p.smem_f1 = off; off = align16(off + sched_n1_max * 16u);
    p.smem_x2 = off; off = align16(off + sched_n2_max * 16u);
    for (int l = 0; l < kDevLevels; ++l)
        for (int k = 0; k < kKinds; ++k) {
            DevTable& t = p.tab[l][k];
            std::memset(&t, 0, sizeof(t));
            if (l >= sched.levels) {
                static const uint32_t zero[2] = {0, 0};
                (void)zero;
                continue;
            }
            const Table& h = sched.tables[l][k];
            t.block_begin = dupload(owned, h.block_begin, stream);
            t.stage_offsets = dupload(owned, h.stage_offsets, stream);
            t.ab = dupload(owned, h.ab, stream);
            t.cd = k == 1 ? dupload(owned, h.cd, stream) : nullptr;
            t.rest = dupload(owned, h.rest, stream);
            t.comp = dupload(owned, h.comp, stream);
            t.stages = h.stages;
            t.max_count = h.max_block_count;
            const uint32_t bytes = h.max_block_count * 4u;
            t.smem_ab = off; off = align16(off + bytes);
            if (k == 1) { t.smem_cd = off; off = align16(off + bytes); }
            t.smem_rest = off; off = align16(off + bytes);
            t.smem_comp = off; off = align16(off + bytes);
            t.smem_lambda = off; off = align16(off + bytes);
        }
    p.smem_total = off;
    for (int l = 1; l < sched.levels; ++l) {
        p.patch_begin[l] = dupload(owned, sched.patch_begin[l], stream);
        p.patch_slots[l] = dupload(owned, sched.patch_slots[l], stream);
    }
    for (int k = 0; k < kKinds; ++k) {
        const GlobalTable& h = sched.global[k];
        DevGlobal& g = p.glob[k];
        g.colour_offsets = dupload(owned, h.colour_offsets, stream);
        g.a = dupload(owned, h.a, stream);
        g.b = dupload(owned, h.b, stream);
        g.c = k == 1 ? dupload(owned, h.c, stream) : nullptr;
        g.d = k == 1 ? dupload(owned, h.d, stream) : nullptr;
        g.rest = dupload(owned, h.rest, stream);
        g.comp = dupload(owned, h.comp, stream);
        g.count = static_cast<uint32_t>(h.a.size());
        g.lambda = dalloc<float>(owned, g.count);
        g.colours = h.colour_offsets.empty() ? 0 : static_cast<int>(h.colour_offsets.size()) - 1;
    }
    p.iface_begin = dupload(owned, sched.iface_begin, stream);
    p.iface_local = dupload(owned, sched.iface_local, stream);
    p.seam_offsets = dupload(owned, sched.seam_stage_offsets, stream);
    p.seam_stages = sched.seam_stage_offsets.empty() ? 0 : static_cast<int>(sched.seam_stage_offsets.size()) - 1;
    p.seam_a = dupload(owned, sched.seam_a, stream);
    p.seam_b = dupload(owned, sched.seam_b, stream);
}

void StructureImpl::finish_build(const swb_solver_options& opt, const cudaDeviceProp& prop) {
    StepParams& p = params;
    const size_t smem_limit_ = dynamic_smem_limit(prop);
    // diagnostics arrays (definition order of distance-like constraints)
    {
        std::vector<uint32_t> a(def.constraints.size()), b(def.constraints.size());
        std::vector<float> rest(def.constraints.size());
        std::vector<uint8_t> kind(def.constraints.size());
        for (size_t i = 0; i < def.constraints.size(); ++i) {
            a[i] = slot_of_node[def.constraints[i].first_node];
            b[i] = slot_of_node[def.constraints[i].second_node];
            rest[i] = static_cast<float>(def.constraints[i].rest_length);
            kind[i] = static_cast<uint8_t>(def.constraints[i].kind);
        }
        d_diag_a = dupload(owned, a, stream);
        d_diag_b = dupload(owned, b, stream);
        d_diag_rest = dupload(owned, rest, stream);
        d_diag_kind = dupload(owned, kind, stream);
        d_diag_partials = dalloc<double>(owned, static_cast<size_t>(kDiagBlocks) * kDiagFields);
        // membrane records: corner slots and record index (constants and
        // residual are per record)
        if (cluster_mode && !def.membranes.empty()) {
            const ClusterKind& K = csched.kinds[2];
            std::vector<uint4> mem(K.def_index.size());
            for (size_t r = 0; r < mem.size(); ++r) {
                const swb_triangle_def& t = def.triangles[def.membranes[K.def_index[r]].triangle];
                mem[r] = make_uint4(static_cast<uint32_t>(slot_of_node[t.nodes[0]]),
                                    static_cast<uint32_t>(slot_of_node[t.nodes[1]]),
                                    static_cast<uint32_t>(slot_of_node[t.nodes[2]]), static_cast<uint32_t>(r));
            }
            d_diag_mem = dupload(owned, mem, stream);
        }
    }

    // suspension
    p.susp_block = -1;
    DevPayloadDef pdef{};
    DevPayloadState pstate{};
    if (def.has_suspension) {
        const swb_suspension_def& s = def.suspension;
        p.susp_block = susp_owner;
        const uint32_t sbase = susp_base;
        pdef.mass = static_cast<float>(s.pilot_mass);
        pdef.com_local = make_float3(s.pilot_com_local.x, s.pilot_com_local.y, s.pilot_com_local.z);
        pdef.inertia = make_float3(s.pilot_principal_inertia.x, s.pilot_principal_inertia.y,
                                   s.pilot_principal_inertia.z);
        std::vector<size_t> horder(def.harness.size()), sorder(def.segments.size());
        std::iota(horder.begin(), horder.end(), 0);
        std::iota(sorder.begin(), sorder.end(), 0);
        std::stable_sort(horder.begin(), horder.end(), [&](size_t x, size_t y) {
            return id_string_less(def.harness[x].stable_id, def.harness[y].stable_id);
        });
        std::stable_sort(sorder.begin(), sorder.end(), [&](size_t x, size_t y) {
            return id_string_less(def.segments[x].stable_id, def.segments[y].stable_id);
        });
        segment_order = sorder;
        pdef.hang_points = static_cast<int>(horder.size());
        for (size_t i = 0; i < horder.size(); ++i) {
            const auto& h = def.harness[horder[i]].local_position;
            pdef.hang_local[i] = make_float3(h.x, h.y, h.z);
        }
        pdef.segments = static_cast<int>(sorder.size());
        for (size_t k = 0; k < sorder.size(); ++k) {
            const swb_suspension_segment& g = def.segments[sorder[k]];
            int node[2] = {-1, -1}, point[2] = {-1, -1};
            const swb_suspension_endpoint* ends[2] = {&g.from, &g.to};
            for (int e = 0; e < 2; ++e) {
                if (ends[e]->kind == SWB_ENDPOINT_SURFACE_ATTACHMENT) {
                    for (const auto& a : def.attachments)
                        if (a.stable_id == ends[e]->stable_id)
                            node[e] = static_cast<int>(slot_of_node[a.node] - sbase);
                } else if (ends[e]->kind == SWB_ENDPOINT_JUNCTION) {
                    for (const auto& j : def.junctions)
                        if (j.stable_id == ends[e]->stable_id)
                            node[e] = static_cast<int>(slot_of_node[j.node] - sbase);
                } else if (ends[e]->kind == SWB_ENDPOINT_PILOT_HARNESS) {
                    for (size_t i = 0; i < horder.size(); ++i)
                        if (def.harness[horder[i]].stable_id == ends[e]->stable_id) point[e] = static_cast<int>(i);
                } else {
                    raise(SWB_INVALID_ARGUMENT, "Unknown structure suspension endpoint kind");
                }
                if (node[e] < 0 && point[e] < 0)
                    raise(SWB_SUSPENSION_ERROR, "suspension segment endpoint does not resolve");
            }
            if (ends[0]->kind == SWB_ENDPOINT_PILOT_HARNESS || ends[1]->kind == SWB_ENDPOINT_SURFACE_ATTACHMENT)
                raise(SWB_SUSPENSION_ERROR, "invalid directed endpoint kinds");
            pdef.from_node[k] = node[0]; pdef.to_node[k] = node[1];
            pdef.from_point[k] = point[0]; pdef.to_point[k] = point[1];
            pdef.rest[k] = static_cast<float>(g.rest_length);
            pdef.stiffness[k] = static_cast<float>(g.axial_stiffness);
            pdef.damping[k] = static_cast<float>(g.axial_damping);
        }
        pdef.max_residual = static_cast<float>(s.maximum_line_residual);
        pdef.min_length = static_cast<float>(s.minimum_line_length);
        // canonical initial orientation (suspension.cpp:771)
        const swb_quat& q0 = s.pilot_initial_body_to_world;
        double n = std::sqrt(q0.w * q0.w + q0.x * q0.x + q0.y * q0.y + q0.z * q0.z);
        double qw = q0.w / n, qx = q0.x / n, qy = q0.y / n, qz = q0.z / n;
        if (qw < 0 || (qw == 0 && (qx < 0 || (qx == 0 && (qy < 0 || (qy == 0 && qz < 0)))))) {
            qw = -qw; qx = -qx; qy = -qy; qz = -qz;
        }
        pstate.com = make_float3(s.pilot_initial_com_world.x - origin0[0], s.pilot_initial_com_world.y - origin0[1],
                                 s.pilot_initial_com_world.z - origin0[2]);
        pstate.q = make_float4(qw, qx, qy, qz);
        pstate.v = make_float3(s.pilot_initial_linear_velocity.x, s.pilot_initial_linear_velocity.y,
                               s.pilot_initial_linear_velocity.z);
        pstate.w = make_float3(s.pilot_initial_angular_velocity.x, s.pilot_initial_angular_velocity.y,
                               s.pilot_initial_angular_velocity.z);
    }
    payload_def_host = pdef;
    d_payload_def = dupload(owned, std::vector<DevPayloadDef>{pdef}, stream);
    for (int i = 0; i < 3; ++i) {
        d_payload[i] = dupload(owned, std::vector<DevPayloadState>{pstate}, stream);
        d_origin[i] = dupload(owned, std::vector<double>{origin0[0], origin0[1], origin0[2]}, stream);
    }
    d_control = dalloc<Control>(owned, 1);
    cuda_check(cudaMemsetAsync(d_control, 0, sizeof(Control), stream), "memset");
    p.payload_def = d_payload_def;
    p.recentre = def.has_suspension ? 1 : 0;
    p.barrier.count = &d_control->count;
    p.barrier.generation = &d_control->generation;
    p.barrier.status = d_control->status;
    p.barrier.blocks = static_cast<unsigned>(G);
    p.status = d_control->status;
    p.shift_out = &d_control->shift;
    const long long budget = opt.sync_budget_cycles > 0 ? opt.sync_budget_cycles : 4000000000LL;
    p.barrier.budget = budget;
    // The staging wait keeps its own ~2 s bound whatever the barrier budget,
    // so a CTA never leaves with bulk copies still in flight.
    p.copy_budget = 4000000000LL;

    if (cluster_mode) {
        if (def.has_contact) setup_contact(opt);
        upload_instances();
        cparams.copy_budget = 4000000000LL;
        // The attribute is a per-kernel limit shared by every structure in
        // the process: it is raised to the device limit, never set to this
        // structure's need (a smaller structure built later would otherwise
        // lower it below what an earlier one launches with).
        const auto kernel = step_kernel();
        cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(smem_limit_)),
                   "shared memory request of the cluster schedule");
        if (G > 8)
            cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1),
                       "non-portable cluster size");
        cudaLaunchConfig_t cfg{};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = static_cast<unsigned>(G);
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(G);
        cfg.blockDim = dim3(threads);
        cfg.dynamicSmemBytes = cluster_smem;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int clusters = 0;
        cuda_check(cudaOccupancyMaxActiveClusters(&clusters, kernel, &cfg), "cluster occupancy");
        if (clusters < 1) raise(SWB_UNSUPPORTED, "a cluster of " + std::to_string(G) + " CTAs cannot be scheduled");
    } else {
        // launch feasibility of the cooperative grid
        if (p.smem_total > smem_limit_)
            raise(SWB_UNSUPPORTED, "shared memory request (mesh patch too large for the block count)");
        cuda_check(cudaFuncSetAttribute(dev::xpbd_step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(smem_limit_)),
                   "shared memory limit of the grid schedule");
        int per_sm = 0;
        cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::xpbd_step_kernel, threads,
                                                                 p.smem_total),
                   "occupancy");
        if (per_sm * sm_count < G)
            raise(SWB_UNSUPPORTED, "persistent grid of " + std::to_string(G) + " CTAs is not co-resident (" +
                                       std::to_string(per_sm) + " per SM)");
    }
    cuda_check(cudaStreamSynchronize(stream), "upload");
}

void StructureImpl::upload_pressure() {
    const uint64_t N = def.nodes.size();
    std::vector<uint4> tri(def.triangles.size());
    std::vector<uint32_t> off(N + 1, 0), list;
    for (size_t t = 0; t < def.triangles.size(); ++t) {
        const auto& tr = def.triangles[t];
        const float pr = static_cast<float>(pressure[t]);
        tri[t] = make_uint4(slot_of_node[tr.nodes[0]], slot_of_node[tr.nodes[1]],
                            slot_of_node[tr.nodes[2]], std::bit_cast<uint32_t>(pr));
        if (pressure[t] == 0.0) continue;
        for (int k = 0; k < 3; ++k) ++off[slot_of_node[tr.nodes[k]] + 1];
    }
    for (uint64_t s = 0; s < N; ++s) off[s + 1] += off[s];
    list.resize(off[N]);
    std::vector<uint32_t> cur(off.begin(), off.end() - 1);
    for (size_t t = 0; t < def.triangles.size(); ++t) {
        if (pressure[t] == 0.0) continue;
        for (int k = 0; k < 3; ++k) list[cur[slot_of_node[def.triangles[t].nodes[k]]]++] = static_cast<uint32_t>(t);
    }
    // The tables keep their addresses for the structure's lifetime (the
    // cluster instance records and batches hold them): allocated once, with
    // room for every triangle under pressure, then overwritten in stream order.
    if (!d_tri) {
        d_tri = dalloc<uint4>(owned, tri.size());
        d_tri_off = dalloc<uint32_t>(owned, N + 1);
        d_tri_list = dalloc<uint32_t>(owned, 3 * def.triangles.size());
    }
    if (!tri.empty())
        cuda_check(cudaMemcpyAsync(d_tri, tri.data(), tri.size() * sizeof(uint4), cudaMemcpyHostToDevice, stream),
                   "pressure upload");
    cuda_check(cudaMemcpyAsync(d_tri_off, off.data(), off.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream),
               "pressure upload");
    if (!list.empty())
        cuda_check(cudaMemcpyAsync(d_tri_list, list.data(), list.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                   stream),
                   "pressure upload");
    cuda_check(cudaStreamSynchronize(stream), "pressure upload");
    params.tri = d_tri;
    params.tri_offsets = d_tri_off;
    params.tri_list = d_tri_list;
    pressure_dirty = false;
}

void StructureImpl::upload_forces() {
    const uint64_t N = def.nodes.size();
    for (uint64_t n = 0; n < N; ++n) {
        const swb_vec3& f = pending[n];
        h_force[slot_of_node[n]] =
            make_float4(static_cast<float>(f.x), static_cast<float>(f.y), static_cast<float>(f.z), 0.0f);
    }
    cuda_check(cudaMemcpyAsync(d_force, h_force, N * sizeof(float4), cudaMemcpyHostToDevice, stream), "force upload");
    forces_dirty = false;
}

void StructureImpl::validate_settings(const swb_step_settings& st) const {
    auto fin = [](const swb_vec3& v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); };
    // SoftBody::step / stepCoupled (soft_body.cpp:982-1003, 1024-1050)
    if (!(st.time_step > 0.0) || !std::isfinite(st.time_step) || st.substeps <= 0 || st.constraint_iterations < 0 ||
        st.cable_sweep_pairs < 0 || st.velocity_damping < 0.0 || !std::isfinite(st.velocity_damping) ||
        !fin(st.gravity) || !fin(st.damping_reference_velocity) ||
        (def.has_suspension && st.constraint_iterations == 0))
        raise(SWB_INVALID_ARGUMENT, def.has_suspension ? "Invalid coupled SoftBody step settings"
                                                        : "Invalid SoftBody step settings");
    if (def.has_suspension && st.constraint_iterations != def.suspension.solver_iterations)
        raise(SWB_INVALID_ARGUMENT,
              "Coupled structural iterations must equal the registered suspension lineIterations contract");
    if (st.cable_sweep_pairs != 0 && !cluster_mode)
        raise(SWB_UNSUPPORTED, "load-path cable sweep pairs need the cluster schedule (the mesh does not fit one)");
}

// Every device table the kernel dereferences must exist before a launch.
void check_params(const StepParams& p) {
    bool ok = p.pos_in && p.vel_in && p.pos_out && p.vel_out && p.prev_out && p.force && p.tri_offsets &&
              p.tri_list && p.tri && p.l1_begin && p.iface_begin && p.iface_local && p.seam_offsets && p.seam_a &&
              p.seam_b && p.payload_def && p.payload_in && p.payload_out && p.shift_out && p.origin_in &&
              p.origin_out && p.status && p.barrier.count && p.barrier.generation && p.barrier.status;
    for (int k = 0; k < 2; ++k)
        ok = ok && p.glob[k].colour_offsets && p.glob[k].a && p.glob[k].b && p.glob[k].rest && p.glob[k].comp &&
             p.glob[k].lambda && (k == 0 || (p.glob[k].c && p.glob[k].d));
    for (int l = 0; l < p.levels; ++l) {
        for (int k = 0; k < 2; ++k) {
            const DevTable& t = p.tab[l][k];
            ok = ok && t.block_begin && t.stage_offsets && t.ab && t.rest && t.comp && (k == 0 || t.cd);
        }
        if (l > 0) ok = ok && p.patch_begin[l] && p.patch_slots[l];
    }
    if (!ok) raise(SWB_CUDA_ERROR, "internal error: a device table is missing; launch refused");
}

// `first`: the first substep of a step clears the status words; later
// substeps keep them, so a failure in any substep fails the whole step (and
// a timed-out grid barrier makes the later substeps' barriers return at
// once).
void StructureImpl::launch_substep(const swb_step_settings& st, int in, int out, bool first) {
    const double dt = st.time_step / st.substeps;
    if (cluster_mode) {
        ClusterParams cp = cparams;
        cp.instances = d_instances + in * 3 + out;
        cp.ctas = G;
        cp.dt = static_cast<float>(dt);
        cp.dt64 = dt;
        cp.inv_dt = static_cast<float>(1.0 / dt);
        cp.inv_dt2 = static_cast<float>(1.0 / (dt * dt));
        cp.damping = static_cast<float>(std::exp(-st.velocity_damping * dt));
        cp.damping_loss = static_cast<float>(-std::expm1(-st.velocity_damping * dt));
        cp.gravity = make_float3(st.gravity.x, st.gravity.y, st.gravity.z);
        cp.ref_velocity = make_float3(st.damping_reference_velocity.x, st.damping_reference_velocity.y,
                                      st.damping_reference_velocity.z);
        cp.iterations = st.constraint_iterations;
        cp.cable_pairs = st.cable_sweep_pairs;
        if (!cp.instances || in == out) raise(SWB_CUDA_ERROR, "internal error: cluster instance table");
        if (first) cuda_check(cudaMemsetAsync(d_control, 0, offsetof(Control, shift), stream), "control reset");
        // contact: the helper clusters join the detection phases; the launch
        // is cooperative so that every cluster is resident at once (a grid
        // barrier spans them)
        cp.helper_clusters = contact_helpers;
        cp.grid = params.barrier;
        cudaLaunchConfig_t cfg{};
        cudaLaunchAttribute attr[2];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = static_cast<unsigned>(G);
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        attr[1].id = cudaLaunchAttributeCooperative;
        attr[1].val.cooperative = 1;
        cfg.gridDim = dim3(G * (1 + contact_helpers));
        cfg.blockDim = dim3(threads);
        cfg.dynamicSmemBytes = cluster_smem;
        cfg.stream = stream;
        cfg.attrs = attr;
        cfg.numAttrs = contact_helpers > 0 ? 2 : 1;
        cudaError_t rc = cudaLaunchKernelEx(&cfg, step_kernel(), cp);
        if (rc != cudaSuccess && contact_helpers > 0) {
            // no cooperative launch of this many clusters: the structure's
            // cluster alone from now on (the results are the same)
            (void)cudaGetLastError();
            contact_helpers = 0;
            cp.helper_clusters = 0;
            cfg.gridDim = dim3(G);
            cfg.numAttrs = 1;
            rc = cudaLaunchKernelEx(&cfg, step_kernel(), cp);
        }
        cuda_check(rc, "cudaLaunchKernelEx (cluster)");
        return;
    }
    StepParams p = params;
    p.pos_in = d_pos[in]; p.vel_in = d_vel[in];
    p.pos_out = d_pos[out]; p.vel_out = d_vel[out]; p.prev_out = d_prev[out];
    p.force = d_force;
    p.payload_in = d_payload[in]; p.payload_out = d_payload[out];
    p.origin_in = d_origin[in]; p.origin_out = d_origin[out];
    p.dt = static_cast<float>(dt);
    p.inv_dt = static_cast<float>(1.0 / dt);
    p.inv_dt2 = static_cast<float>(1.0 / (dt * dt));
    p.damping = static_cast<float>(std::exp(-st.velocity_damping * dt));
    p.damping_loss = static_cast<float>(-std::expm1(-st.velocity_damping * dt));
    p.gravity = make_float3(st.gravity.x, st.gravity.y, st.gravity.z);
    p.ref_velocity = make_float3(st.damping_reference_velocity.x, st.damping_reference_velocity.y,
                                 st.damping_reference_velocity.z);
    p.iterations = st.constraint_iterations;
    check_params(p);
    if (first) cuda_check(cudaMemsetAsync(d_control, 0, offsetof(Control, shift), stream), "control reset");
    void* args[] = {&p};
    cuda_check(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(dev::xpbd_step_kernel), dim3(G), dim3(threads),
                                           args, p.smem_total, stream),
               "cudaLaunchCooperativeKernel");
}

size_t dynamic_smem_limit(const cudaDeviceProp& prop) {
    size_t reserve = 2048;
    for (const void* k : {reinterpret_cast<const void*>(dev::xpbd_cluster_kernel),
                          reinterpret_cast<const void*>(dev::xpbd_cluster_packed_kernel),
                          reinterpret_cast<const void*>(dev::xpbd_cluster_membrane_kernel),
                          reinterpret_cast<const void*>(dev::xpbd_cluster_packed_membrane_kernel),
                          reinterpret_cast<const void*>(dev::xpbd_cluster_contact_kernel),
                          reinterpret_cast<const void*>(dev::xpbd_cluster_contact_membrane_kernel),
                          reinterpret_cast<const void*>(dev::xpbd_cluster_tape_kernel),
                          reinterpret_cast<const void*>(dev::xpbd_cluster_adjoint_kernel),
                          reinterpret_cast<const void*>(dev::xpbd_cluster_adjoint_kernel_narrow),
                          reinterpret_cast<const void*>(dev::xpbd_cluster_adjoint_lines_kernel),
                          reinterpret_cast<const void*>(dev::xpbd_cluster_adjoint_lines_kernel_narrow),
                          reinterpret_cast<const void*>(dev::xpbd_step_kernel)}) {
        cudaFuncAttributes a{};
        if (cudaFuncGetAttributes(&a, k) == cudaSuccess) reserve = std::max(reserve, a.sharedSizeBytes + 256);
    }
    return prop.sharedMemPerBlockOptin > reserve ? prop.sharedMemPerBlockOptin - reserve : 0;
}

cudaError_t packed_kernel_limits(int max_dynamic_smem, bool non_portable_cluster) {
    cudaError_t rc = cudaSuccess;
    for (auto kernel : {dev::xpbd_cluster_packed_kernel, dev::xpbd_cluster_packed_membrane_kernel}) {
        if (rc == cudaSuccess)
            rc = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dynamic_smem);
        if (rc == cudaSuccess && non_portable_cluster)
            rc = cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    }
    return rc;
}

cudaError_t packed_kernel_occupancy(int* clusters, const cudaLaunchConfig_t& cfg, bool membranes) {
    return cudaOccupancyMaxActiveClusters(
        clusters, membranes ? dev::xpbd_cluster_packed_membrane_kernel : dev::xpbd_cluster_packed_kernel, &cfg);
}

cudaError_t packed_kernel_launch(const cudaLaunchConfig_t& cfg, const ClusterParams& params, bool membranes) {
    return cudaLaunchKernelEx(
        &cfg, membranes ? dev::xpbd_cluster_packed_membrane_kernel : dev::xpbd_cluster_packed_kernel, params);
}

cudaError_t plain_cluster_launch(const cudaLaunchConfig_t& cfg, const ClusterParams& params) {
    return cudaLaunchKernelEx(&cfg, dev::xpbd_cluster_kernel, params);
}

cudaError_t tape_kernel_limits(int max_dynamic_smem, bool non_portable_cluster) {
    cudaError_t rc = cudaFuncSetAttribute(dev::xpbd_cluster_tape_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, max_dynamic_smem);
    if (rc == cudaSuccess && non_portable_cluster)
        rc = cudaFuncSetAttribute(dev::xpbd_cluster_tape_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    return rc;
}

cudaError_t tape_kernel_launch(const cudaLaunchConfig_t& cfg, const ClusterParams& params) {
    return cudaLaunchKernelEx(&cfg, dev::xpbd_cluster_tape_kernel, params);
}

cudaError_t adjoint_kernel_limits(int max_dynamic_smem, bool non_portable_cluster) {
    cudaError_t rc = cudaSuccess;
    for (auto kernel : {dev::xpbd_cluster_adjoint_kernel, dev::xpbd_cluster_adjoint_kernel_narrow,
                        dev::xpbd_cluster_adjoint_lines_kernel, dev::xpbd_cluster_adjoint_lines_kernel_narrow}) {
        if (rc == cudaSuccess)
            rc = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dynamic_smem);
        if (rc == cudaSuccess && non_portable_cluster)
            rc = cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    }
    return rc;
}

// Blocks of up to 512 threads take the instantiation with that launch bound
// (registers for the tape prefetch); tapes with line-line contact (their
// line arrays are allocated only then) the instantiation that reverses it.
cudaError_t adjoint_kernel_launch(const cudaLaunchConfig_t& cfg, const AdjointParams& params) {
    const bool narrow = cfg.blockDim.x <= 512, lines = params.tape.line_count != nullptr;
    auto kernel = lines ? (narrow ? dev::xpbd_cluster_adjoint_lines_kernel_narrow : dev::xpbd_cluster_adjoint_lines_kernel)
                        : (narrow ? dev::xpbd_cluster_adjoint_kernel_narrow : dev::xpbd_cluster_adjoint_kernel);
    return cudaLaunchKernelEx(&cfg, kernel, params);
}

swb_status decode_status(const int status[2], std::string& message) {
    if (status[0] == 0) return SWB_OK;
    if (status[0] & dev::kStatusSyncTimeout) {
        message = "device-wide barrier timed out";
        return SWB_SYNC_TIMEOUT;
    }
    if (status[0] & dev::kStatusCopyTimeout) {
        message = "shared-memory staging timed out";
        return SWB_SYNC_TIMEOUT;
    }
    if (status[0] & dev::kStatusContact) {
        static const char* what[] = {
            "contact failure",
            "Contact CCD could not certify a supported feature",
            "Contact endpoint geometry is not certifiable",
            "Contact normal is not finite/unit",
            "Penetrating contact has no movable/compliant response",
            "Non-finite contact projection",
            "Non-finite solved contact geometry",
            "Final contact geometry could not be certified",
            "Final contact closest geometry is not certifiable",
            "Final contact geometry is non-finite",
            "Final contact penetration exceeds the certified gate",
            "Applied contact impulse lost its supported feature",
            "Cleared contact final geometry is not certifiable",
            "Cleared contact failed final geometry certification",
            "Non-finite/positive contact friction work",
            "Contact broadphase input failed: positions must be finite",
            "contact candidates exceed the device list (1,048,576 per phase)",
            "contact features exceed the device multiplier table",
            "contact records exceed the device record book",
            "line-line contact pairs exceed the device list",
            "line-line contact candidates exceed the rollout's tape"};
        message = std::string("ContactStepError: ") + what[std::clamp(status[1], 0, 20)];
        return SWB_CONTACT_ERROR;
    }
    if (status[0] & dev::kStatusMembrane) {
        message = "membrane system is singular or its right-hand side is not finite";
        return SWB_INVALID_ARGUMENT;
    }
    if (status[0] & dev::kStatusSuspension) {
        static const char* what[] = {"suspension failure", "line geometry is non-finite or scale-degenerate",
                                     "invalid unilateral line projection input", "zero generalized effective mass",
                                     "payload trial state is non-finite or unnormalized",
                                     "maximum line residual exceeds configured bound", "invalid payload orientation",
                                     "payload integration produced non-finite state",
                                     "line trial length is non-finite",
                                     "payload velocity reconstruction or line damping failed"};
        message = std::string("SuspensionError: ") + what[std::clamp(status[1] & 0xff, 0, 9)];
        return SWB_SUSPENSION_ERROR;
    }
    message = "trial step produced a non-finite state";
    return SWB_NON_FINITE;
}

swb_status StructureImpl::read_status(std::string& message) {
    Control c{};
    cuda_check(cudaMemcpyAsync(&c, d_control, sizeof(Control), cudaMemcpyDeviceToHost, stream), "status");
    cuda_check(cudaStreamSynchronize(stream), "step");
    last_status[0] = c.status[0];
    last_status[1] = c.status[1];
    return decode_status(c.status, message);
}

// The reference's exception details for a failed step: the phase and entity
// of a SuspensionError (suspension.cpp fail sites, one per device detail
// code) and the feature key of a ContactStepError.  The contact message is
// that of the failing feature first in key order.
swb_error_detail StructureImpl::failure_detail(swb_status status, std::string& message) {
    swb_error_detail d{};
    d.status = static_cast<uint32_t>(status);
    if (status == SWB_SUSPENSION_ERROR) {
        struct Site { uint32_t phase; const char* entity; };
        static const Site sites[] = {
            {SWB_PHASE_CERTIFICATION, "unknown"},          {SWB_PHASE_LINE_SOLVE, nullptr},
            {SWB_PHASE_LINE_SOLVE, "line-projection"},     {SWB_PHASE_LINE_SOLVE, "effective-mass"},
            {SWB_PHASE_CERTIFICATION, "payload"},          {SWB_PHASE_CERTIFICATION, "line-residual"},
            {SWB_PHASE_LINE_SOLVE, "payload"},             {SWB_PHASE_PREDICTION, "payload-step"},
            {SWB_PHASE_CERTIFICATION, nullptr},            {SWB_PHASE_CERTIFICATION, "payload"}};
        const int code = std::clamp(last_status[1] & 0xff, 0, 9);
        const int segment = (last_status[1] >> 8) - 1;
        d.suspension_phase = sites[code].phase;
        std::string entity = sites[code].entity ? sites[code].entity : "segment";
        if (!sites[code].entity && segment >= 0 && static_cast<size_t>(segment) < segment_order.size())
            entity = "segment:" + std::to_string(def.segments[segment_order[segment]].stable_id);
        std::snprintf(d.suspension_entity, sizeof d.suspension_entity, "%s", entity.c_str());
    } else if (status == SWB_CONTACT_ERROR && d_contact) {
        unsigned long long packed = ~0ull;
        cuda_check(cudaMemcpy(&packed, contact_host.fail, sizeof packed, cudaMemcpyDeviceToHost), "read");
        if (packed != ~0ull) {
            const uint64_t row = packed >> 37, col = (packed >> 5) & 0xffffffffull;
            const int detail = static_cast<int>(packed & 31u);
            d.has_contact_key = 1;
            d.contact_key = contact_key_of(contact_surface, row, col);
            const int raw[2] = {dev::kStatusContact, detail};
            decode_status(raw, message);
        }
    }
    return d;
}

void StructureImpl::commit(int new_cur, int steps, const swb_step_settings& st) {
    cur = new_cur;
    swb_vec3 applied{0, 0, 0};
    for (auto& f : pending) {
        applied.x += f.x; applied.y += f.y; applied.z += f.z;
        if (f.x != 0.0 || f.y != 0.0 || f.z != 0.0) forces_dirty = true;
        f = swb_vec3{0, 0, 0};
    }
    last_applied = applied;
    accepted += static_cast<uint64_t>(steps);
    time += st.time_step * steps;
    last_dt = st.time_step / st.substeps;
}

swb_status StructureImpl::step(const swb_step_settings& st, int steps, swb_diagnostics* out) {
    validate_settings(st);
    if (steps < 1) raise(SWB_INVALID_ARGUMENT, "steps must be positive");
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    if (pressure_dirty) upload_pressure();
    if (forces_dirty && !device_forces) upload_forces();
    const int start = cur;
    const int total = steps * st.substeps;
    // Transaction: substeps ping-pong between buffers `start` and `other`;
    // with more than one substep the committed state is first copied to the
    // third buffer so a failure can restore it.
    int backup = -1;
    int a = start, b = (start + 1) % 3;
    if (b == start) b = (start + 2) % 3;
    if (total > 1) {
        backup = 3 - a - b;
        copy_state(a, backup);
    }
    if (d_contact) {
        contact_table_save<<<kDiagBlocks, 256, 0, stream>>>(d_contact, d_table_commit, d_meta_commit);
        cuda_check(cudaGetLastError(), "contact_table_save");
    }
    cuda_check(cudaEventRecord(ev0, stream), "event");
    for (int k = 0; k < total; ++k) {
        launch_substep(st, a, b, k == 0);
        std::swap(a, b);
    }
    cuda_check(cudaEventRecord(ev1, stream), "event");
    std::string message;
    const swb_status status = read_status(message);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    last_ms = ms;
    if (status != SWB_OK) {
        if (backup >= 0) copy_state(backup, start);
        if (d_contact) {
            contact_table_restore<<<kDiagBlocks, 256, 0, stream>>>(d_contact, d_table_commit, d_meta_commit);
            cuda_check(cudaGetLastError(), "contact_table_restore");
        }
        if (backup >= 0 || d_contact) cuda_check(cudaStreamSynchronize(stream), "restore");
        cur = start;
        if (status == SWB_SUSPENSION_ERROR || status == SWB_CONTACT_ERROR) {
            const swb_error_detail detail = failure_detail(status, message);
            throw Error(status, message, detail);
        }
        raise(status, message);
    }
    commit(a, steps, st);
    if (out) diagnostics(out);
    return SWB_OK;
}

void StructureImpl::copy_state(int from, int to) {
    const size_t N = def.nodes.size();
    cuda_check(cudaMemcpyAsync(d_pos[to], d_pos[from], N * sizeof(float4), cudaMemcpyDeviceToDevice, stream), "copy");
    cuda_check(cudaMemcpyAsync(d_vel[to], d_vel[from], N * sizeof(float4), cudaMemcpyDeviceToDevice, stream), "copy");
    cuda_check(cudaMemcpyAsync(d_prev[to], d_prev[from], N * sizeof(float4), cudaMemcpyDeviceToDevice, stream), "copy");
    cuda_check(cudaMemcpyAsync(d_payload[to], d_payload[from], sizeof(DevPayloadState), cudaMemcpyDeviceToDevice,
                               stream), "copy");
    cuda_check(cudaMemcpyAsync(d_origin[to], d_origin[from], 3 * sizeof(double), cudaMemcpyDeviceToDevice, stream),
               "copy");
}

void StructureImpl::fetch(std::vector<float4>& pos, std::vector<float4>& prev, std::vector<float4>& vel,
                          DevPayloadState& pay, double origin[3]) const {
    const size_t N = def.nodes.size();
    pos.resize(N); prev.resize(N); vel.resize(N);
    cuda_check(cudaMemcpyAsync(pos.data(), d_pos[cur], N * sizeof(float4), cudaMemcpyDeviceToHost, stream), "read");
    cuda_check(cudaMemcpyAsync(prev.data(), d_prev[cur], N * sizeof(float4), cudaMemcpyDeviceToHost, stream), "read");
    cuda_check(cudaMemcpyAsync(vel.data(), d_vel[cur], N * sizeof(float4), cudaMemcpyDeviceToHost, stream), "read");
    cuda_check(cudaMemcpyAsync(&pay, d_payload[cur], sizeof(pay), cudaMemcpyDeviceToHost, stream), "read");
    cuda_check(cudaMemcpyAsync(origin, d_origin[cur], 3 * sizeof(double), cudaMemcpyDeviceToHost, stream), "read");
    cuda_check(cudaStreamSynchronize(stream), "read");
}

void StructureImpl::diagnostics(swb_diagnostics* o) const {
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    const uint32_t N = static_cast<uint32_t>(def.nodes.size());
    const uint32_t M = static_cast<uint32_t>(def.constraints.size());
    const uint32_t NM = d_diag_mem ? static_cast<uint32_t>(def.membranes.size()) : 0u;
    diagnostics_kernel<<<kDiagBlocks, 256, 0, stream>>>(d_pos[cur], d_prev[cur], d_vel[cur], N, d_diag_a, d_diag_b,
                                                         d_diag_rest, d_diag_kind, M, d_diag_mem,
                                                         cluster_base.kind[2].aux, d_mres[cur], NM, d_diag_partials);
    cuda_check(cudaGetLastError(), "diagnostics");
    std::vector<double> part(static_cast<size_t>(kDiagBlocks) * kDiagFields);
    DevPayloadState pay{};
    double origin[3];
    cuda_check(cudaMemcpyAsync(part.data(), d_diag_partials, part.size() * sizeof(double), cudaMemcpyDeviceToHost,
                               stream), "read");
    cuda_check(cudaMemcpyAsync(&pay, d_payload[cur], sizeof(pay), cudaMemcpyDeviceToHost, stream), "read");
    cuda_check(cudaMemcpyAsync(origin, d_origin[cur], sizeof(origin), cudaMemcpyDeviceToHost, stream), "read");
    cuda_check(cudaStreamSynchronize(stream), "diagnostics");
    double acc[14] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0};
    for (int b = 0; b < kDiagBlocks; ++b) {
        const double* q = &part[static_cast<size_t>(b) * kDiagFields];
        for (int f = 0; f < 9; ++f) acc[f] += q[f];
        acc[9] = std::min(acc[9], q[9]);
        for (int f = 10; f < 14; ++f) acc[f] = std::max(acc[f], q[f]);
    }
    std::memset(o, 0, sizeof(*o));
    o->node_count = N;
    o->dynamic_node_count = static_cast<uint64_t>(acc[0]);
    o->triangle_count = def.triangles.size();
    o->constraint_count = def.constraints.size();
    o->membrane_count = def.membranes.size();
    o->dihedral_count = def.dihedrals.size();
    double mass = acc[1];
    double wx = acc[2] + acc[1] * origin[0], wy = acc[3] + acc[1] * origin[1], wz = acc[4] + acc[1] * origin[2];
    double px = acc[5], py = acc[6], pz = acc[7], ke = acc[8];
    bool finite = acc[9] > 0.5;
    if (mass > 0.0) o->center_of_mass = {wx / mass, wy / mass, wz / mass};
    if (def.has_suspension) {
        const double m = def.suspension.pilot_mass;
        const double cx = pay.com.x + origin[0], cy = pay.com.y + origin[1], cz = pay.com.z + origin[2];
        wx += cx * m; wy += cy * m; wz += cz * m;
        mass += m;
        o->center_of_mass = {wx / mass, wy / mass, wz / mass};
        px += m * pay.v.x; py += m * pay.v.y; pz += m * pay.v.z;
        // 0.5 m |v|^2 + 0.5 w . (I_world w)
        const double qw = pay.q.x, qx = pay.q.y, qy = pay.q.z, qz = pay.q.w;
        const double R[9] = {1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - qw * qz), 2 * (qx * qz + qw * qy),
                             2 * (qx * qy + qw * qz), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - qw * qx),
                             2 * (qx * qz - qw * qy), 2 * (qy * qz + qw * qx), 1 - 2 * (qx * qx + qy * qy)};
        const double I[3] = {def.suspension.pilot_principal_inertia.x, def.suspension.pilot_principal_inertia.y,
                             def.suspension.pilot_principal_inertia.z};
        const double w[3] = {pay.w.x, pay.w.y, pay.w.z};
        double Rtw[3] = {0, 0, 0};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) Rtw[i] += R[j * 3 + i] * w[j];
        double rot = 0.0;
        for (int i = 0; i < 3; ++i) rot += I[i] * Rtw[i] * Rtw[i];
        ke += 0.5 * m * (double(pay.v.x) * pay.v.x + double(pay.v.y) * pay.v.y + double(pay.v.z) * pay.v.z) +
              0.5 * rot;
        o->suspension_segment_count = def.segments.size();
        o->maximum_suspension_residual = pay.max_residual;
        finite = finite && std::isfinite(cx) && std::isfinite(cy) && std::isfinite(cz) && std::isfinite(ke);
    }
    o->total_dynamic_mass = mass;
    o->linear_momentum = {px, py, pz};
    o->kinetic_energy = ke;
    o->maximum_distance_error = acc[10];
    o->maximum_cable_extension = acc[11];
    o->maximum_absolute_membrane_strain = acc[12];
    o->maximum_membrane_residual = acc[13];
    if (def.has_contact) {
        ContactDiagDev cd{};
        cuda_check(cudaMemcpyAsync(&cd, d_cdiag[cur], sizeof(cd), cudaMemcpyDeviceToHost, stream), "read");
        cuda_check(cudaStreamSynchronize(stream), "diagnostics");
        o->contact_pair_count = 1;
        o->active_contact_count = cd.active;
        o->maximum_contact_penetration = cd.max_penetration;
        finite = finite && std::isfinite(cd.max_penetration);
    }
    swb_vec3 pend{0, 0, 0};
    for (const auto& f : pending) {
        pend.x += f.x; pend.y += f.y; pend.z += f.z;
        finite = finite && std::isfinite(f.x) && std::isfinite(f.y) && std::isfinite(f.z);
    }
    o->pending_external_force = pend;
    o->last_applied_external_force = last_applied;
    o->finite = finite && std::isfinite(acc[10]) && std::isfinite(acc[11]) ? 1u : 0u;
}

}  // namespace swb

using namespace swb;

extern "C" {

void swb_default_solver_options(swb_solver_options* out) {
    std::memset(out, 0, sizeof(*out));
}

double StructureImpl::time_trial(const swb_step_settings& st, int warm, int reps) {
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    if (pressure_dirty) upload_pressure();
    if (forces_dirty && !device_forces) upload_forces();
    const int spare = (cur + 1) % 3;
    for (int k = 0; k < warm; ++k) launch_substep(st, cur, spare, true);
    cuda_check(cudaEventRecord(ev0, stream), "event");
    for (int k = 0; k < reps; ++k) launch_substep(st, cur, spare, true);
    cuda_check(cudaEventRecord(ev1, stream), "event");
    cuda_check(cudaStreamSynchronize(stream), "trial");
    float ms = 0.0f;
    cuda_check(cudaEventElapsedTime(&ms, ev0, ev1), "event");
    std::string message;
    const swb_status status = read_status(message);
    // the next step clears the status words before its first substep
    return status == SWB_OK ? ms / reps : std::numeric_limits<double>::infinity();
}

namespace swb {
namespace {

// The autotuner (SWB_OPT_AUTOTUNE): cluster schedules for block sizes
// (the widest stage, 512 and 768 threads), classic and split stages, the
// smallest cluster that fits and the next wider one; each candidate is
// built in full (its schedule verified) and timed over trial substeps from
// the definition's state; the fastest is kept.  Candidates that do not fit
// or fail to build are skipped.  Options the caller sets (block_threads,
// cluster_ctas) are kept fixed.
std::unique_ptr<swb_structure> autotuned(const swb_structure_definition& definition, swb_solver_options opt) {
    opt.flags &= ~static_cast<uint32_t>(SWB_OPT_AUTOTUNE);
    auto first = std::make_unique<swb_structure>();
    first->s.build(definition, &opt);
    StructureImpl& base = first->s;
    if (!base.cluster_mode || base.def.has_contact) return first;
    swb_step_settings st;
    swb_default_step_settings(&st);
    st.substeps = 1;
    st.constraint_iterations = base.def.has_suspension ? base.def.suspension.solver_iterations : 48;
    std::vector<int> ctas = {opt.cluster_ctas > 0 ? opt.cluster_ctas : base.G};
    if (opt.cluster_ctas <= 0 && base.G * 2 <= kClusterMaxCtas) ctas.push_back(base.G * 2);
    std::vector<int> threads = {opt.block_threads};
    if (opt.block_threads <= 0)
        for (int t : {512, 768}) threads.push_back(t);
    swb_autotune_report report{};
    report.iterations = static_cast<uint32_t>(st.constraint_iterations);
    std::unique_ptr<swb_structure> best;
    double best_ms = std::numeric_limits<double>::infinity();
    for (int c : ctas)
        for (uint32_t split : {0u, 1u})
            for (int t : threads) {
                if (report.candidates == SWB_AUTOTUNE_MAX_CANDIDATES) break;
                swb_solver_options o = opt;
                o.cluster_ctas = c;
                o.block_threads = t;
                o.flags = (opt.flags & ~static_cast<uint32_t>(SWB_OPT_SPLIT_STAGES)) |
                          (split ? static_cast<uint32_t>(SWB_OPT_SPLIT_STAGES) : 0u);
                std::unique_ptr<swb_structure> cand;
                if (first && c == base.G && t == opt.block_threads &&
                    split == ((opt.flags & SWB_OPT_SPLIT_STAGES) ? 1u : 0u)) {
                    cand = std::move(first);
                } else {
                    cand = std::make_unique<swb_structure>();
                    try {
                        cand->s.build(definition, &o);
                    } catch (const Error& e) {
                        if (e.status == SWB_UNSUPPORTED || e.status == SWB_INVALID_ARGUMENT) continue;
                        throw;
                    }
                    if (!cand->s.cluster_mode) continue;
                }
                // duplicates (a block size the default already chose)
                bool seen = false;
                for (uint32_t k = 0; k < report.candidates; ++k) {
                    const swb_autotune_candidate& e = report.entries[k];
                    seen = seen || (e.cluster_ctas == cand->s.G && e.block_threads == cand->s.threads &&
                                    e.split_stages == split);
                }
                if (seen) continue;
                const double ms = cand->s.time_trial(st, 2, 5);
                swb_autotune_candidate& e = report.entries[report.candidates];
                e.cluster_ctas = cand->s.G;
                e.block_threads = cand->s.threads;
                e.split_stages = split;
                e.stages_per_iteration = 0;
                for (int k = 0; k < 3; ++k) e.stages_per_iteration += cand->s.csched.kinds[k].stages;
                e.ms_per_substep = ms;
                if (ms < best_ms) {
                    best_ms = ms;
                    best = std::move(cand);
                    report.chosen = report.candidates;
                }
                ++report.candidates;
            }
    if (!best) return first ? std::move(first) : nullptr;
    best->s.tune = report;
    return best;
}

}  // namespace
}  // namespace swb

swb_status swb_structure_create(const swb_structure_definition* definition, const swb_solver_options* options,
                                swb_structure** out) {
    return guarded([&] {
        if (!definition || !out) raise(SWB_INVALID_ARGUMENT, "null argument");
        if (options && (options->flags & SWB_OPT_AUTOTUNE) &&
            !(options->flags & (SWB_OPT_GRID | SWB_OPT_GLOBAL_ONLY))) {
            auto tuned = autotuned(*definition, *options);
            if (!tuned) raise(SWB_UNSUPPORTED, "no autotuner candidate could be built");
            *out = tuned.release();
            return;
        }
        auto impl = std::make_unique<swb_structure>();
        impl->s.build(*definition, options);
        *out = impl.release();
    });
}

swb_status swb_structure_autotune_report(const swb_structure* s, swb_autotune_report* out) {
    return guarded([&] {
        if (!s || !out) raise(SWB_INVALID_ARGUMENT, "null argument");
        *out = s->s.tune;
    });
}

void swb_structure_destroy(swb_structure* s) {
    if (s && !s->borrowed) delete s;
}

uint64_t swb_structure_fingerprint(const swb_structure* s) { return s ? s->s.fingerprint : 0; }
uint64_t swb_structure_accepted_steps(const swb_structure* s) { return s ? s->s.accepted : 0; }
double swb_structure_simulation_time(const swb_structure* s) { return s ? s->s.time : 0.0; }
uint64_t swb_structure_node_count(const swb_structure* s) { return s ? s->s.def.nodes.size() : 0; }
double swb_structure_last_step_ms(const swb_structure* s) { return s ? s->s.last_ms : 0.0; }

swb_status swb_structure_clear_external_forces(swb_structure* s) {
    return guarded([&] {
        if (!s) raise(SWB_INVALID_ARGUMENT, "null structure");
        for (auto& f : s->s.pending) f = swb_vec3{0, 0, 0};
        s->s.forces_dirty = true;
    });
}

swb_status swb_structure_add_external_force(swb_structure* s, uint64_t node, const swb_vec3* force) {
    return guarded([&] {
        if (!s || !force) raise(SWB_INVALID_ARGUMENT, "null argument");
        if (node >= s->s.pending.size()) raise(SWB_OUT_OF_RANGE, "Structure force node is out of range");
        if (!std::isfinite(force->x) || !std::isfinite(force->y) || !std::isfinite(force->z))
            raise(SWB_INVALID_ARGUMENT, "Structure force must be finite");
        s->s.pending[node].x += force->x;
        s->s.pending[node].y += force->y;
        s->s.pending[node].z += force->z;
        s->s.forces_dirty = true;
    });
}

swb_status swb_structure_set_external_forces(swb_structure* s, const swb_vec3* forces, uint64_t count) {
    return guarded([&] {
        if (!s) raise(SWB_INVALID_ARGUMENT, "null structure");
        if (count != s->s.pending.size()) raise(SWB_INVALID_ARGUMENT, "Structure force count must equal the node count");
        if (count && !forces) raise(SWB_INVALID_ARGUMENT, "null forces");
        for (uint64_t i = 0; i < count; ++i)
            if (!std::isfinite(forces[i].x) || !std::isfinite(forces[i].y) || !std::isfinite(forces[i].z))
                raise(SWB_INVALID_ARGUMENT, "Structure forces must be finite");
        std::copy(forces, forces + count, s->s.pending.begin());
        s->s.forces_dirty = true;
    });
}

swb_status swb_structure_set_face_pressure(swb_structure* s, uint64_t triangle, double dp) {
    return guarded([&] {
        if (!s) raise(SWB_INVALID_ARGUMENT, "null structure");
        if (triangle >= s->s.pressure.size()) raise(SWB_OUT_OF_RANGE, "Triangle index is out of range");
        if (!std::isfinite(dp)) raise(SWB_INVALID_ARGUMENT, "Pressure difference must be finite");
        s->s.pressure[triangle] = dp;
        s->s.pressure_dirty = true;
    });
}

swb_status swb_structure_set_line_contact(swb_structure* s, const swb_line_contact* lc) {
    return guarded([&] {
        if (!s) raise(SWB_INVALID_ARGUMENT, "null structure");
        StructureImpl& m = s->s;
        if (!lc || !lc->enabled) {
            if (m.line_contact) {
                m.line_contact = false;
                m.upload_instances();
            }
            return;
        }
        if (!std::isfinite(lc->radius) || !(lc->radius > 0.0) || !std::isfinite(lc->margin) || lc->margin < 0.0)
            raise(SWB_INVALID_ARGUMENT, "line contact radius must be finite and positive, margin finite and >= 0");
        if (!m.cluster_mode) raise(SWB_UNSUPPORTED, "line-line contact needs the cluster schedule");
        if (!m.d_lines) m.setup_line_contact();
        LineContactDev L = m.lines_host;
        L.radius = static_cast<float>(lc->radius);
        L.reach = static_cast<float>(lc->radius + 0.5 * lc->margin);
        m.lines_host = L;
        cuda_check(cudaMemcpyAsync(m.d_lines, &L, sizeof(L), cudaMemcpyHostToDevice, m.stream), "line contact");
        m.line_contact = true;
        m.upload_instances();
    });
}

swb_status swb_structure_set_ground(swb_structure* s, const swb_ground* g) {
    return guarded([&] {
        if (!s) raise(SWB_INVALID_ARGUMENT, "null structure");
        StructureImpl& m = s->s;
        if (!g || !g->enabled) {
            m.cparams.ground = 0;
            return;
        }
        const double nn = g->normal.x * g->normal.x + g->normal.y * g->normal.y + g->normal.z * g->normal.z;
        if (!std::isfinite(nn) || std::fabs(nn - 1.0) > 1e-9)
            raise(SWB_INVALID_ARGUMENT, "ground normal must be a unit vector");
        if (!std::isfinite(g->offset) || !std::isfinite(g->friction) || g->friction < 0.0)
            raise(SWB_INVALID_ARGUMENT, "ground offset and friction must be finite, friction >= 0");
        if (!m.cluster_mode) raise(SWB_UNSUPPORTED, "the ground plane needs the cluster schedule");
        m.cparams.ground = 1;
        m.cparams.ground_normal = make_float3(static_cast<float>(g->normal.x), static_cast<float>(g->normal.y),
                                              static_cast<float>(g->normal.z));
        m.cparams.ground_offset = g->offset;
        m.cparams.ground_friction = static_cast<float>(g->friction);
    });
}

swb_status swb_structure_set_uniform_pressure(swb_structure* s, double dp) {
    return guarded([&] {
        if (!s) raise(SWB_INVALID_ARGUMENT, "null structure");
        if (!std::isfinite(dp)) raise(SWB_INVALID_ARGUMENT, "Pressure difference must be finite");
        for (auto& p : s->s.pressure) p = dp;
        s->s.pressure_dirty = true;
    });
}

swb_status swb_structure_step(swb_structure* s, const swb_step_settings* settings, swb_diagnostics* out) {
    return guarded([&] {
        if (!s || !settings) raise(SWB_INVALID_ARGUMENT, "null argument");
        s->s.step(*settings, 1, out);
    });
}

swb_status swb_structure_step_many(swb_structure* s, const swb_step_settings* settings, int32_t steps,
                                   swb_diagnostics* out) {
    return guarded([&] {
        if (!s || !settings) raise(SWB_INVALID_ARGUMENT, "null argument");
        s->s.step(*settings, steps, out);
    });
}

swb_status swb_structure_diagnostics(const swb_structure* s, swb_diagnostics* out) {
    return guarded([&] {
        if (!s || !out) raise(SWB_INVALID_ARGUMENT, "null argument");
        s->s.diagnostics(out);
    });
}

swb_status swb_structure_read_nodes(const swb_structure* s, swb_node_state* out, uint64_t count) {
    return guarded([&] {
        if (!s || (!out && count)) raise(SWB_INVALID_ARGUMENT, "null argument");
        if (count != s->s.def.nodes.size()) raise(SWB_INVALID_ARGUMENT, "node count mismatch");
        std::vector<float4> pos, prev, vel;
        DevPayloadState pay;
        double o[3];
        s->s.fetch(pos, prev, vel, pay, o);
        for (uint64_t n = 0; n < count; ++n) {
            const uint32_t sl = s->s.slot_of_node[n];
            out[n].position = {pos[sl].x + o[0], pos[sl].y + o[1], pos[sl].z + o[2]};
            out[n].previous_position = {prev[sl].x + o[0], prev[sl].y + o[1], prev[sl].z + o[2]};
            out[n].velocity = {vel[sl].x, vel[sl].y, vel[sl].z};
        }
    });
}

swb_status swb_structure_read_positions_f32(const swb_structure* s, float* out, uint64_t count) {
    return guarded([&] {
        if (!s || (!out && count)) raise(SWB_INVALID_ARGUMENT, "null argument");
        if (count != s->s.def.nodes.size()) raise(SWB_INVALID_ARGUMENT, "node count mismatch");
        std::vector<float4> pos, prev, vel;
        DevPayloadState pay;
        double o[3];
        s->s.fetch(pos, prev, vel, pay, o);
        for (uint64_t n = 0; n < count; ++n) {
            const uint32_t sl = s->s.slot_of_node[n];
            out[3 * n + 0] = static_cast<float>(pos[sl].x + o[0]);
            out[3 * n + 1] = static_cast<float>(pos[sl].y + o[1]);
            out[3 * n + 2] = static_cast<float>(pos[sl].z + o[2]);
        }
    });
}

swb_status swb_structure_write_nodes(swb_structure* s, const swb_node_state* in, uint64_t count) {
    return guarded([&] {
        if (!s || (!in && count)) raise(SWB_INVALID_ARGUMENT, "null argument");
        StructureImpl& m = s->s;
        if (count != m.def.nodes.size()) raise(SWB_INVALID_ARGUMENT, "node count mismatch");
        std::vector<float4> pos, prev, vel;
        DevPayloadState pay;
        double o[3];
        m.fetch(pos, prev, vel, pay, o);
        for (uint64_t n = 0; n < count; ++n) {
            const auto& st = in[n];
            if (!std::isfinite(st.position.x) || !std::isfinite(st.position.y) || !std::isfinite(st.position.z) ||
                !std::isfinite(st.velocity.x) || !std::isfinite(st.velocity.y) || !std::isfinite(st.velocity.z) ||
                !std::isfinite(st.previous_position.x) || !std::isfinite(st.previous_position.y) ||
                !std::isfinite(st.previous_position.z))
                raise(SWB_INVALID_ARGUMENT, "node state must be finite");
        }
        if (!m.def.has_suspension && count) {
            // without a pilot to follow, the origin moves to the centre of
            // the written positions' bounding box (a suspension structure's
            // origin follows its pilot: swb_structure_write_payload)
            double lo[3], hi[3];
            for (int k = 0; k < 3; ++k) lo[k] = hi[k] = (&in[0].position.x)[k];
            for (uint64_t n = 0; n < count; ++n)
                for (int k = 0; k < 3; ++k) {
                    lo[k] = std::min(lo[k], (&in[n].position.x)[k]);
                    hi[k] = std::max(hi[k], (&in[n].position.x)[k]);
                }
            for (int k = 0; k < 3; ++k) o[k] = origin_grid(0.5 * (lo[k] + hi[k]));
            cuda_check(cudaMemcpyAsync(m.d_origin[m.cur], o, sizeof(o), cudaMemcpyHostToDevice, m.stream), "write");
        }
        for (uint64_t n = 0; n < count; ++n) {
            const auto& st = in[n];
            const uint32_t sl = m.slot_of_node[n];
            const float w = m.inv_mass[sl];
            pos[sl] = make_float4(st.position.x - o[0], st.position.y - o[1], st.position.z - o[2], w);
            prev[sl] = make_float4(st.previous_position.x - o[0], st.previous_position.y - o[1],
                                   st.previous_position.z - o[2], w);
            vel[sl] = make_float4(st.velocity.x, st.velocity.y, st.velocity.z, 0.0f);
        }
        const size_t N = m.def.nodes.size();
        cuda_check(cudaMemcpyAsync(m.d_pos[m.cur], pos.data(), N * sizeof(float4), cudaMemcpyHostToDevice, m.stream), "write");
        cuda_check(cudaMemcpyAsync(m.d_prev[m.cur], prev.data(), N * sizeof(float4), cudaMemcpyHostToDevice, m.stream), "write");
        cuda_check(cudaMemcpyAsync(m.d_vel[m.cur], vel.data(), N * sizeof(float4), cudaMemcpyHostToDevice, m.stream), "write");
        cuda_check(cudaStreamSynchronize(m.stream), "write");
    });
}

swb_status swb_structure_read_suspension(const swb_structure* s, swb_payload_state* payload,
                                         swb_segment_state* segments, uint64_t capacity, swb_wrench* wrench) {
    return guarded([&] {
        if (!s) raise(SWB_INVALID_ARGUMENT, "null structure");
        const StructureImpl& m = s->s;
        if (!m.def.has_suspension) raise(SWB_INVALID_ARGUMENT, "structure has no suspension");
        std::vector<float4> pos, prev, vel;
        DevPayloadState pay;
        double o[3];
        m.fetch(pos, prev, vel, pay, o);
        if (payload) {
            payload->center_of_mass = {pay.com.x + o[0], pay.com.y + o[1], pay.com.z + o[2]};
            payload->body_to_world = {pay.q.x, pay.q.y, pay.q.z, pay.q.w};
            payload->linear_velocity = {pay.v.x, pay.v.y, pay.v.z};
            payload->angular_velocity = {pay.w.x, pay.w.y, pay.w.z};
        }
        if (wrench) {
            wrench->force = {pay.line_force.x, pay.line_force.y, pay.line_force.z};
            wrench->moment = {pay.line_moment.x, pay.line_moment.y, pay.line_moment.z};
        }
        // segment states in definition order (Structure::suspensionState)
        const uint64_t nseg = m.def.segments.size();
        for (uint64_t k = 0; segments && k < nseg && k < capacity; ++k) {
            // device index of definition segment k
            size_t dk = 0;
            for (size_t q = 0; q < m.segment_order.size(); ++q)
                if (m.segment_order[q] == k) dk = q;
            const DevPayloadDef& d = m.payload_def_host;
            auto endpoint = [&](int node, int point) {
                double r[3];
                if (node >= 0) {
                    const float4 X = pos[m.susp_base + node];
                    r[0] = X.x; r[1] = X.y; r[2] = X.z;
                } else {
                    const double qw = pay.q.x, qx = pay.q.y, qy = pay.q.z, qz = pay.q.w;
                    const double R[9] = {1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - qw * qz), 2 * (qx * qz + qw * qy),
                                         2 * (qx * qy + qw * qz), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - qw * qx),
                                         2 * (qx * qz - qw * qy), 2 * (qy * qz + qw * qx), 1 - 2 * (qx * qx + qy * qy)};
                    const double l[3] = {d.hang_local[point].x - d.com_local.x, d.hang_local[point].y - d.com_local.y,
                                         d.hang_local[point].z - d.com_local.z};
                    const double c[3] = {pay.com.x, pay.com.y, pay.com.z};
                    for (int i = 0; i < 3; ++i) r[i] = c[i] + R[i * 3] * l[0] + R[i * 3 + 1] * l[1] + R[i * 3 + 2] * l[2];
                }
                return std::array<double, 3>{r[0], r[1], r[2]};
            };
            const auto a = endpoint(d.from_node[dk], d.from_point[dk]);
            const auto b = endpoint(d.to_node[dk], d.to_point[dk]);
            const double len = std::sqrt((b[0] - a[0]) * (b[0] - a[0]) + (b[1] - a[1]) * (b[1] - a[1]) +
                                         (b[2] - a[2]) * (b[2] - a[2]));
            segments[k].stable_id = m.def.segments[k].stable_id;
            segments[k].current_length = m.accepted ? len : m.def.segments[k].rest_length;
            segments[k].commanded_rest_length = m.def.segments[k].rest_length;
            segments[k].tension = m.accepted ? pay.lambda[dk] / (m.last_dt * m.last_dt) : 0.0;
        }
    });
}

swb_status swb_structure_write_payload(swb_structure* s, const swb_payload_state* in) {
    return guarded([&] {
        if (!s || !in) raise(SWB_INVALID_ARGUMENT, "null argument");
        StructureImpl& m = s->s;
        if (!m.def.has_suspension) raise(SWB_INVALID_ARGUMENT, "structure has no suspension");
        std::vector<float4> pos, prev, vel;
        DevPayloadState pay;
        double o[3];
        m.fetch(pos, prev, vel, pay, o);
        const double c[3] = {in->center_of_mass.x, in->center_of_mass.y, in->center_of_mass.z};
        if (!std::isfinite(c[0]) || !std::isfinite(c[1]) || !std::isfinite(c[2]))
            raise(SWB_INVALID_ARGUMENT, "payload state must be finite");
        // the origin follows the pilot, as the step's recentring keeps it:
        // the node offsets are re-expressed from the new origin, so the
        // pilot's first step from an imported state is taken in small
        // coordinates too
        const double n[3] = {origin_grid(c[0]), origin_grid(c[1]), origin_grid(c[2])};
        if (std::max({std::fabs(n[0] - o[0]), std::fabs(n[1] - o[1]), std::fabs(n[2] - o[2])}) > 0.25) {
            for (auto* v : {&pos, &prev})
                for (float4& x : *v) {
                    x.x = static_cast<float>(static_cast<double>(x.x) + (o[0] - n[0]));
                    x.y = static_cast<float>(static_cast<double>(x.y) + (o[1] - n[1]));
                    x.z = static_cast<float>(static_cast<double>(x.z) + (o[2] - n[2]));
                }
            for (int k = 0; k < 3; ++k) o[k] = n[k];
            const size_t N = pos.size();
            cuda_check(cudaMemcpyAsync(m.d_pos[m.cur], pos.data(), N * sizeof(float4), cudaMemcpyHostToDevice, m.stream),
                       "write");
            cuda_check(cudaMemcpyAsync(m.d_prev[m.cur], prev.data(), N * sizeof(float4), cudaMemcpyHostToDevice,
                                       m.stream), "write");
            cuda_check(cudaMemcpyAsync(m.d_origin[m.cur], o, sizeof(o), cudaMemcpyHostToDevice, m.stream), "write");
        }
        pay.com = make_float3(c[0] - o[0], c[1] - o[1], c[2] - o[2]);
        pay.q = make_float4(in->body_to_world.w, in->body_to_world.x, in->body_to_world.y, in->body_to_world.z);
        pay.v = make_float3(in->linear_velocity.x, in->linear_velocity.y, in->linear_velocity.z);
        pay.w = make_float3(in->angular_velocity.x, in->angular_velocity.y, in->angular_velocity.z);
        cuda_check(cudaMemcpyAsync(m.d_payload[m.cur], &pay, sizeof(pay), cudaMemcpyHostToDevice, m.stream), "write");
        cuda_check(cudaStreamSynchronize(m.stream), "write");
    });
}

swb_status swb_structure_sweep_order(const swb_structure* s, uint32_t which, uint64_t* order, uint64_t count) {
    return guarded([&] {
        if (!s || (!order && count)) raise(SWB_INVALID_ARGUMENT, "null argument");
        const StructureImpl& m = s->s;
        if (which > SWB_SWEEP_MEMBRANE) raise(SWB_INVALID_ARGUMENT, "unknown sweep");
        static const std::vector<uint64_t> none;
        const auto& v = m.cluster_mode
                            ? (which == SWB_SWEEP_DISTANCE
                                   ? m.csched.distance_order
                                   : (which == SWB_SWEEP_DIHEDRAL ? m.csched.dihedral_order : m.csched.membrane_order))
                            : (which == SWB_SWEEP_DISTANCE ? m.sched.distance_order
                                                           : (which == SWB_SWEEP_DIHEDRAL ? m.sched.dihedral_order : none));
        if (count != v.size()) raise(SWB_INVALID_ARGUMENT, "order count mismatch");
        std::copy(v.begin(), v.end(), order);
    });
}

swb_status swb_structure_contact_candidates(const swb_structure* s, swb_contact_key* keys, uint64_t capacity,
                                            uint64_t* count) {
    return guarded([&] {
        if (!s || !count || (capacity && !keys)) raise(SWB_INVALID_ARGUMENT, "null argument");
        const StructureImpl& m = s->s;
        if (!m.def.has_contact) raise(SWB_UNSUPPORTED, "the structure has no fabric self-contact");
        cuda_check(cudaSetDevice(m.device), "cudaSetDevice");
        ContactDiagDev cd{};
        cuda_check(cudaMemcpyAsync(&cd, m.d_cdiag[m.cur], sizeof(cd), cudaMemcpyDeviceToHost, m.stream), "read");
        cuda_check(cudaStreamSynchronize(m.stream), "read");
        *count = cd.candidates;
        if (cd.candidates > capacity) raise(SWB_OUT_OF_RANGE, "candidate capacity too small");
        std::vector<unsigned long long> codes(cd.candidates);
        if (!codes.empty())
            cuda_check(cudaMemcpy(codes.data(), m.contact_host.cand, codes.size() * sizeof(unsigned long long),
                                  cudaMemcpyDeviceToHost), "read");
        for (size_t k = 0; k < codes.size(); ++k)
            keys[k] = contact_key_of(m.contact_surface, codes[k] >> 32, codes[k] & 0xffffffffull);
    });
}

swb_status swb_structure_schedule_report(const swb_structure* s, swb_schedule_report* out) {
    return guarded([&] {
        if (!s || !out) raise(SWB_INVALID_ARGUMENT, "null argument");
        const StructureImpl& m = s->s;
        const Schedule& S = m.sched;
        std::memset(out, 0, sizeof(*out));
        out->blocks = m.G;
        out->block_threads = m.threads;
        if (m.cluster_mode) {
            const ClusterSchedule& C = m.csched;
            out->cluster_ctas = C.ctas;
            out->local_stages_per_iteration = total_stages(C);
            out->cluster_barriers_per_iteration = cluster_barriers_per_iteration(C);
            out->max_patch_nodes = static_cast<int32_t>(C.max_patch);
            out->shared_bytes = static_cast<int32_t>(m.cluster_smem);
            out->level_constraints[0] = m.def.constraints.size() + m.def.dihedrals.size();
            return;
        }
        out->partition_levels = S.levels;
        int phases = 0, stages = 0;
        for (int k = 0; k < kKinds; ++k) {
            bool outer = S.global[k].colour_offsets.size() > 1;
            for (int l = 0; l < S.levels; ++l) {
                stages += S.tables[l][k].stages;
                if (l > 0 && S.tables[l][k].stages > 0) { outer = true; ++phases; }
            }
            const int gc = S.global[k].colour_offsets.empty() ? 0 : static_cast<int>(S.global[k].colour_offsets.size()) - 1;
            out->global_colours_per_iteration += gc;
            phases += gc + (outer ? 1 : 0);
        }
        out->device_phases_per_iteration = phases;
        out->local_stages_per_iteration = stages;
        out->max_patch_nodes = S.max_patch_nodes;
        out->shared_bytes = static_cast<int32_t>(m.params.smem_total);
        for (int l = 0; l < 4; ++l) out->level_constraints[l] = S.level_constraints[l];
        out->global_constraints = S.global_constraints;
    });
}

}  // extern "C"
