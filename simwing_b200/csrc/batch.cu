// Batched structures: many independent structures stepped by one packed
// cluster launch per substep, the launches of a block of steps captured in
// one CUDA graph.
//
// Layout.  Each structure is an ordinary StructureImpl built with its own
// cluster schedule over g ranks (g = its node count over the target patch
// size).  The batch packs the structures' rank ranges into clusters of C
// ranks (first fit, largest first) and runs xpbd_cluster_packed_kernel: a CTA
// looks up its structure and rank base in a slot table, every cluster loops
// over the largest stage count among its structures, so all its CTAs take
// the same barriers.
//
// Transactions.  Per structure, buffer b (its committed state) is never
// written during a block: the first launch reads b and writes b+1, later
// launches ping-pong between b+1 and b+2.  After the block the host reads
// one status pair per structure and commits the last buffer of every
// structure whose status is clean; a failed structure keeps buffer b, which
// is its state before the block.  Per-structure rotation (which buffer is b)
// is a small device array read by the kernel, so one captured graph serves
// every block whatever the structures' rotations.
#include "structure_impl.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>
#include <thread>

namespace swb {
namespace {

uint32_t align16u(uint32_t v) { return (v + 15u) & ~15u; }

template <class T>
T* batch_alloc(std::vector<void*>& owned, size_t count) {
    void* p = nullptr;
    cuda_check(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)), "cudaMalloc");
    owned.push_back(p);
    return static_cast<T*>(p);
}

// Structures built for one target patch size, packed into clusters.
struct Packing {
    int target = 0;
    std::vector<std::unique_ptr<swb_structure>> members;
    std::vector<int> ranks;            // per structure
    std::vector<ClusterSlot> slots;    // per CTA
    int clusters = 0;
    int idle = 0;
    int threads = 0;
    int max_stages = 0;
    uint32_t smem_v = 0, smem_offsets = 0, smem = 0;
    std::vector<uint32_t> lambda_offset[3];  // per structure and kind
    bool membranes = false;                  // a structure carries membrane elements
};

int initial_ranks(uint64_t nodes, int target, int cluster) {
    // 5 % headroom for the bisection's balance tolerance
    const double per = std::max(64.0, 0.95 * target);
    const int g = static_cast<int>(std::ceil(static_cast<double>(nodes) / per));
    return std::clamp(g, 1, cluster);
}

// Builds structure `def` on the fewest ranks >= `g` that fit the cluster
// schedule; UNSUPPORTED when even `cluster` ranks do not fit.
std::unique_ptr<swb_structure> build_member(const swb_structure_definition& def, int device, int g, int cluster,
                                            int& ranks_out) {
    for (int r = g; r <= cluster; ++r) {
        swb_solver_options opt;
        swb_default_solver_options(&opt);
        opt.device = device;
        opt.cluster_ctas = r;  // classic stages: a packed cluster takes the same barriers on every rank
        auto m = std::make_unique<swb_structure>();
        try {
            if (def.fabric_self_contact)
                raise(SWB_UNSUPPORTED, "fabric self-contact is not available in batches (single structures only)");
            m->s.build(def, &opt);
        } catch (const Error& e) {
            if (e.status == SWB_UNSUPPORTED) continue;
            throw;
        }
        ranks_out = r;
        return m;
    }
    raise(SWB_UNSUPPORTED, "a structure of the batch does not fit a cluster of " + std::to_string(cluster) + " CTAs");
}

void build_members(const std::vector<const swb_structure_definition*>& defs, int device, int target, int cluster,
                   Packing& P) {
    const size_t n = defs.size();
    P.target = target;
    P.members.resize(n);
    P.ranks.assign(n, 0);
    std::atomic<size_t> next{0};
    std::vector<std::string> errors(n);
    std::vector<swb_status> codes(n, SWB_OK);
    auto work = [&] {
        cudaSetDevice(device);
        for (size_t i = next++; i < n; i = next++) {
            try {
                uint64_t nodes = defs[i]->node_count;
                P.members[i] = build_member(*defs[i], device, initial_ranks(nodes, target, cluster), cluster,
                                            P.ranks[i]);
                P.members[i]->borrowed = true;
            } catch (const Error& e) {
                codes[i] = e.status;
                errors[i] = e.what();
            } catch (const std::exception& e) {
                codes[i] = SWB_INVALID_ARGUMENT;
                errors[i] = e.what();
            }
        }
    };
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t workers = std::min<size_t>(n, std::min(hw, 16u));
    std::vector<std::thread> pool;
    for (size_t w = 1; w < workers; ++w) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    for (size_t i = 0; i < n; ++i)
        if (codes[i] != SWB_OK) raise(codes[i], "structure " + std::to_string(i) + ": " + errors[i]);
}

void pack(Packing& P, int cluster, int threads_opt, size_t smem_limit) {
    const size_t n = P.members.size();
    std::vector<size_t> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return P.ranks[a] > P.ranks[b]; });
    std::vector<int> free_ranks;               // per cluster
    std::vector<std::vector<size_t>> content;  // per cluster, in rank order
    for (size_t i : order) {
        size_t c = 0;
        while (c < free_ranks.size() && free_ranks[c] < P.ranks[i]) ++c;
        if (c == free_ranks.size()) {
            free_ranks.push_back(cluster);
            content.emplace_back();
        }
        free_ranks[c] -= P.ranks[i];
        content[c].push_back(i);
    }
    P.clusters = static_cast<int>(content.size());
    P.slots.assign(static_cast<size_t>(P.clusters) * cluster, ClusterSlot{});
    P.idle = 0;
    P.max_stages = 0;
    for (int c = 0; c < P.clusters; ++c) {
        int stages = 0, seam = 0, susp = 0, guard = 0;
        for (size_t i : content[c]) {
            const StructureImpl& m = P.members[i]->s;
            stages = std::max(stages, total_stages(m.csched));
            seam = std::max(seam, m.csched.seam_stages);
            susp |= m.def.has_suspension ? 1 : 0;
            guard |= m.momentum_guard ? 1 : 0;
        }
        P.max_stages = std::max(P.max_stages, stages);
        int rank = 0;
        for (size_t i : content[c])
            for (int r = 0; r < P.ranks[i]; ++r, ++rank) {
                ClusterSlot& s = P.slots[static_cast<size_t>(c) * cluster + rank];
                s.instance = static_cast<int>(i);
                s.rank_base = rank - r;
                s.ctas = P.ranks[i];
            }
        for (; rank < cluster; ++rank) {
            P.slots[static_cast<size_t>(c) * cluster + rank].instance = -1;
            ++P.idle;
        }
        for (int r = 0; r < cluster; ++r) {
            ClusterSlot& s = P.slots[static_cast<size_t>(c) * cluster + r];
            s.stages = stages;
            s.seam_stages = seam;
            s.suspension = susp;
            s.guard = guard;
        }
    }
    // shared memory: node arrays for the largest patch, then per-structure
    // multipliers, then stage offsets
    uint32_t max_patch = 0, lambda_bytes = 0, offset_bytes = 0;
    int threads = 32;
    for (size_t i = 0; i < n; ++i) {
        const StructureImpl& m = P.members[i]->s;
        max_patch = std::max(max_patch, m.csched.max_patch);
        lambda_bytes = std::max(lambda_bytes, align16u(m.csched.kinds[0].max_cta_records * 4u) +
                                                  align16u(m.csched.kinds[1].max_cta_records * 4u) +
                                                  align16u(m.csched.kinds[2].max_cta_records * 12u));
        offset_bytes = std::max(offset_bytes, align16u((total_stages(m.csched) + 3) * 4u));
        P.membranes = P.membranes || !m.def.membranes.empty();
        threads = std::max(threads, m.threads);
    }
    P.smem_v = align16u(max_patch * 16u);
    const uint32_t lambda_base = P.smem_v + align16u(max_patch * 16u);
    for (int k = 0; k < 3; ++k) P.lambda_offset[k].assign(n, 0);
    for (size_t i = 0; i < n; ++i) {
        const StructureImpl& m = P.members[i]->s;
        P.lambda_offset[0][i] = lambda_base;
        P.lambda_offset[1][i] = lambda_base + align16u(m.csched.kinds[0].max_cta_records * 4u);
        P.lambda_offset[2][i] = P.lambda_offset[1][i] + align16u(m.csched.kinds[1].max_cta_records * 4u);
    }
    P.smem_offsets = lambda_base + lambda_bytes;
    P.smem = P.smem_offsets + offset_bytes;
    if (P.smem > smem_limit)
        raise(SWB_UNSUPPORTED, "batch shared memory " + std::to_string(P.smem) + " B exceeds the device limit");
    if (threads_opt > 0) threads = threads_opt;
    P.threads = std::clamp((threads + 31) / 32 * 32, 64, dev::kClusterMaxThreads);
}

}  // namespace

struct BatchImpl {
    int device = 0;
    int cluster = 16;
    uint32_t flags = 0;
    int graph_steps = 120;
    Packing P;
    std::vector<void*> owned;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    ClusterInstance* d_records = nullptr;
    ClusterSlot* d_slots = nullptr;
    int* d_rotation = nullptr;
    int* d_status = nullptr;
    int* h_rotation = nullptr;   // pinned
    int* h_status = nullptr;     // pinned
    int resident = 0;
    size_t smem_limit = 0;
    cudaLaunchAttribute launch_attr[1] = {};
    double last_ms = 0.0;
    swb_ground ground{};   // the launch's ground plane (enabled = 0: none)
    std::vector<int> candidates;
    std::vector<int> candidate_threads;
    std::vector<double> candidate_ms;
    // captured graph and what it was captured for
    cudaGraphExec_t graph = nullptr;
    int graph_launches = 0;
    std::vector<double> graph_key;

    ~BatchImpl() {
        cudaSetDevice(device);
        if (graph) cudaGraphExecDestroy(graph);
        for (void* p : owned) cudaFree(p);
        if (h_rotation) cudaFreeHost(h_rotation);
        if (h_status) cudaFreeHost(h_status);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }

    size_t size() const { return P.members.size(); }

    void release_tables() {
        if (graph) {
            cudaGraphExecDestroy(graph);
            graph = nullptr;
        }
        for (void* p : owned) cudaFree(p);
        owned.clear();
        d_records = nullptr;
        d_slots = nullptr;
        d_rotation = nullptr;
        d_status = nullptr;
    }

    // Device tables of the current packing.
    void upload_tables() {
        release_tables();
        const size_t n = size();
        std::vector<ClusterInstance> rec(n * 9);
        d_status = batch_alloc<int>(owned, 2 * n);
        for (size_t i = 0; i < n; ++i) {
            const StructureImpl& m = P.members[i]->s;
            for (int b = 0; b < 3; ++b)
                for (int role = 0; role < 3; ++role) {
                    const int t1 = (b + 1) % 3, t2 = (b + 2) % 3;
                    const int in = role == 0 ? b : (role == 1 ? t1 : t2);
                    const int out = role == 0 ? t1 : (role == 1 ? t2 : t1);
                    ClusterInstance c = m.cluster_base;
                    c.pos_in = m.d_pos[in]; c.vel_in = m.d_vel[in];
                    c.pos_out = m.d_pos[out]; c.vel_out = m.d_vel[out]; c.prev_out = m.d_prev[out];
                    c.force = m.d_force;
                    c.tri_offsets = m.d_tri_off; c.tri_list = m.d_tri_list; c.tri = m.d_tri;
                    c.susp_cta = m.def.has_suspension ? m.susp_owner : -1;
                    c.payload_def = m.d_payload_def;
                    c.payload_in = m.d_payload[in]; c.payload_out = m.d_payload[out];
                    c.origin_in = m.d_origin[in]; c.origin_out = m.d_origin[out];
                    c.status = d_status + 2 * i;
                    c.recentre = m.def.has_suspension ? 1 : 0;
                    c.kind[0].smem_lambda = P.lambda_offset[0][i];
                    c.kind[1].smem_lambda = P.lambda_offset[1][i];
                    c.kind[2].smem_lambda = P.lambda_offset[2][i];
                    c.membrane_residual = m.d_mres[out];
                    rec[(i * 3 + b) * 3 + role] = c;
                }
        }
        d_records = batch_alloc<ClusterInstance>(owned, rec.size());
        cuda_check(cudaMemcpyAsync(d_records, rec.data(), rec.size() * sizeof(ClusterInstance),
                                   cudaMemcpyHostToDevice, stream), "batch upload");
        d_slots = batch_alloc<ClusterSlot>(owned, P.slots.size());
        cuda_check(cudaMemcpyAsync(d_slots, P.slots.data(), P.slots.size() * sizeof(ClusterSlot),
                                   cudaMemcpyHostToDevice, stream), "batch upload");
        d_rotation = batch_alloc<int>(owned, n);
        if (h_rotation) cudaFreeHost(h_rotation);
        if (h_status) cudaFreeHost(h_status);
        h_rotation = nullptr;
        h_status = nullptr;
        cuda_check(cudaMallocHost(&h_rotation, std::max<size_t>(n, 1) * sizeof(int)), "cudaMallocHost");
        cuda_check(cudaMallocHost(&h_status, std::max<size_t>(2 * n, 1) * sizeof(int)), "cudaMallocHost");
        // the attribute is a per-kernel limit shared by every batch in the
        // process, so it is set to the device limit, never lowered
        cuda_check(packed_kernel_limits(static_cast<int>(smem_limit), cluster > 8), "batch kernel limits");
        cudaLaunchConfig_t cfg = launch_config();
        cuda_check(packed_kernel_occupancy(&resident, cfg, P.membranes), "cluster occupancy");
        if (resident < 1) raise(SWB_UNSUPPORTED, "the batch's cluster shape cannot be scheduled");
        cuda_check(cudaStreamSynchronize(stream), "batch upload");
    }

    cudaLaunchConfig_t launch_config() {
        cudaLaunchAttribute* attr = launch_attr;
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = static_cast<unsigned>(cluster);
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(static_cast<unsigned>(P.clusters * cluster));
        cfg.blockDim = dim3(static_cast<unsigned>(P.threads));
        cfg.dynamicSmemBytes = P.smem;
        cfg.stream = stream;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        return cfg;
    }

    ClusterParams params(const swb_step_settings& st, int role) const {
        const double dt = st.time_step / st.substeps;
        ClusterParams cp{};
        cp.instances = d_records;
        cp.ctas = cluster;
        cp.slots = d_slots;
        cp.rotation = d_rotation;
        cp.role = role;
        cp.dt = static_cast<float>(dt);
        cp.inv_dt = static_cast<float>(1.0 / dt);
        cp.inv_dt2 = static_cast<float>(1.0 / (dt * dt));
        cp.damping = static_cast<float>(std::exp(-st.velocity_damping * dt));
        cp.damping_loss = static_cast<float>(-std::expm1(-st.velocity_damping * dt));
        cp.gravity = make_float3(st.gravity.x, st.gravity.y, st.gravity.z);
        cp.ref_velocity = make_float3(st.damping_reference_velocity.x, st.damping_reference_velocity.y,
                                      st.damping_reference_velocity.z);
        cp.iterations = st.constraint_iterations;
        cp.copy_budget = 4000000000LL;
        cp.smem_x = 0;
        cp.smem_v = P.smem_v;
        cp.smem_offsets = P.smem_offsets;
        if (ground.enabled) {
            cp.ground = 1;
            cp.ground_normal = make_float3(static_cast<float>(ground.normal.x), static_cast<float>(ground.normal.y),
                                           static_cast<float>(ground.normal.z));
            cp.ground_offset = ground.offset;
            cp.ground_friction = static_cast<float>(ground.friction);
        }
        return cp;
    }

    // Status clear and `launches` launches (role 0, then 1, 2, 1, 2, ...).
    void enqueue(const swb_step_settings& st, int launches) {
        cuda_check(cudaMemsetAsync(d_status, 0, 2 * size() * sizeof(int), stream), "status clear");
        cudaLaunchConfig_t cfg = launch_config();
        for (int k = 0; k < launches; ++k) {
            const ClusterParams cp = params(st, k == 0 ? 0 : (k % 2 ? 1 : 2));
            cuda_check(packed_kernel_launch(cfg, cp, P.membranes), "batch launch");
        }
    }

    void run_block(const swb_step_settings& st, int steps) {
        const int launches = steps * st.substeps;
        const bool use_graph = !(flags & SWB_OPT_NO_GRAPH);
        if (use_graph) {
            const std::vector<double> key = {st.time_step, double(st.substeps), double(st.constraint_iterations),
                                             st.gravity.x, st.gravity.y, st.gravity.z, st.velocity_damping,
                                             st.damping_reference_velocity.x, st.damping_reference_velocity.y,
                                             st.damping_reference_velocity.z, double(launches)};
            if (!graph || key != graph_key) {
                if (graph) {
                    cudaGraphExecDestroy(graph);
                    graph = nullptr;
                }
                cudaGraph_t g = nullptr;
                cuda_check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "graph capture");
                try {
                    enqueue(st, launches);
                } catch (...) {
                    cudaStreamEndCapture(stream, &g);
                    if (g) cudaGraphDestroy(g);
                    throw;
                }
                cuda_check(cudaStreamEndCapture(stream, &g), "graph capture");
                const cudaError_t rc = cudaGraphInstantiate(&graph, g, 0);
                cudaGraphDestroy(g);
                cuda_check(rc, "graph instantiate");
                graph_key = key;
                graph_launches = launches;
            }
            cuda_check(cudaGraphLaunch(graph, stream), "graph launch");
        } else {
            enqueue(st, launches);
        }
    }

    swb_status step(const swb_step_settings& st, int steps, int32_t* statuses, std::string& first_message) {
        if (steps < 1) raise(SWB_INVALID_ARGUMENT, "steps must be positive");
        const size_t n = size();
        for (size_t i = 0; i < n; ++i) {
            P.members[i]->s.validate_settings(st);
            if (P.members[i]->s.line_contact)
                raise(SWB_UNSUPPORTED, "line-line contact is not available in batches (single structures only)");
        }
        if (st.cable_sweep_pairs != 0) raise(SWB_UNSUPPORTED, "load-path cable sweep pairs are not available in batches");
        cuda_check(cudaSetDevice(device), "cudaSetDevice");
        std::vector<char> alive(n, 1);
        std::vector<swb_status> result(n, SWB_OK);
        double total_ms = 0.0;
        for (int done = 0; done < steps;) {
            const int block = std::min(graph_steps, steps - done);
            // loads and pressure of every structure, then the rotations
            for (size_t i = 0; i < n; ++i) {
                StructureImpl& m = P.members[i]->s;
                if (m.pressure_dirty) m.upload_pressure();
                if (m.forces_dirty) m.upload_forces();
                cuda_check(cudaStreamSynchronize(m.stream), "batch loads");
                h_rotation[i] = m.cur;
            }
            cuda_check(cudaMemcpyAsync(d_rotation, h_rotation, n * sizeof(int), cudaMemcpyHostToDevice, stream),
                       "rotation upload");
            cuda_check(cudaEventRecord(ev0, stream), "event");
            run_block(st, block);
            cuda_check(cudaEventRecord(ev1, stream), "event");
            cuda_check(cudaMemcpyAsync(h_status, d_status, 2 * n * sizeof(int), cudaMemcpyDeviceToHost, stream),
                       "status read");
            cuda_check(cudaStreamSynchronize(stream), "batch step");
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, ev0, ev1);
            total_ms += ms;
            const int launches = block * st.substeps;
            for (size_t i = 0; i < n; ++i) {
                if (!alive[i]) continue;
                StructureImpl& m = P.members[i]->s;
                std::string message;
                const swb_status s = decode_status(h_status + 2 * i, message);
                if (s == SWB_OK) {
                    const int b = m.cur;
                    m.commit(launches == 1 || launches % 2 ? (b + 1) % 3 : (b + 2) % 3, block, st);
                } else {
                    alive[i] = 0;
                    result[i] = s;
                    if (first_message.empty())
                        first_message = "structure " + std::to_string(i) + ": " + message;
                }
            }
            done += block;
            if (std::find(alive.begin(), alive.end(), 1) == alive.end()) break;
        }
        last_ms = total_ms;
        swb_status first = SWB_OK;
        for (size_t i = 0; i < n; ++i) {
            if (statuses) statuses[i] = result[i];
            if (first == SWB_OK) first = result[i];
        }
        return first;
    }

    // ms per trial launch of the current packing; the launches read the
    // committed buffers and write the trial buffers only (role 0), so the
    // structures' states are not advanced.
    double time_trial(const swb_step_settings& st, int warm, int timed) {
        const size_t n = size();
        for (size_t i = 0; i < n; ++i) h_rotation[i] = P.members[i]->s.cur;
        cuda_check(cudaMemcpyAsync(d_rotation, h_rotation, n * sizeof(int), cudaMemcpyHostToDevice, stream),
                   "rotation upload");
        cudaLaunchConfig_t cfg = launch_config();
        const ClusterParams cp = params(st, 0);
        for (int k = 0; k < warm; ++k)
            cuda_check(packed_kernel_launch(cfg, cp, P.membranes), "trial launch");
        cuda_check(cudaEventRecord(ev0, stream), "event");
        for (int k = 0; k < timed; ++k)
            cuda_check(packed_kernel_launch(cfg, cp, P.membranes), "trial launch");
        cuda_check(cudaEventRecord(ev1, stream), "event");
        cuda_check(cudaStreamSynchronize(stream), "trial");
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ev0, ev1);
        return ms / timed;
    }
};

}  // namespace swb

struct swb_batch {
    swb::BatchImpl b;
};

using namespace swb;

extern "C" {

void swb_default_batch_options(swb_batch_options* out) {
    if (!out) return;
    std::memset(out, 0, sizeof(*out));
    out->cluster_ctas = 16;
    out->graph_steps = 120;
    out->autotune_iterations = 48;
}

swb_status swb_batch_create(const swb_structure_definition* const* definitions, uint64_t count,
                            const swb_batch_options* options, swb_batch** out) {
    return guarded([&] {
        if (!definitions || !out || count == 0) raise(SWB_INVALID_ARGUMENT, "a batch needs definitions");
        if (count > (1u << 20)) raise(SWB_INVALID_ARGUMENT, "too many structures");
        swb_batch_options opt;
        swb_default_batch_options(&opt);
        if (options) opt = *options;
        if (opt.cluster_ctas == 0) opt.cluster_ctas = 16;
        if (opt.cluster_ctas < 1 || opt.cluster_ctas > kClusterMaxCtas)
            raise(SWB_INVALID_ARGUMENT, "cluster_ctas must be in 1..16");
        if (opt.graph_steps == 0) opt.graph_steps = 120;
        if (opt.graph_steps < 1) raise(SWB_INVALID_ARGUMENT, "graph_steps must be positive");
        if (opt.target_patch_nodes < 0 || opt.target_patch_nodes > static_cast<int>(kClusterPatchNodes))
            raise(SWB_INVALID_ARGUMENT, "target_patch_nodes must be in 0..4096");
        if (opt.block_threads < 0 || opt.block_threads > dev::kClusterMaxThreads)
            raise(SWB_INVALID_ARGUMENT, "block_threads must be in 0..768");
        std::vector<const swb_structure_definition*> defs(definitions, definitions + count);
        for (const auto* d : defs)
            if (!d) raise(SWB_INVALID_ARGUMENT, "null definition");
        auto h = std::make_unique<swb_batch>();
        BatchImpl& B = h->b;
        B.device = opt.device;
        B.cluster = opt.cluster_ctas;
        B.flags = opt.flags;
        B.graph_steps = opt.graph_steps;
        cuda_check(cudaSetDevice(B.device), "cudaSetDevice");
        cudaDeviceProp prop{};
        cuda_check(cudaGetDeviceProperties(&prop, B.device), "cudaGetDeviceProperties");
        const size_t smem_limit = dynamic_smem_limit(prop);
        B.smem_limit = smem_limit;
        cuda_check(cudaStreamCreateWithFlags(&B.stream, cudaStreamNonBlocking), "cudaStreamCreate");
        cuda_check(cudaEventCreate(&B.ev0), "cudaEventCreate");
        cuda_check(cudaEventCreate(&B.ev1), "cudaEventCreate");

        std::vector<int> targets;
        if (opt.target_patch_nodes > 0) targets = {opt.target_patch_nodes};
        else if (opt.flags & SWB_BATCH_AUTOTUNE) targets = {1024, 2048, 4096};
        else targets = {2048};
        swb_step_settings trial;
        swb_default_step_settings(&trial);
        trial.substeps = 1;
        trial.constraint_iterations = opt.autotune_iterations > 0 ? opt.autotune_iterations : 48;
        // block sizes: the caller's, or with the autotuner also 512 threads
        // beside enough for the widest stage
        std::vector<int> thread_choices = {opt.block_threads};
        if ((opt.flags & SWB_BATCH_AUTOTUNE) && opt.block_threads == 0) thread_choices.push_back(512);
        const bool tuning = targets.size() * thread_choices.size() > 1;
        double best = 1e300;
        Packing best_packing;
        for (const int target : targets) {
            Packing P;
            build_members(defs, B.device, target, B.cluster, P);
            if (!tuning) {
                pack(P, B.cluster, thread_choices[0], smem_limit);
                best_packing = std::move(P);
                break;
            }
            // the trial settings must be valid for every structure (a pilot
            // fixes the iteration count)
            swb_step_settings st = trial;
            for (const auto& m : P.members)
                if (m->s.def.has_suspension) st.constraint_iterations = m->s.def.suspension.solver_iterations;
            int best_threads = -1;
            for (const int block_threads : thread_choices) {
                pack(P, B.cluster, block_threads, smem_limit);
                B.P = std::move(P);
                B.upload_tables();
                const double ms = B.time_trial(st, 2, 3);
                B.release_tables();
                P = std::move(B.P);
                B.P = Packing{};
                B.candidates.push_back(target);
                B.candidate_threads.push_back(block_threads);
                B.candidate_ms.push_back(ms);
                if (ms < best) {
                    best = ms;
                    best_threads = block_threads;
                }
            }
            if (best_threads >= 0) {
                pack(P, B.cluster, best_threads, smem_limit);
                best_packing = std::move(P);
            }
        }
        B.P = std::move(best_packing);
        B.upload_tables();
        *out = h.release();
    });
}

void swb_batch_destroy(swb_batch* batch) { delete batch; }

uint64_t swb_batch_size(const swb_batch* batch) { return batch ? batch->b.size() : 0; }

swb_structure* swb_batch_structure(swb_batch* batch, uint64_t index) {
    if (!batch || index >= batch->b.size()) return nullptr;
    return batch->b.P.members[index].get();
}

swb_status swb_batch_step(swb_batch* batch, const swb_step_settings* settings, int32_t steps, int32_t* statuses) {
    swb_status result = SWB_OK;
    std::string message;
    const swb_status call = guarded([&] {
        if (!batch || !settings) raise(SWB_INVALID_ARGUMENT, "null argument");
        result = batch->b.step(*settings, steps, statuses, message);
    });
    if (call != SWB_OK) return call;
    if (result != SWB_OK) set_last_error(message);
    return result;
}

swb_status swb_batch_set_ground(swb_batch* batch, const swb_ground* g) {
    return swb::guarded([&] {
        if (!batch) swb::raise(SWB_INVALID_ARGUMENT, "null batch");
        swb::BatchImpl& b = batch->b;
        if (!g || !g->enabled) {
            b.ground = swb_ground{};
        } else {
            const double nn = g->normal.x * g->normal.x + g->normal.y * g->normal.y + g->normal.z * g->normal.z;
            if (!std::isfinite(nn) || std::fabs(nn - 1.0) > 1e-9)
                swb::raise(SWB_INVALID_ARGUMENT, "ground normal must be a unit vector");
            if (!std::isfinite(g->offset) || !std::isfinite(g->friction) || g->friction < 0.0)
                swb::raise(SWB_INVALID_ARGUMENT, "ground offset and friction must be finite, friction >= 0");
            b.ground = *g;
        }
        // the captured graph holds the old parameters
        if (b.graph) {
            cudaGraphExecDestroy(b.graph);
            b.graph = nullptr;
        }
    });
}

swb_status swb_batch_get_report(const swb_batch* batch, swb_batch_report* out) {
    return guarded([&] {
        if (!batch || !out) raise(SWB_INVALID_ARGUMENT, "null argument");
        const BatchImpl& B = batch->b;
        std::memset(out, 0, sizeof(*out));
        out->structures = static_cast<int32_t>(B.size());
        out->clusters = B.P.clusters;
        out->cluster_ctas = B.cluster;
        out->idle_ctas = B.P.idle;
        out->block_threads = B.P.threads;
        out->target_patch_nodes = B.P.target;
        out->shared_bytes = static_cast<int32_t>(B.P.smem);
        out->max_cluster_stages = B.P.max_stages;
        out->resident_clusters = B.resident;
        out->colours_per_sync = 1;
        out->autotune_candidates = static_cast<int32_t>(std::min<size_t>(B.candidates.size(), 8));
        for (int k = 0; k < out->autotune_candidates; ++k) {
            out->candidate_patch_nodes[k] = B.candidates[k];
            out->candidate_ms_per_step[k] = B.candidate_ms[k];
            out->candidate_block_threads[k] = B.candidate_threads[k];
        }
    });
}

double swb_batch_last_step_ms(const swb_batch* batch) { return batch ? batch->b.last_ms : 0.0; }

}  // extern "C"
