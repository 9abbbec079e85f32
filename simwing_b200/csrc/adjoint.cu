// Differentiable rollouts: the forward / backward pair of the adjoint.
//
// forward: `steps` steps from the structure's committed state (which it
// leaves untouched) on the structure's own schedule, keeping a checkpoint of
// the state every `interval` steps, then the loss
//     L = sum_i w_i |x_i(T) - target_i|^2 / sum_i w_i
// over the world positions at the end.
// backward: per segment of `interval` steps, last first: the segment is
// stepped again from its checkpoint by the taping kernel, which records the
// inputs of every projection, line iteration and pilot finish, then the
// reverse kernel runs the segment's steps backwards, carrying the adjoint of
// the state (positions, velocities, pilot) and accumulating the parameter
// adjoints (every constraint's rest length and compliance, every dihedral's
// compliance, every suspension segment's rest length, the pilot mass).
// The re-centring shift of the frame is constant in each step, so the
// adjoint of a position passes through it unchanged.
#include "structure_impl.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace swb {
namespace {

uint32_t al16(uint32_t v) { return (v + 15u) & ~15u; }

template <class T>
T* ralloc(std::vector<void*>& owned, size_t count) {
    void* p = nullptr;
    cuda_check(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)), "cudaMalloc (rollout)");
    owned.push_back(p);
    return static_cast<T*>(p);
}

struct StateBuf {
    float4* pos = nullptr;
    float4* vel = nullptr;
    float4* prev = nullptr;
    DevPayloadState* pay = nullptr;
    double* origin = nullptr;
};

}  // namespace

struct RolloutImpl {
    StructureImpl* S = nullptr;
    int steps = 0, interval = 16, segments = 0;
    std::vector<void*> owned;
    std::vector<StateBuf> ck, sg;      // checkpoints (segments + 1), segment states (interval + 1)
    std::vector<TapeStep> tape;        // per step of a segment
    int tape_iterations = -1;
    bool tape_lines = false;           // the tapes hold line-line contact arrays
    std::vector<ClusterInstance> rec_host;  // d_records' host copy
    bool rec_lines = false;            // d_records carry the structure's line-line contact
    bool fwd_lines = false;            // the last forward ran with line-line contact
    static constexpr uint32_t kLineTapeCap = 4096;  // line-line candidates a tape step holds
    float* line_jac = nullptr;  // per-iteration line-iteration Jacobians of the reverse step
    ClusterInstance* d_records = nullptr;  // step k of a segment: sg[k] -> sg[k + 1]
    AdjointPilot* d_pilot = nullptr;
    int pilot_segments = 0, pilot_slots = 0;
    float4* xb[2] = {};
    float4* vb[2] = {};
    float* pb[2] = {};
    float4* fbar = nullptr;
    double* g_rest0 = nullptr;
    double* g_comp0 = nullptr;
    double* g_comp1 = nullptr;
    double* g_seg = nullptr;
    double* g_mass = nullptr;
    uint32_t r0 = 0, r1 = 0, rs = 0;
    uint32_t smem = 0;
    AdjointParams base{};
    swb_step_settings settings{};
    bool have_forward = false;
    std::vector<float4> xbar_T;        // slot order
    std::vector<double> final_world;   // definition order, xyz
    double loss = 0.0;
    double forward_ms = 0.0, backward_ms = 0.0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    ~RolloutImpl() {
        if (S) cudaSetDevice(S->device);
        for (void* p : owned) cudaFree(p);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
    }

    StateBuf state_buffers() {
        const size_t N = S->def.nodes.size();
        StateBuf b;
        b.pos = ralloc<float4>(owned, N);
        b.vel = ralloc<float4>(owned, N);
        b.prev = ralloc<float4>(owned, N);
        b.pay = ralloc<DevPayloadState>(owned, 1);
        b.origin = ralloc<double>(owned, 3);
        return b;
    }

    void copy_state(const StateBuf& from, const StateBuf& to) {
        const size_t N = S->def.nodes.size();
        cudaStream_t st = S->stream;
        cuda_check(cudaMemcpyAsync(to.pos, from.pos, N * sizeof(float4), cudaMemcpyDeviceToDevice, st), "copy");
        cuda_check(cudaMemcpyAsync(to.vel, from.vel, N * sizeof(float4), cudaMemcpyDeviceToDevice, st), "copy");
        cuda_check(cudaMemcpyAsync(to.pay, from.pay, sizeof(DevPayloadState), cudaMemcpyDeviceToDevice, st), "copy");
        cuda_check(cudaMemcpyAsync(to.origin, from.origin, 3 * sizeof(double), cudaMemcpyDeviceToDevice, st), "copy");
    }

    void build(StructureImpl& s, int n_steps, int every) {
        S = &s;
        if (!S->cluster_mode)
            raise(SWB_UNSUPPORTED, "differentiable rollouts need the cluster schedule (the mesh does not fit one)");
        if (S->momentum_guard)
            raise(SWB_UNSUPPORTED, "differentiable rollouts of free structures (momentum guard) are not available");
        if (!S->def.membranes.empty())
            raise(SWB_UNSUPPORTED, "differentiable rollouts of structures with membrane elements are not available");
        if (S->def.has_contact)
            raise(SWB_UNSUPPORTED, "differentiable rollouts of structures with fabric self-contact are not available");
        if (n_steps < 1) raise(SWB_INVALID_ARGUMENT, "a rollout needs at least one step");
        if (every < 1) raise(SWB_INVALID_ARGUMENT, "checkpoint interval must be positive");
        steps = n_steps;
        interval = std::min(every, n_steps);
        segments = (steps + interval - 1) / interval;
        cuda_check(cudaSetDevice(S->device), "cudaSetDevice");
        cuda_check(cudaEventCreate(&ev0), "cudaEventCreate");
        cuda_check(cudaEventCreate(&ev1), "cudaEventCreate");
        const ClusterSchedule& cs = S->csched;
        r0 = static_cast<uint32_t>(cs.kinds[0].ab.size());
        r1 = static_cast<uint32_t>(cs.kinds[1].ab.size());
        rs = static_cast<uint32_t>(cs.seam_ab.size());
        const size_t N = S->def.nodes.size();
        for (int c = 0; c <= segments; ++c) ck.push_back(state_buffers());
        for (int k = 0; k <= interval; ++k) sg.push_back(state_buffers());
        // the pilot as the adjoint sees it: distinct endpoint nodes as slots
        AdjointPilot ap{};
        if (S->def.has_suspension) {
            const DevPayloadDef& d = S->payload_def_host;
            std::vector<int> nodes;
            auto slot_of = [&](int node) {
                if (node < 0) return -1;
                auto it = std::find(nodes.begin(), nodes.end(), node);
                if (it != nodes.end()) return static_cast<int>(it - nodes.begin());
                nodes.push_back(node);
                return static_cast<int>(nodes.size() - 1);
            };
            ap.segments = d.segments;
            for (int k = 0; k < d.segments; ++k) {
                ap.from_slot[k] = slot_of(d.from_node[k]);
                ap.to_slot[k] = slot_of(d.to_node[k]);
                ap.from_point[k] = d.from_point[k];
                ap.to_point[k] = d.to_point[k];
                ap.rest[k] = d.rest[k];
                ap.stiffness[k] = d.stiffness[k];
                ap.damping[k] = d.damping[k];
            }
            if (nodes.size() > 16) raise(SWB_UNSUPPORTED, "more than 16 suspension endpoint nodes");
            ap.slots = static_cast<int>(nodes.size());
            for (size_t q = 0; q < nodes.size(); ++q) {
                ap.slot_node[q] = nodes[q];
                ap.slot_w[q] = S->inv_mass[S->susp_base + nodes[q]];
            }
            for (int k = 0; k < d.hang_points; ++k) ap.hang_local[k] = d.hang_local[k];
            ap.com_local = d.com_local;
            ap.inertia = d.inertia;
            ap.mass = d.mass;
            ap.min_length = d.min_length;
        }
        pilot_segments = ap.segments;
        pilot_slots = ap.slots;
        d_pilot = ralloc<AdjointPilot>(owned, 1);
        cuda_check(cudaMemcpyAsync(d_pilot, &ap, sizeof(ap), cudaMemcpyHostToDevice, S->stream), "pilot upload");
        // records of a segment's steps
        std::vector<ClusterInstance> rec(interval);
        for (int k = 0; k < interval; ++k) {
            ClusterInstance c = S->cluster_base;
            c.pos_in = sg[k].pos; c.vel_in = sg[k].vel;
            c.pos_out = sg[k + 1].pos; c.vel_out = sg[k + 1].vel; c.prev_out = sg[k + 1].prev;
            c.force = S->d_force;
            c.tri_offsets = S->d_tri_off; c.tri_list = S->d_tri_list; c.tri = S->d_tri;
            c.susp_cta = S->def.has_suspension ? S->susp_owner : -1;
            c.payload_def = S->d_payload_def;
            c.payload_in = sg[k].pay; c.payload_out = sg[k + 1].pay;
            c.origin_in = sg[k].origin; c.origin_out = sg[k + 1].origin;
            c.status = S->d_control->status;
            c.recentre = S->def.has_suspension ? 1 : 0;
            rec[k] = c;
        }
        rec_host = rec;
        d_records = ralloc<ClusterInstance>(owned, rec.size());
        cuda_check(cudaMemcpyAsync(d_records, rec.data(), rec.size() * sizeof(ClusterInstance), cudaMemcpyHostToDevice,
                                   S->stream), "records upload");
        for (int k = 0; k < 2; ++k) {
            xb[k] = ralloc<float4>(owned, N);
            vb[k] = ralloc<float4>(owned, N);
            pb[k] = ralloc<float>(owned, 16);
        }
        fbar = ralloc<float4>(owned, N);
        g_rest0 = ralloc<double>(owned, r0);
        g_comp0 = ralloc<double>(owned, r0);
        g_comp1 = ralloc<double>(owned, r1);
        g_seg = ralloc<double>(owned, 8);
        g_mass = ralloc<double>(owned, 1);
        // reverse kernel shared memory
        const uint32_t P = cs.max_patch;
        const uint32_t m0 = cs.kinds[0].max_cta_records, m1 = cs.kinds[1].max_cta_records;
        uint32_t off = 0;
        base.smem_xb = off; off = al16(off + P * 16u);
        base.smem_vb = off; off = al16(off + P * 16u);
        base.smem_lam0 = off; off = al16(off + m0 * 4u);
        base.smem_lam1 = off; off = al16(off + m1 * 4u);
        base.smem_acc0r = off; off = al16(off + m0 * 4u);
        base.smem_acc0c = off; off = al16(off + m0 * 4u);
        base.smem_acc1c = off; off = al16(off + m1 * 4u);
        base.smem_offsets = off; off = al16(off + (cs.kinds[0].stages + cs.kinds[1].stages + 2) * 4u);
        smem = off;
        cudaDeviceProp prop{};
        cuda_check(cudaGetDeviceProperties(&prop, S->device), "cudaGetDeviceProperties");
        const size_t limit = dynamic_smem_limit(prop);
        if (smem > limit)
            raise(SWB_UNSUPPORTED, "the reverse sweep needs " + std::to_string(smem) +
                                       " B of shared memory per CTA; build the structure with more cluster CTAs");
        cuda_check(adjoint_kernel_limits(static_cast<int>(limit), S->G > 8), "adjoint kernel limits");
        cuda_check(tape_kernel_limits(static_cast<int>(limit), S->G > 8), "taping kernel limits");
        cuda_check(cudaStreamSynchronize(S->stream), "rollout setup");
    }

    // The step records carry the structure's line-line contact when it is
    // set (its candidate lists are the structure's scratch).
    void sync_records() {
        const bool want = S->line_contact;
        if (want == rec_lines) return;
        for (ClusterInstance& c : rec_host) c.lines = want ? S->d_lines : nullptr;
        cuda_check(cudaMemcpyAsync(d_records, rec_host.data(), rec_host.size() * sizeof(ClusterInstance),
                                   cudaMemcpyHostToDevice, S->stream),
                   "records upload");
        rec_lines = want;
    }

    void ensure_tapes(int iterations) {
        if (!tape.empty() && tape_iterations == iterations && tape_lines == S->line_contact) return;
        for (TapeStep& t : tape)
            for (void* q : {static_cast<void*>(t.dist), static_cast<void*>(t.dih), static_cast<void*>(t.seam),
                            static_cast<void*>(t.line), static_cast<void*>(t.finish), static_cast<void*>(t.ground),
                            static_cast<void*>(t.line_pairs), static_cast<void*>(t.line_level_off),
                            static_cast<void*>(t.line_count), static_cast<void*>(t.line_in)}) {
                if (!q) continue;
                cudaFree(q);
                owned.erase(std::remove(owned.begin(), owned.end(), q), owned.end());
            }
        tape.clear();
        const size_t it = static_cast<size_t>(std::max(iterations, 1));
        for (int k = 0; k < interval; ++k) {
            TapeStep t{};
            t.dist = ralloc<float4>(owned, it * 2 * r0);
            t.dih = ralloc<float4>(owned, it * 4 * r1);
            t.seam = ralloc<float4>(owned, 2 * static_cast<size_t>(rs));
            t.line = ralloc<PilotTape>(owned, it);
            t.finish = ralloc<PilotTape>(owned, 1);
            t.ground = ralloc<uint8_t>(owned, it * S->def.nodes.size());
            if (S->line_contact) {
                t.line_cap = kLineTapeCap;
                t.line_pairs = ralloc<uint32_t>(owned, kLineTapeCap);
                t.line_level_off = ralloc<uint32_t>(owned, kLineTapeCap + 1);
                t.line_count = ralloc<uint32_t>(owned, 2);
                cuda_check(cudaMemsetAsync(t.line_count, 0, 2 * sizeof(uint32_t), S->stream), "memset");
                t.line_in = ralloc<float4>(owned, it * kLineTapeCap * 4);
            }
            t.r0 = r0;
            t.r1 = r1;
            t.rs = rs;
            t.pilot = d_pilot;
            tape.push_back(t);
        }
        if (line_jac) {
            cudaFree(line_jac);
            owned.erase(std::remove(owned.begin(), owned.end(), static_cast<void*>(line_jac)), owned.end());
            line_jac = nullptr;
        }
        if (S->def.has_suspension) {
            const size_t nin = 8 + 2 * static_cast<size_t>(pilot_segments) + 3 * static_cast<size_t>(pilot_slots);
            const size_t nout = 7 + static_cast<size_t>(pilot_segments) + 3 * static_cast<size_t>(pilot_slots);
            line_jac = ralloc<float>(owned, it * nin * nout);
        }
        tape_iterations = iterations;
        tape_lines = S->line_contact;
    }

    ClusterParams step_params(int k, const TapeStep* t) const {
        ClusterParams cp = S->cparams;
        const double dt = settings.time_step;
        cp.instances = d_records + k;
        cp.ctas = S->G;
        cp.dt = static_cast<float>(dt);
        cp.inv_dt = static_cast<float>(1.0 / dt);
        cp.inv_dt2 = static_cast<float>(1.0 / (dt * dt));
        cp.damping = static_cast<float>(std::exp(-settings.velocity_damping * dt));
        cp.damping_loss = static_cast<float>(-std::expm1(-settings.velocity_damping * dt));
        cp.gravity = make_float3(settings.gravity.x, settings.gravity.y, settings.gravity.z);
        cp.ref_velocity = make_float3(settings.damping_reference_velocity.x, settings.damping_reference_velocity.y,
                                      settings.damping_reference_velocity.z);
        cp.iterations = settings.constraint_iterations;
        if (t) cp.tape = *t;
        return cp;
    }

    cudaLaunchConfig_t config(uint32_t dyn, cudaLaunchAttribute* attr) const {
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = static_cast<unsigned>(S->G);
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(static_cast<unsigned>(S->G));
        cfg.blockDim = dim3(static_cast<unsigned>(S->threads));
        cfg.dynamicSmemBytes = dyn;
        cfg.stream = S->stream;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        return cfg;
    }

    void run_segment_forward(int c, bool with_tape) {
        const int K = std::min(interval, steps - c * interval);
        copy_state(ck[c], sg[0]);
        cudaLaunchAttribute attr[1];
        const cudaLaunchConfig_t cfg = config(S->cluster_smem, attr);
        for (int k = 0; k < K; ++k) {
            const ClusterParams cp = step_params(k, with_tape ? &tape[k] : nullptr);
            cuda_check(with_tape ? tape_kernel_launch(cfg, cp) : plain_cluster_launch(cfg, cp), "rollout step");
        }
        if (!with_tape) copy_state(sg[K], ck[c + 1]);
    }

    void check_status() {
        std::string message;
        const swb_status st = S->read_status(message);
        if (st != SWB_OK) raise(st, "rollout: " + message);
    }

    void forward(const swb_step_settings& st, const double* target, const double* weights, double* out_loss) {
        forward_launch(st, target, weights);
        forward_collect(target, weights, out_loss);
    }

    // The forward's launches on the structure's stream (no wait for them).
    void forward_launch(const swb_step_settings& st, const double* target, const double* weights) {
        S->validate_settings(st);
        if (st.cable_sweep_pairs != 0)
            raise(SWB_UNSUPPORTED, "differentiable rollouts with load-path cable sweep pairs are not available");
        if (st.substeps != 1) raise(SWB_UNSUPPORTED, "differentiable rollouts take one substep per step");
        if (S->cparams.ground && S->cparams.ground_friction > 0.0f)
            raise(SWB_UNSUPPORTED, "differentiable rollouts take a frictionless ground plane");
        const size_t N = S->def.nodes.size();
        double wsum = 0.0;
        for (size_t i = 0; i < N; ++i) {
            if (!std::isfinite(weights[i]) || weights[i] < 0.0)
                raise(SWB_INVALID_ARGUMENT, "weights must be finite and >= 0");
            if (!std::isfinite(target[3 * i]) || !std::isfinite(target[3 * i + 1]) || !std::isfinite(target[3 * i + 2]))
                raise(SWB_INVALID_ARGUMENT, "target positions must be finite");
            wsum += weights[i];
        }
        if (!(wsum > 0.0)) raise(SWB_INVALID_ARGUMENT, "weights must not all be zero");
        settings = st;
        have_forward = false;
        cuda_check(cudaSetDevice(S->device), "cudaSetDevice");
        sync_records();
        fwd_lines = S->line_contact;
        if (S->pressure_dirty) S->upload_pressure();
        if (S->forces_dirty) S->upload_forces();
        cuda_check(cudaMemsetAsync(S->d_control, 0, offsetof(Control, shift), S->stream), "control reset");
        const int cur = S->cur;
        const StateBuf committed{S->d_pos[cur], S->d_vel[cur], S->d_prev[cur], S->d_payload[cur], S->d_origin[cur]};
        copy_state(committed, ck[0]);
        cuda_check(cudaEventRecord(ev0, S->stream), "event");
        for (int c = 0; c < segments; ++c) run_segment_forward(c, false);
        cuda_check(cudaEventRecord(ev1, S->stream), "event");
    }

    // Waits for the forward's launches; the loss and the final state.
    void forward_collect(const double* target, const double* weights, double* out_loss) {
        const size_t N = S->def.nodes.size();
        double wsum = 0.0;
        for (size_t i = 0; i < N; ++i) wsum += weights[i];
        check_status();
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ev0, ev1);
        forward_ms = ms;
        // loss on the world positions of the final state
        std::vector<float4> pos(N);
        double origin[3];
        cuda_check(cudaMemcpyAsync(pos.data(), ck[segments].pos, N * sizeof(float4), cudaMemcpyDeviceToHost, S->stream),
                   "read");
        cuda_check(cudaMemcpyAsync(origin, ck[segments].origin, sizeof(origin), cudaMemcpyDeviceToHost, S->stream),
                   "read");
        cuda_check(cudaStreamSynchronize(S->stream), "read");
        xbar_T.assign(N, make_float4(0, 0, 0, 0));
        final_world.assign(3 * N, 0.0);
        double L = 0.0;
        for (size_t i = 0; i < N; ++i) {
            const uint32_t s = S->slot_of_node[i];
            const double w[3] = {origin[0] + pos[s].x, origin[1] + pos[s].y, origin[2] + pos[s].z};
            double d2 = 0.0;
            float g[3];
            for (int k = 0; k < 3; ++k) {
                final_world[3 * i + k] = w[k];
                const double d = w[k] - target[3 * i + k];
                d2 += d * d;
                g[k] = static_cast<float>(2.0 * weights[i] * d / wsum);
            }
            L += weights[i] * d2;
            xbar_T[s] = make_float4(g[0], g[1], g[2], 0.0f);
        }
        loss = L / wsum;
        if (out_loss) *out_loss = loss;
        have_forward = true;
    }

    void backward(const swb_rollout_gradient* out) {
        backward_launch();
        backward_collect(out);
    }

    // The backward's launches on the structure's stream (no wait for them).
    void backward_launch() {
        if (!have_forward) raise(SWB_INVALID_ARGUMENT, "backward needs a forward first");
        if (S->line_contact != fwd_lines)
            raise(SWB_INVALID_ARGUMENT, "line-line contact was switched between the forward and the backward");
        cuda_check(cudaSetDevice(S->device), "cudaSetDevice");
        sync_records();
        const size_t N = S->def.nodes.size();
        ensure_tapes(settings.constraint_iterations);
        cudaStream_t st = S->stream;
        cuda_check(cudaMemsetAsync(S->d_control, 0, offsetof(Control, shift), st), "control reset");
        cuda_check(cudaMemcpyAsync(xb[0], xbar_T.data(), N * sizeof(float4), cudaMemcpyHostToDevice, st), "upload");
        cuda_check(cudaMemsetAsync(vb[0], 0, N * sizeof(float4), st), "memset");
        cuda_check(cudaMemsetAsync(pb[0], 0, 16 * sizeof(float), st), "memset");
        cuda_check(cudaMemsetAsync(g_rest0, 0, std::max<size_t>(r0, 1) * sizeof(double), st), "memset");
        cuda_check(cudaMemsetAsync(g_comp0, 0, std::max<size_t>(r0, 1) * sizeof(double), st), "memset");
        cuda_check(cudaMemsetAsync(g_comp1, 0, std::max<size_t>(r1, 1) * sizeof(double), st), "memset");
        cuda_check(cudaMemsetAsync(g_seg, 0, 8 * sizeof(double), st), "memset");
        cuda_check(cudaMemsetAsync(g_mass, 0, sizeof(double), st), "memset");
        const double dt = settings.time_step;
        AdjointParams ap = base;
        ap.fbar = fbar;
        ap.line_jac = line_jac;
        ap.g_rest0 = g_rest0;
        ap.g_comp0 = g_comp0;
        ap.g_comp1 = g_comp1;
        ap.g_seg_rest = g_seg;
        ap.g_mass = g_mass;
        ap.ctas = S->G;
        ap.dt = static_cast<float>(dt);
        ap.inv_dt = static_cast<float>(1.0 / dt);
        ap.inv_dt2 = static_cast<float>(1.0 / (dt * dt));
        ap.damping = static_cast<float>(std::exp(-settings.velocity_damping * dt));
        ap.gravity = make_float3(settings.gravity.x, settings.gravity.y, settings.gravity.z);
        ap.iterations = settings.constraint_iterations;
        ap.ground = S->cparams.ground;
        ap.ground_normal = S->cparams.ground_normal;
        cudaLaunchAttribute attr[1];
        const cudaLaunchConfig_t cfg = config(smem, attr);
        int cur = 0;
        cuda_check(cudaEventRecord(ev0, st), "event");
        for (int c = segments - 1; c >= 0; --c) {
            run_segment_forward(c, true);
            const int K = std::min(interval, steps - c * interval);
            for (int k = K - 1; k >= 0; --k) {
                ap.inst = d_records + k;
                ap.tape = tape[k];
                ap.xb_out = xb[cur]; ap.vb_out = vb[cur]; ap.pb_out = pb[cur];
                ap.xb_in = xb[1 - cur]; ap.vb_in = vb[1 - cur]; ap.pb_in = pb[1 - cur];
                cuda_check(adjoint_kernel_launch(cfg, ap), "reverse step");
                cur = 1 - cur;
            }
        }
        cuda_check(cudaEventRecord(ev1, st), "event");
    }

    // Waits for the backward's launches; the gradients in definition order.
    void backward_collect(const swb_rollout_gradient* out) {
        cudaStream_t st = S->stream;
        check_status();
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ev0, ev1);
        backward_ms = ms;
        // parameter adjoints back to definition order
        std::vector<double> rest0(r0), comp0(r0), comp1(r1), seg(8);
        double mass = 0.0;
        if (r0) {
            cuda_check(cudaMemcpyAsync(rest0.data(), g_rest0, r0 * sizeof(double), cudaMemcpyDeviceToHost, st), "read");
            cuda_check(cudaMemcpyAsync(comp0.data(), g_comp0, r0 * sizeof(double), cudaMemcpyDeviceToHost, st), "read");
        }
        if (r1)
            cuda_check(cudaMemcpyAsync(comp1.data(), g_comp1, r1 * sizeof(double), cudaMemcpyDeviceToHost, st), "read");
        cuda_check(cudaMemcpyAsync(seg.data(), g_seg, 8 * sizeof(double), cudaMemcpyDeviceToHost, st), "read");
        cuda_check(cudaMemcpyAsync(&mass, g_mass, sizeof(double), cudaMemcpyDeviceToHost, st), "read");
        cuda_check(cudaStreamSynchronize(st), "read");
        bool finite = std::isfinite(mass);
        for (const std::vector<double>* v : {&rest0, &comp0, &comp1, &seg})
            for (double x : *v) finite = finite && std::isfinite(x);
        if (out) write_gradient(out, rest0, comp0, comp1, seg, mass);
        if (!finite)
            raise(SWB_NON_FINITE,
                  "the gradient is not finite: the FP32 reverse sweep overflowed (the rollout's sensitivity to its "
                  "parameters outgrew FP32's range over its length, as an unstable flutter makes it); the output "
                  "arrays hold the values reached");
    }

    void write_gradient(const swb_rollout_gradient* out, const std::vector<double>& rest0,
                        const std::vector<double>& comp0, const std::vector<double>& comp1,
                        const std::vector<double>& seg, double mass) const {
        const ClusterSchedule& cs = S->csched;
        const size_t M = S->def.constraints.size(), H = S->def.dihedrals.size();
        if (out->d_rest || out->d_compliance)
            for (uint32_t r = 0; r < r0; ++r) {
                const uint32_t i = cs.kinds[0].def_index[r];
                if (i >= M) continue;
                if (out->d_rest) out->d_rest[i] = rest0[r];
                if (out->d_compliance) out->d_compliance[i] = comp0[r];
            }
        if (out->d_dihedral_compliance)
            for (uint32_t r = 0; r < r1; ++r) {
                const uint32_t i = cs.kinds[1].def_index[r];
                if (i < H) out->d_dihedral_compliance[i] = comp1[r];
            }
        if (out->d_segment_rest)
            for (size_t k = 0; k < S->segment_order.size(); ++k) out->d_segment_rest[S->segment_order[k]] = seg[k];
        if (out->d_pilot_mass) *out->d_pilot_mass = S->def.has_suspension ? mass : 0.0;
    }
};

}  // namespace swb

struct swb_rollout {
    swb::RolloutImpl r;
};

using namespace swb;

extern "C" {

swb_status swb_rollout_create(swb_structure* structure, int32_t steps, int32_t checkpoint_interval,
                              swb_rollout** out) {
    return guarded([&] {
        if (!structure || !out) raise(SWB_INVALID_ARGUMENT, "null argument");
        auto h = std::make_unique<swb_rollout>();
        h->r.build(structure->s, steps, checkpoint_interval > 0 ? checkpoint_interval : 16);
        *out = h.release();
    });
}

void swb_rollout_destroy(swb_rollout* rollout) { delete rollout; }

swb_status swb_rollout_forward(swb_rollout* rollout, const swb_step_settings* settings, const double* target_xyz,
                               const double* weights, double* loss) {
    return guarded([&] {
        if (!rollout || !settings || !target_xyz || !weights) raise(SWB_INVALID_ARGUMENT, "null argument");
        rollout->r.forward(*settings, target_xyz, weights, loss);
    });
}

swb_status swb_rollout_backward(swb_rollout* rollout, const swb_rollout_gradient* gradient) {
    return guarded([&] {
        if (!rollout) raise(SWB_INVALID_ARGUMENT, "null argument");
        rollout->r.backward(gradient);
    });
}

swb_status swb_rollout_forward_many(swb_rollout* const* rollouts, uint64_t count, const swb_step_settings* settings,
                                    const double* const* targets_xyz, const double* const* weights,
                                    double* losses, int32_t* statuses) {
    return guarded([&] {
        if ((!rollouts || !targets_xyz || !weights) && count) raise(SWB_INVALID_ARGUMENT, "null argument");
        if (!settings) raise(SWB_INVALID_ARGUMENT, "null argument");
        for (uint64_t k = 0; k < count; ++k)
            if (!rollouts[k] || !targets_xyz[k] || !weights[k]) raise(SWB_INVALID_ARGUMENT, "null argument");
        // every rollout's launches first, each on its structure's stream, so
        // that the structures run side by side; then each is waited for
        std::vector<swb_status> st(count, SWB_OK);
        std::vector<std::string> msg(count);
        auto run = [&](uint64_t k, auto&& body) {
            if (st[k] != SWB_OK) return;
            try {
                body();
            } catch (const Error& e) {
                st[k] = e.status;
                msg[k] = e.what();
            }
        };
        for (uint64_t k = 0; k < count; ++k)
            run(k, [&] { rollouts[k]->r.forward_launch(*settings, targets_xyz[k], weights[k]); });
        for (uint64_t k = 0; k < count; ++k)
            run(k, [&] { rollouts[k]->r.forward_collect(targets_xyz[k], weights[k], losses ? losses + k : nullptr); });
        for (uint64_t k = 0; k < count; ++k) {
            if (statuses) statuses[k] = st[k];
        }
        for (uint64_t k = 0; k < count; ++k)
            if (st[k] != SWB_OK) raise(st[k], "rollout " + std::to_string(k) + ": " + msg[k]);
    });
}

swb_status swb_rollout_backward_many(swb_rollout* const* rollouts, uint64_t count,
                                     const swb_rollout_gradient* gradients, int32_t* statuses) {
    return guarded([&] {
        if (!rollouts && count) raise(SWB_INVALID_ARGUMENT, "null argument");
        for (uint64_t k = 0; k < count; ++k)
            if (!rollouts[k]) raise(SWB_INVALID_ARGUMENT, "null argument");
        std::vector<swb_status> st(count, SWB_OK);
        std::vector<std::string> msg(count);
        auto run = [&](uint64_t k, auto&& body) {
            if (st[k] != SWB_OK) return;
            try {
                body();
            } catch (const Error& e) {
                st[k] = e.status;
                msg[k] = e.what();
            }
        };
        for (uint64_t k = 0; k < count; ++k) run(k, [&] { rollouts[k]->r.backward_launch(); });
        for (uint64_t k = 0; k < count; ++k)
            run(k, [&] { rollouts[k]->r.backward_collect(gradients ? gradients + k : nullptr); });
        for (uint64_t k = 0; k < count; ++k) {
            if (statuses) statuses[k] = st[k];
        }
        for (uint64_t k = 0; k < count; ++k)
            if (st[k] != SWB_OK) raise(st[k], "rollout " + std::to_string(k) + ": " + msg[k]);
    });
}

swb_status swb_rollout_final_positions(const swb_rollout* rollout, double* xyz, uint64_t count) {
    return guarded([&] {
        if (!rollout || !xyz) raise(SWB_INVALID_ARGUMENT, "null argument");
        const RolloutImpl& r = rollout->r;
        if (!r.have_forward) raise(SWB_INVALID_ARGUMENT, "no forward has run");
        if (count != r.final_world.size() / 3) raise(SWB_INVALID_ARGUMENT, "count must equal the node count");
        std::memcpy(xyz, r.final_world.data(), r.final_world.size() * sizeof(double));
    });
}

double swb_rollout_forward_ms(const swb_rollout* rollout) { return rollout ? rollout->r.forward_ms : 0.0; }
double swb_rollout_backward_ms(const swb_rollout* rollout) { return rollout ? rollout->r.backward_ms : 0.0; }

}  // extern "C"
