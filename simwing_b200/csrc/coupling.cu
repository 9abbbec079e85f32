// Coupling callers with device-resident loads: the structural side of
// simwing::fsi::ConservativeMacroStepCoupling (src/fsi/coupling.cpp:806-911).
// A flow solver that keeps its interface impulses (or endpoint tractions) in
// device memory hands them over without a host round trip: one kernel turns
// them into the step's nodal forces, summed per structure node in FP64 in the
// order the reference's addExternalForce loop adds them (binding order), on
// top of the loads already pending; the structure then steps on that force
// buffer.
#include "common.h"
#include "structure_impl.h"

#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

struct swb_coupling {
    swb_structure* structure = nullptr;
    uint64_t bindings = 0;
    std::vector<uint64_t> node_of_binding;
    // per structure slot, the bindings that load it (binding order)
    uint32_t* d_offsets = nullptr;  // [slots + 1]
    uint32_t* d_items = nullptr;    // [bindings]
    double* d_pending = nullptr;    // [slots][3] the loads pending before the call
    double* d_applied = nullptr;    // [3] the total applied force (node order)
    int* d_flag = nullptr;          // 1: a non-finite load
    std::vector<double> pending_host;  // staging of the pending loads
    std::vector<void*> owned;
    ~swb_coupling() {
        for (void* p : owned) cudaFree(p);
    }
};

namespace swb {
namespace {

// Forces of every slot: pending + sum over its bindings of the binding's
// average load (impulse / duration, or the mean of the start and end loads).
__global__ void gather_loads_kernel(uint32_t slots, const uint32_t* __restrict__ offsets,
                                    const uint32_t* __restrict__ items, const double* __restrict__ pending,
                                    const double* __restrict__ a, const double* __restrict__ b, double scale,
                                    int endpoints, float4* __restrict__ force, double* __restrict__ total64,
                                    int* flag) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= slots) return;
    double f[3] = {pending[3 * s], pending[3 * s + 1], pending[3 * s + 2]};
    bool bad = false;
    for (uint32_t k = offsets[s]; k < offsets[s + 1]; ++k) {
        const uint32_t i = items[k];
        for (int c = 0; c < 3; ++c) {
            const double x = a[3 * static_cast<size_t>(i) + c];
            double load;
            if (endpoints) {
                const double y = b[3 * static_cast<size_t>(i) + c];
                bad = bad || !isfinite(x) || !isfinite(y);
                load = 0.5 * (x + y);
            } else {
                bad = bad || !isfinite(x);
                load = x * scale;
            }
            bad = bad || !isfinite(load);
            f[c] += load;
        }
    }
    if (bad) atomicOr(flag, 1);
    force[s] = make_float4(static_cast<float>(f[0]), static_cast<float>(f[1]), static_cast<float>(f[2]), 0.0f);
    total64[3 * s] = f[0];
    total64[3 * s + 1] = f[1];
    total64[3 * s + 2] = f[2];
}

// Total of the applied forces: each thread sums a contiguous run of nodes in
// node order, then the partial sums are added in thread order (one block, a
// fixed order: the same total on every call).
__global__ void applied_total_kernel(uint64_t nodes, const uint32_t* __restrict__ slot_of_node,
                                     const double* __restrict__ total64, double* out) {
    __shared__ double part[3][1024];
    const uint32_t t = threadIdx.x, threads = blockDim.x;
    const uint64_t chunk = (nodes + threads - 1) / threads;
    const uint64_t start = static_cast<uint64_t>(t) * chunk;
    const uint64_t lo = start < nodes ? start : nodes;
    const uint64_t hi = lo + chunk < nodes ? lo + chunk : nodes;
    double x = 0.0, y = 0.0, z = 0.0;
    for (uint64_t n = lo; n < hi; ++n) {
        const uint32_t s = slot_of_node[n];
        x += total64[3 * s];
        y += total64[3 * s + 1];
        z += total64[3 * s + 2];
    }
    part[0][t] = x;
    part[1][t] = y;
    part[2][t] = z;
    __syncthreads();
    if (t < 3) {
        double sum = 0.0;
        for (uint32_t k = 0; k < threads; ++k) sum += part[t][k];
        out[t] = sum;
    }
}

template <class T>
T* alloc(std::vector<void*>& owned, size_t n) {
    void* p = nullptr;
    cuda_check(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)), "cudaMalloc (coupling)");
    owned.push_back(p);
    return static_cast<T*>(p);
}

swb_status advance(swb_coupling* c, const double* a, const double* b, double scale, int endpoints,
                   const swb_step_settings* settings, swb_diagnostics* out) {
    return guarded([&] {
        StructureImpl& S = c->structure->s;
        S.validate_settings(*settings);
        cuda_check(cudaSetDevice(S.device), "cudaSetDevice");
        const uint32_t slots = static_cast<uint32_t>(S.def.nodes.size());
        // the loads pending before the call, by slot (cleared when none is)
        const bool any_pending = std::any_of(S.pending.begin(), S.pending.end(), [](const swb_vec3& f) {
            return f.x != 0.0 || f.y != 0.0 || f.z != 0.0;
        });
        if (any_pending) {
            c->pending_host.assign(3 * static_cast<size_t>(slots), 0.0);
            for (uint64_t n = 0; n < S.def.nodes.size(); ++n) {
                const uint32_t s = S.slot_of_node[n];
                c->pending_host[3 * s] = S.pending[n].x;
                c->pending_host[3 * s + 1] = S.pending[n].y;
                c->pending_host[3 * s + 2] = S.pending[n].z;
            }
            cuda_check(cudaMemcpy(c->d_pending, c->pending_host.data(), c->pending_host.size() * sizeof(double),
                                  cudaMemcpyHostToDevice), "pending upload");
        } else {
            cuda_check(cudaMemsetAsync(c->d_pending, 0, 3 * static_cast<size_t>(slots) * sizeof(double), S.stream),
                       "memset");
        }
        cuda_check(cudaMemsetAsync(c->d_flag, 0, sizeof(int), S.stream), "memset");
        double* total64 = c->d_pending;  // overwritten in place, slot by slot
        gather_loads_kernel<<<(slots + 255) / 256, 256, 0, S.stream>>>(slots, c->d_offsets, c->d_items,
                                                                        c->d_pending, a, b, scale, endpoints,
                                                                        S.d_force, total64, c->d_flag);
        cuda_check(cudaGetLastError(), "gather_loads_kernel");
        int flag = 0;
        cuda_check(cudaMemcpyAsync(&flag, c->d_flag, sizeof(int), cudaMemcpyDeviceToHost, S.stream), "read");
        cuda_check(cudaStreamSynchronize(S.stream), "gather");
        if (flag) {
            S.forces_dirty = true;  // the device buffer no longer holds the pending loads
            raise(SWB_INVALID_ARGUMENT, "time-integrated transfer has invalid nodal bindings or non-finite loads");
        }
        S.device_forces = true;
        try {
            S.step(*settings, 1, out);
        } catch (...) {
            S.device_forces = false;
            S.forces_dirty = true;  // restore: the next step uploads the pending loads again
            throw;
        }
        S.device_forces = false;
        // the step consumed the loads: the applied total, in node order
        static_assert(sizeof(swb_vec3) == 3 * sizeof(double), "swb_vec3 layout");
        applied_total_kernel<<<1, 1024, 0, S.stream>>>(S.def.nodes.size(), c->d_items + c->bindings, total64,
                                                       c->d_applied);
        cuda_check(cudaGetLastError(), "applied_total_kernel");
        swb_vec3 applied{};
        cuda_check(cudaMemcpyAsync(&applied, c->d_applied, sizeof(applied), cudaMemcpyDeviceToHost, S.stream),
                   "read");
        cuda_check(cudaStreamSynchronize(S.stream), "applied");
        S.last_applied = applied;
        S.forces_dirty = true;  // the buffer holds this call's loads; pending is empty again
        if (out) out->last_applied_external_force = applied;
    });
}

}  // namespace
}  // namespace swb

using namespace swb;

swb_status swb_coupling_create(swb_structure* structure, const uint64_t* structure_nodes, uint64_t bindings,
                               swb_coupling** out) {
    return guarded([&] {
        if (!structure || !out || (bindings && !structure_nodes)) raise(SWB_INVALID_ARGUMENT, "null argument");
        if (structure->borrowed)
            raise(SWB_UNSUPPORTED, "a structure of a batch steps with its batch; couple a plain structure");
        StructureImpl& S = structure->s;
        const uint64_t N = S.def.nodes.size();
        auto c = std::make_unique<swb_coupling>();
        c->structure = structure;
        c->bindings = bindings;
        c->node_of_binding.assign(structure_nodes, structure_nodes + bindings);
        std::vector<uint32_t> counts(N + 1, 0);
        for (uint64_t i = 0; i < bindings; ++i) {
            if (structure_nodes[i] >= N) raise(SWB_OUT_OF_RANGE, "coupling binding names an unknown structure node");
            ++counts[S.slot_of_node[structure_nodes[i]] + 1];
        }
        for (uint64_t s = 0; s < N; ++s) counts[s + 1] += counts[s];
        std::vector<uint32_t> items(bindings + N);  // bindings by slot, then the slot of every node
        std::vector<uint32_t> fill(counts.begin(), counts.end() - 1);
        for (uint64_t i = 0; i < bindings; ++i) items[fill[S.slot_of_node[structure_nodes[i]]]++] = static_cast<uint32_t>(i);
        for (uint64_t n = 0; n < N; ++n) items[bindings + n] = S.slot_of_node[n];
        cuda_check(cudaSetDevice(S.device), "cudaSetDevice");
        c->d_offsets = alloc<uint32_t>(c->owned, N + 1);
        c->d_items = alloc<uint32_t>(c->owned, items.size());
        c->d_pending = alloc<double>(c->owned, 3 * N);
        c->d_applied = alloc<double>(c->owned, 3);
        c->d_flag = alloc<int>(c->owned, 1);
        cuda_check(cudaMemcpy(c->d_offsets, counts.data(), (N + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice),
                   "upload");
        cuda_check(cudaMemcpy(c->d_items, items.data(), items.size() * sizeof(uint32_t), cudaMemcpyHostToDevice),
                   "upload");
        *out = c.release();
    });
}

void swb_coupling_destroy(swb_coupling* coupling) { delete coupling; }

swb_status swb_coupling_advance_impulses(swb_coupling* coupling, const double* impulses, double duration,
                                         const swb_step_settings* settings, swb_diagnostics* out) {
    if (!coupling || !settings || (coupling->bindings && !impulses))
        return guarded([] { raise(SWB_INVALID_ARGUMENT, "null argument"); });
    if (!(duration > 0.0) || !std::isfinite(duration) || settings->time_step != duration)
        return guarded([] {
            raise(SWB_INVALID_ARGUMENT, "time-integrated transfer does not match this structure macro-step");
        });
    return advance(coupling, impulses, nullptr, 1.0 / duration, 0, settings, out);
}

swb_status swb_coupling_advance_endpoint_loads(swb_coupling* coupling, const double* start_loads,
                                               const double* end_loads, const swb_step_settings* settings,
                                               swb_diagnostics* out) {
    if (!coupling || !settings || (coupling->bindings && (!start_loads || !end_loads)))
        return guarded([] { raise(SWB_INVALID_ARGUMENT, "null argument"); });
    return advance(coupling, start_loads, end_loads, 0.0, 1, settings, out);
}
