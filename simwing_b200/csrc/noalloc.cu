// swb_diagnostics_noalloc: structure diagnostics of caller-owned device
// arrays, computed without allocating any device memory.
//
// Who needs it: callers whose device memory is not theirs to grow.  The
// coupled flow solver of a fluid-structure run reserves the GPU's memory in
// its own pool at start-up and keeps the structural state in that pool; a
// cudaMalloc from a library behind its back either fails (the pool holds
// the memory) or fragments the pool it sized for the whole run.  Fixed-budget
// control loops have the same constraint for a second reason: cudaMalloc and
// cudaFree may synchronize the device and stall the step.  Such a caller has
// no swb_structure (creating one allocates); it has its node and constraint
// arrays in device memory and wants the reductions of Structure::diagnostics
// (src/fsi/structure.cpp:833-959) over them.
//
// How it avoids allocating: the per-block partial sums live in one
// file-scope `static __device__` array of fixed size (kScratchBytes, below),
// resolved once per device with cudaGetSymbolAddress.  The call issues one
// cudaMemsetAsync (the ticket word that must start at zero), one kernel and
// one cudaMemcpyAsync of the 13 result words into a host stack array, all on
// the legacy default stream, then waits for that stream.  It calls no
// cudaMalloc, cudaFree, cudaMallocHost or any allocating library routine.
//
// Every call shares the one scratch array.  Two calls whose work overlaps on
// the GPU would race on it (on the ticket and the partials).  Calls from this
// entry point cannot overlap in one process: each holds a per-device host lock
// from its first launch until its result is back on the host.
#include "common.h"

#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

namespace swb {
namespace {

constexpr int kNoallocThreads = 256;
constexpr int kNoallocItemsPerThread = 4;
constexpr uint32_t kNoallocBlockItems = kNoallocThreads * kNoallocItemsPerThread;  // 1024
constexpr uint32_t kNoallocMaxBlocks = 512;
constexpr int kNoallocFields = 16;  // 13 used, padded to 128 B per block
constexpr int kNoallocUsed = 13;
static_assert(static_cast<uint64_t>(kNoallocMaxBlocks) * kNoallocBlockItems == SWB_NOALLOC_MAX_NODES,
              "header maximum and scratch size disagree");
static_assert(SWB_NOALLOC_MAX_NODES == SWB_NOALLOC_MAX_CONSTRAINTS, "one block covers nodes and constraints");

// Scratch layout (bytes): block partials | result words | ticket.
constexpr size_t kPartialBytes = static_cast<size_t>(kNoallocMaxBlocks) * kNoallocFields * sizeof(double);
constexpr size_t kResultOffset = kPartialBytes;
constexpr size_t kTicketOffset = kResultOffset + kNoallocFields * sizeof(double);
constexpr size_t kScratchBytes = kTicketOffset + 256;  // 65,920 B

static __device__ __align__(256) unsigned char swb_noalloc_scratch[kScratchBytes];

// Fields: 0 dynamic count, 1 mass, 2-4 sum m x, 5-7 sum m v, 8 kinetic
// energy, 9 finite (min), 10 max |distance error|, 11 max cable extension,
// 12 constraints naming a node outside [0, n).
__device__ __forceinline__ double combine(int f, double a, double b) {
    if (f == 9) return fmin(a, b);
    if (f == 10 || f == 11) return fmax(a, b);
    return a + b;
}

__device__ __forceinline__ double field_start(int f) { return f == 9 ? 1.0 : 0.0; }

// Variant of the structure's diagnostics kernel: a fixed number of items
// per block (no grid-stride loop, so the block count, and with it the
// scratch, is bounded by the input size), partials into the static scratch,
// and the last block to finish folds the partials in block order, so the
// result does not depend on the order in which blocks ran.
__global__ void __launch_bounds__(kNoallocThreads)
diagnostics_noalloc_kernel(const float4* __restrict__ pos, const float4* __restrict__ prev,
                           const float4* __restrict__ vel, uint32_t n, const uint32_t* __restrict__ ca,
                           const uint32_t* __restrict__ cb, const float* __restrict__ rest,
                           const uint8_t* __restrict__ kind, uint32_t m, unsigned char* scratch) {
    double acc[kNoallocUsed];
#pragma unroll
    for (int f = 0; f < kNoallocUsed; ++f) acc[f] = field_start(f);
    const uint32_t base = blockIdx.x * kNoallocBlockItems;
#pragma unroll
    for (int k = 0; k < kNoallocItemsPerThread; ++k) {
        const uint32_t i = base + k * kNoallocThreads + threadIdx.x;
        if (i < n) {
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
        if (i < m) {
            const uint32_t a = ca[i], b = cb[i];
            if (a >= n || b >= n) {
                acc[12] += 1.0;  // reported as SWB_OUT_OF_RANGE; the node is not read
            } else {
                const float4 A = pos[a], B = pos[b];
                const double dx = double(B.x) - A.x, dy = double(B.y) - A.y, dz = double(B.z) - A.z;
                const double e = sqrt(dx * dx + dy * dy + dz * dz) - rest[i];
                if (kind[i] == SWB_CONSTRAINT_CABLE) acc[11] = fmax(acc[11], fmax(0.0, e));
                else acc[10] = fmax(acc[10], fabs(e));
            }
        }
    }
    __shared__ double red[kNoallocThreads / 32][kNoallocUsed];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int f = 0; f < kNoallocUsed; ++f) {
        double v = acc[f];
        for (int o = 16; o > 0; o >>= 1) v = combine(f, v, __shfl_down_sync(0xffffffffu, v, o));
        if (lane == 0) red[warp][f] = v;
    }
    __syncthreads();
    double* partials = reinterpret_cast<double*>(scratch);
    if (threadIdx.x < kNoallocUsed) {
        const int f = threadIdx.x;
        double v = red[0][f];
        for (int w = 1; w < kNoallocThreads / 32; ++w) v = combine(f, v, red[w][f]);
        partials[blockIdx.x * kNoallocFields + f] = v;
    }
    // publish this block's partials, then take a ticket; the last block folds
    __threadfence();
    __syncthreads();
    __shared__ bool last;
    if (threadIdx.x == 0) {
        unsigned long long* ticket = reinterpret_cast<unsigned long long*>(scratch + kTicketOffset);
        last = atomicAdd(ticket, 1ull) == static_cast<unsigned long long>(gridDim.x) - 1ull;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x < kNoallocUsed) {
        const int f = threadIdx.x;
        double v = field_start(f);
        for (uint32_t b = 0; b < gridDim.x; ++b) v = combine(f, v, __ldcg(partials + b * kNoallocFields + f));
        reinterpret_cast<double*>(scratch + kResultOffset)[f] = v;
    }
}

// Scratch address per device, resolved once (with that device current).
constexpr int kMaxDevices = 64;
std::mutex g_setup_lock;
unsigned char* g_scratch[kMaxDevices] = {};
std::mutex g_call_lock[kMaxDevices];

unsigned char* scratch_for(int device) {
    std::lock_guard<std::mutex> guard(g_setup_lock);
    if (!g_scratch[device]) {
        void* ptr = nullptr;
        const cudaError_t rc = cudaGetSymbolAddress(&ptr, swb_noalloc_scratch);
        if (rc != cudaSuccess || ptr == nullptr)
            raise(SWB_CUDA_ERROR, std::string("cudaGetSymbolAddress(swb_noalloc_scratch) failed: ") +
                                      cudaGetErrorString(rc));
        g_scratch[device] = static_cast<unsigned char*>(ptr);
    }
    return g_scratch[device];
}

// The array [p, p + bytes) must be device memory of `device`, inside one
// allocation, so that the kernel's reads stay in bounds.
using GetAddressRange = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);

void check_device_array(const void* p, uint64_t bytes, const char* name, int device, GetAddressRange range) {
    if (bytes == 0) return;
    if (!p) raise(SWB_INVALID_ARGUMENT, std::string(name) + " is null");
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess || attr.device != device ||
        (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged)) {
        cudaGetLastError();
        raise(SWB_INVALID_ARGUMENT, std::string(name) + " is not device memory of device " + std::to_string(device));
    }
    if (range) {
        CUdeviceptr base = 0;
        size_t size = 0;
        if (range(&base, &size, reinterpret_cast<CUdeviceptr>(p)) != CUDA_SUCCESS)
            raise(SWB_INVALID_ARGUMENT, std::string(name) + ": address range unknown");
        const uint64_t offset = reinterpret_cast<CUdeviceptr>(p) - base;
        if (offset + bytes > size)
            raise(SWB_INVALID_ARGUMENT, std::string(name) + " extends past the end of its allocation");
    }
}

GetAddressRange address_range_query() {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return reinterpret_cast<GetAddressRange>(fn);
}

void check(cudaError_t rc, const char* what) {
    if (rc != cudaSuccess) raise(SWB_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(rc));
}

// Restores the caller's current device on every exit path.
struct CurrentDevice {
    int saved = -1;
    explicit CurrentDevice(int device) {
        check(cudaGetDevice(&saved), "cudaGetDevice");
        check(cudaSetDevice(device), "cudaSetDevice");
    }
    ~CurrentDevice() {
        if (saved >= 0) cudaSetDevice(saved);
    }
};

}  // namespace
}  // namespace swb

using namespace swb;

extern "C" swb_status swb_diagnostics_noalloc(int32_t device, const void* positions, const void* previous_positions,
                                              const void* velocities, uint64_t node_count,
                                              const uint32_t* first_nodes, const uint32_t* second_nodes,
                                              const float* rest_lengths, const uint8_t* kinds,
                                              uint64_t constraint_count, swb_diagnostics* out) {
    return guarded([&] {
        if (!out) raise(SWB_INVALID_ARGUMENT, "null diagnostics output");
        if (node_count > SWB_NOALLOC_MAX_NODES)
            raise(SWB_INVALID_ARGUMENT, "node_count " + std::to_string(node_count) +
                                            " exceeds the no-alloc maximum of " +
                                            std::to_string(SWB_NOALLOC_MAX_NODES) + " nodes");
        if (constraint_count > SWB_NOALLOC_MAX_CONSTRAINTS)
            raise(SWB_INVALID_ARGUMENT, "constraint_count " + std::to_string(constraint_count) +
                                            " exceeds the no-alloc maximum of " +
                                            std::to_string(SWB_NOALLOC_MAX_CONSTRAINTS) + " constraints");
        int devices = 0;
        check(cudaGetDeviceCount(&devices), "cudaGetDeviceCount");
        if (device < 0 || device >= devices || device >= kMaxDevices)
            raise(SWB_INVALID_ARGUMENT, "device ordinal " + std::to_string(device) + " out of range");
        const CurrentDevice current(device);
        const GetAddressRange range = address_range_query();
        check_device_array(positions, node_count * 16, "positions", device, range);
        check_device_array(previous_positions, node_count * 16, "previous_positions", device, range);
        check_device_array(velocities, node_count * 16, "velocities", device, range);
        check_device_array(first_nodes, constraint_count * 4, "first_nodes", device, range);
        check_device_array(second_nodes, constraint_count * 4, "second_nodes", device, range);
        check_device_array(rest_lengths, constraint_count * 4, "rest_lengths", device, range);
        check_device_array(kinds, constraint_count, "kinds", device, range);
        unsigned char* scratch = scratch_for(device);

        double r[kNoallocUsed];
        for (int f = 0; f < kNoallocUsed; ++f) r[f] = f == 9 ? 1.0 : 0.0;
        const uint64_t items = node_count > constraint_count ? node_count : constraint_count;
        if (items > 0) {
            const uint32_t blocks = static_cast<uint32_t>((items + kNoallocBlockItems - 1) / kNoallocBlockItems);
            std::lock_guard<std::mutex> guard(g_call_lock[device]);
            check(cudaMemsetAsync(scratch + kTicketOffset, 0, sizeof(unsigned long long), 0), "clear ticket");
            diagnostics_noalloc_kernel<<<blocks, kNoallocThreads, 0, 0>>>(
                static_cast<const float4*>(positions), static_cast<const float4*>(previous_positions),
                static_cast<const float4*>(velocities), static_cast<uint32_t>(node_count), first_nodes,
                second_nodes, rest_lengths, kinds, static_cast<uint32_t>(constraint_count), scratch);
            check(cudaGetLastError(), "diagnostics_noalloc_kernel launch");
            check(cudaMemcpyAsync(r, scratch + kResultOffset, sizeof(r), cudaMemcpyDeviceToHost, 0), "read result");
            check(cudaStreamSynchronize(0), "diagnostics_noalloc_kernel");
        }
        if (r[12] > 0.0)
            raise(SWB_OUT_OF_RANGE, std::to_string(static_cast<uint64_t>(r[12])) +
                                        " constraints name a node outside [0, node_count)");
        std::memset(out, 0, sizeof(*out));
        out->node_count = node_count;
        out->dynamic_node_count = static_cast<uint64_t>(r[0]);
        out->constraint_count = constraint_count;
        out->total_dynamic_mass = r[1];
        if (r[1] > 0.0) out->center_of_mass = {r[2] / r[1], r[3] / r[1], r[4] / r[1]};
        out->linear_momentum = {r[5], r[6], r[7]};
        out->kinetic_energy = r[8];
        out->maximum_distance_error = r[10];
        out->maximum_cable_extension = r[11];
        out->finite = r[9] > 0.5 ? 1u : 0u;
    });
}
