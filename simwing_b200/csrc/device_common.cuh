// Device helpers: vector math, the bounded device-wide barrier and the
// bulk-copy staging primitives used by the persistent XPBD kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace swb {
namespace dev {

// Status bits written by kernels (atomicOr into status[0]); status[1] holds
// a detail code of the first suspension failure (low byte; the failing
// segment + 1 above it, where the failure belongs to a segment).
enum : int {
    kStatusSyncTimeout = 1,
    kStatusNonFinite = 2,
    kStatusSuspension = 4,
    kStatusCopyTimeout = 8,
    kStatusMembrane = 16,
    kStatusContact = 32,   // status[1]: a kContact* detail code
};

// Suspension detail codes, each one (phase, entity) of the reference's
// SuspensionError (suspension.cpp):
enum : int {
    kSuspLineGeometry = 1,   // LineSolve, the segment (:2247-2252)
    kSuspLineInput = 2,      // LineSolve, "line-projection" (:1141-1150)
    kSuspEffectiveMass = 3,  // LineSolve, "effective-mass" (:1110-1120)
    kSuspPayload = 4,        // Certification, "payload" (:2325-2333)
    kSuspResidual = 5,       // Certification, "line-residual" (:2350-2358)
    kSuspOrientation = 6,    // LineSolve, "payload": the pilot's pose is unusable
    kSuspPredict = 7,        // Prediction, "payload-step" (:1080-1100)
    kSuspCertifyLength = 8,  // Certification, the segment (:2339-2341)
    kSuspFinish = 9,         // Certification, "payload": velocity reconstruction or line damping
};

__device__ __forceinline__ float3 f3(float4 v) { return make_float3(v.x, v.y, v.z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float length(float3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ bool finite3(float3 a) {
    return isfinite(a.x) && isfinite(a.y) && isfinite(a.z);
}

// ---- bounded device-wide barrier -------------------------------------------
// Sense-reversing barrier over all CTAs of a cooperative launch.  Thread 0
// of each CTA arrives with a release fence and spins with acquire loads on
// the generation word.  The spin is bounded by `budget` clock64 cycles;
// when it runs out the CTA records kStatusSyncTimeout and every later
// barrier returns immediately, so the kernel always terminates.
struct GridBarrier {
    unsigned int* count;
    unsigned int* generation;
    int* status;
    long long budget;
    unsigned int blocks;
};

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_relaxed_status(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Returns false when the barrier (or an earlier one) timed out.
__device__ __forceinline__ bool grid_sync(const GridBarrier& g) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = (ld_relaxed_status(g.status) & kStatusSyncTimeout) == 0;
        if (ok) {
            const unsigned int gen = ld_acquire(g.generation);
            __threadfence();
            const unsigned int arrived = atomicAdd(g.count, 1u) + 1u;
            if (arrived == g.blocks) {
                atomicExch(g.count, 0u);
                __threadfence();
                atomicAdd(g.generation, 1u);
            } else {
                const long long start = clock64();
                unsigned int polls = 0, pause = 32;
                while (ld_acquire(g.generation) == gen) {
                    if (clock64() - start > g.budget) {
                        atomicOr(g.status, kStatusSyncTimeout);
                        ok = 0;
                        break;
                    }
                    // a long wait (a contact helper cluster waiting for the
                    // structure's sweep) backs off, so that the spinning
                    // CTAs do not load the memory system the others use
                    if (++polls > 64) {
                        __nanosleep(pause);
                        if (pause < 1024) pause *= 2;
                    }
                }
            }
            __threadfence();
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// ---- bulk global->shared staging (cp.async.bulk + mbarrier) ------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// A node record (float4) at a cluster shared-memory address, read or
// written from any CTA of the cluster.
__device__ __forceinline__ float4 ld_node(uint32_t addr) {
    float4 v;
    asm volatile("ld.shared::cluster.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "r"(addr)
                 : "memory");
    return v;
}
__device__ __forceinline__ void st_node(uint32_t addr, float4 v) {
    asm volatile("st.shared::cluster.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(v.x), "f"(v.y), "f"(v.z),
                 "f"(v.w)
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// One bulk copy; dst/src 16-byte aligned, bytes a non-zero multiple of 16.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait for phase `parity` of the barrier; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long budget) {
    const long long start = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - start > budget) return false;
    }
    return true;
}

}  // namespace dev
}  // namespace swb
