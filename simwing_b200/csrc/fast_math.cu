// swb_fast_math_eval: the device forms of fast_atan2 and fast_rcp
// (fast_math.h) over host arrays, so that they can be checked on the GPU
// they run on.
#include "common.h"
#include "fast_math.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <string>

namespace swb {
namespace {

__global__ void fast_math_kernel(uint32_t which, const float* a, const float* b, float* out, uint64_t n) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        out[i] = which == SWB_FAST_ATAN2 ? fast_atan2(a[i], b[i]) : fast_rcp(a[i]);
}

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) raise(SWB_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace
}  // namespace swb

extern "C" swb_status swb_fast_math_eval(uint32_t which, const float* a, const float* b, float* out,
                                         uint64_t count) {
    using namespace swb;
    return guarded([&] {
        if (which > SWB_FAST_RCP) raise(SWB_INVALID_ARGUMENT, "unknown function");
        if (count && (!a || !out || (which == SWB_FAST_ATAN2 && !b))) raise(SWB_INVALID_ARGUMENT, "null argument");
        if (!count) return;
        float* d = nullptr;
        const size_t bytes = count * sizeof(float);
        check(cudaMalloc(&d, 3 * bytes), "cudaMalloc");
        struct Free {
            float* p;
            ~Free() { cudaFree(p); }
        } guard{d};
        check(cudaMemcpy(d, a, bytes, cudaMemcpyHostToDevice), "copy");
        if (which == SWB_FAST_ATAN2) check(cudaMemcpy(d + count, b, bytes, cudaMemcpyHostToDevice), "copy");
        const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((count + 255) / 256, 148u * 8u));
        fast_math_kernel<<<blocks, 256>>>(which, d, d + count, d + 2 * count, count);
        check(cudaGetLastError(), "launch");
        check(cudaMemcpy(out, d + 2 * count, bytes, cudaMemcpyDeviceToHost), "copy");
    });
}
