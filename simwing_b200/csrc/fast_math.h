// Short single-precision replacements for the two slow calls of the
// projection math, host and device.
//
// fast_atan2: atan2 by octant reduction to a = min(|x|,|y|) / max(|x|,|y|)
// in [0, 1] and an odd polynomial atan(a) ~ a + a s P(s), s = a^2, whose
// seven coefficients were fitted for this project by iteratively reweighted
// least squares (Lawson's algorithm towards the minimax fit) against atan on
// [0, 1]; evaluated in FP32 the polynomial's error is below 1.1e-7 rad and
// the result's, with the octant reflections, below 4e-7 rad.  The device form
// divides with the approximate division (about 2 ulp), the host form exactly.
// fast_rcp: 1/x with the approximate reciprocal on the device (about 1 ulp).
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define SWB_FM __host__ __device__ __forceinline__
#else
#define SWB_FM inline
#endif

namespace swb {

SWB_FM float fast_rcp(float x) {
#if defined(__CUDA_ARCH__)
    return __fdividef(1.0f, x);
#else
    return 1.0f / x;
#endif
}

SWB_FM float fast_atan2(float y, float x) {
    if (x != x || y != y) return x + y;  // NaN in, NaN out
    const float ax = fabsf(x), ay = fabsf(y);
    const float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
    if (!(mx > 0.0f)) return x < 0.0f ? copysignf(3.14159265358979324f, y) : copysignf(0.0f, y);
#if defined(__CUDA_ARCH__)
    const float a = __fdividef(mn, mx);
#else
    const float a = mn / mx;
#endif
    const float s = a * a;
    float p = -0.0043553877621889114f;
    p = p * s + 0.023040074855089188f;
    p = p * s - 0.05777350813150406f;
    p = p * s + 0.0979422926902771f;
    p = p * s - 0.13976579904556274f;
    p = p * s + 0.19962704181671143f;
    p = p * s - 0.3333165943622589f;
    float r = a + a * s * p;
    if (ay > ax) r = 1.57079632679489662f - r;
    if (x < 0.0f) r = 3.14159265358979324f - r;
    return copysignf(r, y);
}

}  // namespace swb
