// fast_atan2 and fast_rcp (simwing_b200/csrc/fast_math.h) against the C++
// library on the host, over every octant, near the octant boundaries and at
// the special points.  Exits non-zero when the error bound is exceeded.
#include "../../simwing_b200/csrc/fast_math.h"

#include <cmath>
#include <cstdio>
#include <random>

int main() {
    std::mt19937_64 rng(11);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    double worst = 0.0;
    auto check = [&](float y, float x) {
        const double e = std::fabs(static_cast<double>(swb::fast_atan2(y, x)) - std::atan2((double)y, (double)x));
        if (e > worst) worst = e;
    };
    for (int i = 0; i < 2000000; ++i) {
        const float scale = static_cast<float>(std::pow(10.0, 6.0 * u(rng)));
        check(static_cast<float>(u(rng)) * scale, static_cast<float>(u(rng)) * scale);
    }
    for (float t : {1.0f, 1.0000001f, 0.9999999f, 1e-30f, 1e30f})
        for (float sy : {1.0f, -1.0f})
            for (float sx : {1.0f, -1.0f}) {
                check(sy * t, sx * 1.0f);
                check(sy * 1.0f, sx * t);
            }
    const bool zero = swb::fast_atan2(0.0f, 0.0f) == 0.0f && swb::fast_atan2(0.0f, 1.0f) == 0.0f &&
                      std::fabs(swb::fast_atan2(0.0f, -1.0f) - 3.14159265f) < 1e-6f &&
                      std::isnan(swb::fast_atan2(NAN, 1.0f));
    std::printf("fast_atan2 max abs error %.3e rad, special points %s\n", worst, zero ? "ok" : "FAIL");
    const bool ok = worst <= 4.0e-7 && zero && swb::fast_rcp(4.0f) == 0.25f;
    std::printf("%s\n", ok ? "ok" : "FAIL");
    return ok ? 0 : 1;
}
