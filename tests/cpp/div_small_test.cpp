// div_small (pmath.hpp) against IEEE float division: every significand of
// the binade [1, 2) for every divisor d in [1, 256].  Division by d commutes
// with scaling x by a power of two while x, q and the remainder stay normal,
// so this covers every such x (and, by symmetry of round-to-nearest, -x).
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "cctag_b200/portable/pmath.hpp"

int main()
{
    long long bad = 0;
    for (int d = 1; d <= 256; ++d) {
        volatile float dv = float(d);
        const float y = 1.0f / dv;
        for (uint32_t m = 0; m < (1u << 23); ++m) {
            const uint32_t bits = 0x3F800000u | m;
            float x;
            std::memcpy(&x, &bits, 4);
            volatile float ref = x / dv;
            const float got = cctagb::pm::div_small(x, float(d), y);
            if (got != ref) {
                if (++bad < 10) std::printf("d=%d x=%.9g got %.9g want %.9g\n", d, x, got, (float)ref);
            }
        }
    }
    std::printf("%lld mismatches\n", bad);
    return bad != 0;
}
