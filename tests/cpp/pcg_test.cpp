// PCG32 jump-ahead (used by the GPU outlier removal to generate a random
// stream in parallel) equals stepping the generator one output at a time.
#include <cstdio>

#include "geometry.hpp"

int main()
{
    using cctagb::geo::Pcg32;
    int bad = 0;
    for (uint64_t stream : {0ull, 1ull, 12345ull, (3ull << 32) | 77ull}) {
        Pcg32 ref(271828, stream);
        for (uint64_t k = 0; k < 3000; ++k) {
            Pcg32 j(271828, stream);
            j.advance(k);
            if (j.next() != Pcg32::output(ref.state) || j.state != (ref.next(), ref.state)) ++bad;
        }
    }
    std::printf("mismatches %d\n", bad);
    return bad == 0 ? 0 : 1;
}
