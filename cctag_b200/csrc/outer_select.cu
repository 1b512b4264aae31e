// The outer points of each marker sorted by angle around its ellipse center
// and uniformly subsampled (getSortedOuterPoints, geometry/Ellipse.cpp:259-300),
// on the GPU before the cut selection: one block per marker.  Built with
// --fmad=false: the angle is pmath's correctly rounded float atan2 (double
// arithmetic, no contraction), the same bits as the host's; the sort key
// (angle, index) is a total order, so a bitonic sort gives the reference's
// std::sort order; the subsampling repeats the reference's float step.
#include <cstdint>
#include <string>

#include "common.hpp"
#include "ident_host.hpp"

namespace cctagb {

namespace {

constexpr int kThreads = kMaxOuterPoints;

__global__ void __launch_bounds__(kThreads) k_outer_select(const CutSelectIn* __restrict__ ins,
                                                           const DirPoint* __restrict__ pts, int nOuterReq,
                                                           int16_t* __restrict__ sel, int* __restrict__ nsel)
{
    __shared__ unsigned long long s_key[kCutSortCap];
    const CutSelectIn in = ins[blockIdx.x];
    int16_t* out = sel + size_t(blockIdx.x) * kMaxOuterPoints;
    const int t = threadIdx.x;
    if (in.presorted) {  // the host sorted and subsampled them
        for (int k = t; k < in.count; k += kThreads) out[k] = int16_t(k);
        if (t == 0) nsel[blockIdx.x] = in.count;
        return;
    }
    const int n = in.count;  // <= kCutSortCap (the host presorts larger sets)
    int m = 1;
    while (m < n) m <<= 1;
    for (int j = t; j < m; j += kThreads) {
        unsigned long long key = ~0ull;
        if (j < n) {
            const DirPoint p = pts[in.first + j];
            const float a = pm::atan2f_(p.y - in.cy, p.x - in.cx);
            key = (unsigned long long)geo::order_key(a) << 32 | unsigned(j);
        }
        s_key[j] = key;
    }
    __syncthreads();
    for (int k = 2; k <= m; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = t; i < m; i += kThreads) {
                const int o = i ^ j;
                if (o > i) {
                    const bool up = (i & k) == 0;
                    const unsigned long long a = s_key[i], b = s_key[o];
                    if ((a > b) == up) {
                        s_key[i] = b;
                        s_key[o] = a;
                    }
                }
            }
            __syncthreads();
        }
    // pick k is the sorted point int(k * step) while that is < n; nothing
    // with fewer than two points (the reference's step divides by zero)
    const int nOuter = min(nOuterReq, n);
    int count = 0;
    if (nOuter >= 2) {
        const float step = fmaxf(1.f, __fdiv_rn(float(n), float(nOuter - 1)));
        const int i = int(__fmul_rn(float(t), step));
        const bool pick = i < n;
        if (pick) out[t] = int16_t(s_key[i] & 0xffffffffu);
        // k * step reaches n before k = nOuter <= kThreads, and i grows with k
        count = __syncthreads_count(pick);
    }
    if (t == 0) nsel[blockIdx.x] = count;
}

}  // namespace

void launch_outer_select(const CutSelectIn* d_ins, const DirPoint* d_pts, int nOuterReq, int16_t* d_sel, int* d_nsel,
                         int n, cudaStream_t s)
{
    if (n <= 0) return;
    if (nOuterReq < 0 || nOuterReq > kMaxOuterPoints)
        throw Error{CCTAGB_BAD_ARG, "nSamplesOuterEllipse above " + std::to_string(kMaxOuterPoints)};
    k_outer_select<<<n, kThreads, 0, s>>>(d_ins, d_pts, nOuterReq, d_sel, d_nsel);
    CCTAGB_CUDA(cudaGetLastError());
}

}  // namespace cctagb
