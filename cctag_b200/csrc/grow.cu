// Ellipse growing on the GPU: flow_component_grow of the host candidate stage
// (Detection.cpp:190-267, EllipseGrowing.cpp:345-551), one block per
// candidate.  Built with --fmad=false: every float operation is the host
// code's (compiled with -ffp-contract=off), in the same order, and the fits
// are the shared FP64 cores summing in point order, so a candidate's outer
// points, their order and its ellipse are the host's bit for bit.
//
// The reference grows the outer point list with a depth-first search from
// every point already in it (connectedPoint, EllipseGrowing.cpp:378-422),
// through 8-neighbours that lie in the hull around the current ellipse, point
// away from its center and are not yet in the list; the order in which it
// meets them is the list's order, which the fits and the later random draws
// depend on.  A pass here keeps that search but moves its data on chip:
//   1. the block gathers every edge point of the hull (the exact is_in_hull
//      test over the bitmap words of the hull's bounding box) into a shared
//      memory hash keyed by pixel position, with per point whether it passes
//      the gradient test and whether it is already listed;
//   2. one thread runs the reference's depth-first search from the listed
//      points, in list order, reading neighbours from that hash only (listed
//      points with no eligible neighbour are found in parallel beforehand and
//      skipped: marks only grow during a pass, so they would find nothing).
#include "grow.hpp"

#include <cfloat>
#include <cstring>
#include <string>

#include "cctag_b200/portable/fit_core.hpp"
#include "geometry.hpp"

namespace cctagb {

namespace {

constexpr int kThreads = 256;
constexpr int kGCap = 2048;                // hull edge points one pass holds
constexpr int kGHash = 2 * kGCap;          // open addressing, load <= 1/2
constexpr int kMaxGrowIters = 256;         // passes of one growing loop (the reference has no cap)
constexpr uint8_t kQual = 1, kListed = 2, kVisited = 4;

struct GrowLevel {
    int W, H, WW, E;
    const int32_t* exy;
    const int32_t* grad;
    const uint2* bitidx;
};
struct GrowLevels {
    GrowLevel l[kMaxLevels];
};

struct GrowArgs {
    GrowLevels lv;
    const GrowTask* tasks;
    const int32_t* pts;
    GrowResult* res;
    int32_t* outer;
    float width;
    float thrMedian;
    int cap;           // outer points a block may hold (<= kGrowMaxOuter)
};

// Shared state of one block.
struct Smem {
    int32_t pid[kGrowMaxOuter];   // the outer list: point index ...
    int32_t xy[kGrowMaxOuter];    // ... and x | y << 16
    int32_t gkey[kGHash];         // hull points: position key, -1 empty
    int16_t gat[kGHash];          // -> hull point
    int32_t gpos[kGCap];
    int32_t gpid[kGCap];
    uint8_t gflag[kGCap];         // kQual | kListed | kVisited
    uint8_t start[kGrowMaxOuter]; // listed point with an eligible neighbour
    int32_t stk[kGrowMaxOuter];   // depth-first stack: position and next neighbour
    uint8_t stk_k[kGrowMaxOuter];
    int16_t found[kGrowMaxOuter]; // hull points a pass adds, in order
    uint32_t keys[kGrowMaxOuter]; // median sort / scratch
    int fitOk;
    unsigned long long best;      // argmin scratch
    int first;                    // first-index scratch
    int nOuter, nG, nFound, err, cnt;
    int lens[kMaxGrowIters + 1];  // growing loop with a circle init: outer size after each pass
    float ells[kMaxGrowIters + 1][5];
    float e[5];                   // current ellipse: cx, cy, a, b, angle
    geo::Mat3 Q;                  // and its conic
    geo::Mat3 qin, qout;          // hull of the current pass
    float qinCx, qinCy;
};

__device__ __forceinline__ float px(int xy) { return float(xy & 0xffff); }
__device__ __forceinline__ float py(int xy) { return float(xy >> 16); }
__device__ __forceinline__ float gdx(const GrowLevel& L, int i) { return float(int16_t(L.grad[i] & 0xffff)); }
__device__ __forceinline__ float gdy(const GrowLevel& L, int i) { return float(int16_t(L.grad[i] >> 16)); }

__device__ __forceinline__ uint32_t hpos(int key) { return (uint32_t(key) * 2654435761u) >> 20 & (kGHash - 1); }

// Hull point at position key, -1 if none.
__device__ __forceinline__ int gfind(const Smem& S, int key)
{
    for (uint32_t h = hpos(key), n = 0; n < kGHash; h = (h + 1) & (kGHash - 1), ++n) {
        const int k = S.gkey[h];
        if (k == key) return S.gat[h];
        if (k < 0) return -1;
    }
    return -1;
}

// Sets the current ellipse from its parameters (Ellipse::from_params); false
// when a semi axis is negative (the reference throws).
__device__ bool set_ellipse(Smem& S, float cx, float cy, float a, float b, float angle)
{
    if (a < 0.f || b < 0.f) return false;
    S.e[0] = cx;
    S.e[1] = cy;
    S.e[2] = a;
    S.e[3] = b;
    S.e[4] = angle;
    S.Q = geo::conic_of_params(cx, cy, a, b, angle);
    return true;
}

// Fits of the outer list in order (fit_points / fit_circle_points): one
// thread runs the shared FP64 core (its sums in point order), all threads
// wait.  Returns whether the fit succeeded (the reference throws otherwise);
// the current ellipse is the fit's.
__device__ bool fit_outer(Smem& S, bool circle)
{
    if (threadIdx.x == 0) {
        auto pt = [&](size_t i, float& x, float& y) {
            const int v = S.xy[i];
            x = px(v);
            y = py(v);
        };
        bool ok;
        if (circle) {
            double xc, yc, r;
            ok = geo::fit_circle_core(pt, size_t(S.nOuter), xc, yc, r) &&
                 set_ellipse(S, float(xc), float(yc), float(r), float(r), 0.f);
        } else {
            float cx, cy, a, b, angle;
            ok = geo::fit_ellipse_core(pt, size_t(S.nOuter), cx, cy, a, b, angle) == geo::kFitOk &&
                 set_ellipse(S, cx, cy, a, b, angle);
        }
        S.fitOk = ok;
    }
    __syncthreads();
    const bool ok = S.fitOk;
    __syncthreads();
    return ok;
}

// compute_hull (EllipseGrowing.cpp:424-441) of the current ellipse.
__device__ void set_hull(Smem& S, float delta)
{
    const float a = S.e[2], b = S.e[3];
    S.qin = geo::conic_of_params(S.e[0], S.e[1], fmaxf(a - delta, 0.001f), fmaxf(b - delta, 0.001f), S.e[4]);
    S.qout = geo::conic_of_params(S.e[0], S.e[1], a + delta, b + delta, S.e[4]);
    S.qinCx = S.e[0];
    S.qinCy = S.e[1];
}

// count_in_hull: outer points strictly between the hull's conics (all threads).
__device__ int count_in_hull(Smem& S, float delta)
{
    if (threadIdx.x == 0) {
        set_hull(S, delta);
        S.cnt = 0;
    }
    __syncthreads();
    int c = 0;
    for (int i = threadIdx.x; i < S.nOuter; i += kThreads) {
        const int v = S.xy[i];
        c += geo::is_in_hull_q(S.qin, S.qout, px(v), py(v)) ? 1 : 0;
    }
    if (c) atomicAdd(&S.cnt, c);
    __syncthreads();
    const int r = S.cnt;
    __syncthreads();
    return r;
}

// ellipse_hull (EllipseGrowing.cpp:443-457): one growing pass around the
// current ellipse.  Returns false when the block ran out of room.
__device__ bool grow_pass(Smem& S, const GrowLevel& L, float delta, int cap)
{
    // neighbour k at (x + xoff[k], y + yoff[k]), xoff = 1 1 0 -1 -1 -1 0 1 and
    // yoff = 0 -1 -1 -1 0 1 1 1 (EllipseGrowing.cpp:386-387), one nibble + 1 each
    constexpr uint32_t kXoff = 0x21000122u, kYoff = 0x22210001u;
    if (threadIdx.x == 0) {
        set_hull(S, delta);
        S.nG = 0;
        S.nFound = 0;
    }
    for (int i = threadIdx.x; i < kGHash; i += kThreads) S.gkey[i] = -1;
    __syncthreads();
    // 1. the hull's edge points: the bitmap words of its bounding box (the
    // outer conic's semi axes plus a margin), each set bit through the exact
    // hull test
    const float R = fmaxf(S.e[2], S.e[3]) + delta + 2.f;
    const int y0 = max(0, int(floorf(S.e[1] - R))), y1 = min(L.H - 1, int(ceilf(S.e[1] + R)));
    const int x0 = max(0, int(floorf(S.e[0] - R))), x1 = min(L.W - 1, int(ceilf(S.e[0] + R)));
    if (y0 <= y1 && x0 <= x1) {
        const int w0 = x0 >> 5, nw = (x1 >> 5) - w0 + 1;
        const int items = (y1 - y0 + 1) * nw;
        for (int it = threadIdx.x; it < items; it += kThreads) {
            const int y = y0 + it / nw, w = w0 + it % nw;
            const uint2 v = L.bitidx[size_t(y) * L.WW + w];
            uint32_t bits = v.x;
            while (bits) {
                const int b = __ffs(bits) - 1;
                bits &= bits - 1;
                const int pid = int(v.y) + __popc(v.x & ((1u << b) - 1u));
                if (pid >= L.E) break;
                const int x = (w << 5) + b;
                if (!geo::is_in_hull_q(S.qin, S.qout, float(x), float(y))) continue;
                const int g = atomicAdd(&S.nG, 1);
                if (g >= kGCap) {
                    S.err = 1;
                    break;
                }
                const int key = x | (y << 16);
                S.gpos[g] = key;
                S.gpid[g] = pid;
                for (uint32_t h = hpos(key);; h = (h + 1) & (kGHash - 1))
                    if (atomicCAS(&S.gkey[h], -1, key) == -1) {
                        S.gat[h] = int16_t(g);
                        break;
                    }
            }
        }
    }
    __syncthreads();
    if (S.err) return false;
    const int nG = S.nG;
    // the gradient test (the gradient points away from the hull's center)
    for (int g = threadIdx.x; g < nG; g += kThreads) {
        const int key = S.gpos[g], q = S.gpid[g];
        const float ox = S.qinCx - px(key), oy = S.qinCy - py(key);
        S.gflag[g] = gdx(L, q) * ox + gdy(L, q) * oy < 0 ? kQual : 0;
    }
    __syncthreads();
    const int nOuter0 = S.nOuter;
    for (int i = threadIdx.x; i < nOuter0; i += kThreads) {
        const int g = gfind(S, S.xy[i]);
        if (g >= 0) S.gflag[g] |= kListed;  // the same value from every thread that lists it
    }
    __syncthreads();
    // listed points with an eligible neighbour
    for (int i = threadIdx.x; i < nOuter0; i += kThreads) {
        const int v = S.xy[i];
        const int x = v & 0xffff, y = v >> 16;
        bool any = false;
        for (int k = 0; k < 8 && !any; ++k) {
            const int sx = x + int((kXoff >> (4 * k)) & 15u) - 1, sy = y + int((kYoff >> (4 * k)) & 15u) - 1;
            if (sx < 0 || sx >= L.W || sy < 0 || sy >= L.H) continue;
            const int g = gfind(S, sx | (sy << 16));
            any = g >= 0 && (S.gflag[g] & (kQual | kListed)) == kQual;
        }
        S.start[i] = any ? 1 : 0;
    }
    __syncthreads();
    // 2. the reference's depth-first search, one thread
    if (threadIdx.x == 0) {
        int nf = 0;
        for (int i = 0; i < nOuter0 && !S.err; ++i) {
            if (!S.start[i]) continue;
            int sp = 0;
            S.stk[0] = S.xy[i];
            S.stk_k[0] = 0;
            while (sp >= 0) {
                const int k = S.stk_k[sp];
                if (k >= 8) {
                    --sp;
                    continue;
                }
                S.stk_k[sp] = uint8_t(k + 1);
                const int v = S.stk[sp];
                const int sx = (v & 0xffff) + int((kXoff >> (4 * k)) & 15u) - 1;
                const int sy = (v >> 16) + int((kYoff >> (4 * k)) & 15u) - 1;
                if (sx < 0 || sx >= L.W || sy < 0 || sy >= L.H) continue;
                const int g = gfind(S, sx | (sy << 16));
                if (g < 0 || S.gflag[g] != kQual) continue;  // no hull edge point, listed, visited or gradient
                if (nOuter0 + nf >= cap) {
                    S.err = 1;
                    break;
                }
                S.gflag[g] = kQual | kVisited;
                S.found[nf++] = int16_t(g);
                ++sp;
                S.stk[sp] = S.gpos[g];
                S.stk_k[sp] = 0;
            }
        }
        S.nFound = nf;
    }
    __syncthreads();
    if (S.err) return false;
    const int nf = S.nFound;
    for (int j = threadIdx.x; j < nf; j += kThreads) {
        const int g = S.found[j];
        S.pid[nOuter0 + j] = S.gpid[g];
        S.xy[nOuter0 + j] = S.gpos[g];
    }
    __syncthreads();
    if (threadIdx.x == 0) S.nOuter = nOuter0 + nf;
    __syncthreads();
    return true;
}

// median_ref of the outer points' distances to the current ellipse (all threads).
__device__ float median_distance(Smem& S)
{
    const int n = S.nOuter;
    int m = 1;
    while (m < n) m <<= 1;
    for (int i = threadIdx.x; i < m; i += kThreads) {
        uint32_t key = 0xffffffffu;
        if (i < n) {
            const int v = S.xy[i];
            key = geo::order_key(geo::dist_point_ellipse(S.Q, px(v), py(v)));
        }
        S.keys[i] = key;
    }
    __syncthreads();
    for (int k = 2; k <= m; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < m; i += kThreads) {
                const int o = i ^ j;
                if (o > i) {
                    const bool up = (i & k) == 0;
                    const uint32_t a = S.keys[i], b = S.keys[o];
                    if ((a > b) == up) {
                        S.keys[i] = b;
                        S.keys[o] = a;
                    }
                }
            }
            __syncthreads();
        }
    const uint32_t key = S.keys[n / 2];
    __syncthreads();
    const uint32_t u = (key & 0x80000000u) ? (key & 0x7fffffffu) : ~key;
    return __uint_as_float(u);
}

// The normalised gradient inner product of points p and q (inner_prod_min's
// expression, the same float operations).
__device__ __forceinline__ float grad_ip(const GrowLevel& L, float gxp, float gyp, int q)
{
    const float ng = sqrtf(gdx(L, q) * gdx(L, q) + gdy(L, q) * gdy(L, q));
    return gxp * (gdx(L, q) / ng) + gyp * (gdy(L, q) / ng);
}

// inner_prod_min (Detection.cpp:87-113 via isGoodEGPoints), all threads: the
// reference's loop returns at the first product <= thr, else tracks the
// minimum (first occurrence), so the products are computed in parallel and
// the first index and the argmin found by reductions.
__device__ float inner_prod_min(Smem& S, const GrowLevel& L, const int32_t* fc, int n, float thr)
{
    if (n == 0) return 1.1f;
    float* ip = reinterpret_cast<float*>(S.keys);
    const int p0 = fc[0];
    float ng = sqrtf(gdx(L, p0) * gdx(L, p0) + gdy(L, p0) * gdy(L, p0));
    const float gx0 = gdx(L, p0) / ng, gy0 = gdy(L, p0) / ng;
    if (threadIdx.x == 0) {
        S.first = n;
        S.best = ~0ull;
    }
    __syncthreads();
    for (int i = 1 + threadIdx.x; i < n; i += kThreads) {
        const float v = grad_ip(L, gx0, gy0, fc[i]);
        ip[i] = v;
        if (v <= thr) atomicMin(&S.first, i);
        if (v < 1.1f) atomicMin(&S.best, (unsigned long long)geo::order_key(v) << 32 | unsigned(i));
    }
    __syncthreads();
    float res;
    if (S.first < n) {
        res = ip[S.first];
    } else if (S.best == ~0ull) {
        res = 1.1f;
    } else {
        const int pA = fc[int(S.best & 0xffffffffu)];
        ng = sqrtf(gdx(L, pA) * gdx(L, pA) + gdy(L, pA) * gdy(L, pA));
        const float gxm = gdx(L, pA) / ng, gym = gdy(L, pA) / ng;
        __syncthreads();
        if (threadIdx.x == 0) {
            S.first = n;
            S.best = ~0ull;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += kThreads) {
            const float v = grad_ip(L, gxm, gym, fc[i]);
            ip[i] = v;
            if (v <= thr) atomicMin(&S.first, i);
            if (v < 1.f) atomicMin(&S.best, (unsigned long long)geo::order_key(v) << 32 | unsigned(i));
        }
        __syncthreads();
        res = S.first < n ? ip[S.first] : S.best == ~0ull ? 1.f : ip[int(S.best & 0xffffffffu)];
    }
    __syncthreads();
    return res;
}

__global__ void __launch_bounds__(kThreads) k_grow(GrowArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem& S = *reinterpret_cast<Smem*>(smem_raw);
    const GrowTask T = a.tasks[blockIdx.x];
    const GrowLevel& L = a.lv.l[T.level];
    const int32_t* fc = a.pts + T.first;
    GrowResult* R = a.res + blockIdx.x;
    int32_t* out = a.outer + size_t(blockIdx.x) * kGrowMaxOuter;
    __shared__ int s_status, s_good;
    if (T.count > a.cap) {  // the host grows it
        if (threadIdx.x == 0) {
            R->status = kGrowHost;
            R->nOuter = 0;
        }
        return;
    }
    // outer = fc (EllipseGrowing.cpp:463-467)
    for (int i = threadIdx.x; i < T.count; i += kThreads) {
        S.pid[i] = fc[i];
        S.xy[i] = L.exy[fc[i]];
    }
    if (threadIdx.x == 0) {
        S.err = 0;
        S.nOuter = T.count;
        s_status = kGrowKeep;
    }
    // ellipseGrowingInit (EllipseGrowing.cpp:359-376)
    const bool good = inner_prod_min(S, L, fc, T.count, 0.25f) <= 0.25f;
    if (threadIdx.x == 0) s_good = good;
    if (!fit_outer(S, !good) && threadIdx.x == 0) s_status = kGrowDrop;
    __syncthreads();
    const float width = a.width;
    auto fail = [&](int st) {
        if (threadIdx.x == 0) s_status = st;
        __syncthreads();
    };
    if (s_status == kGrowKeep && !s_good) {
        // ellipseGrowing2, circle start (EllipseGrowing.cpp:470-506)
        int newSize = S.nOuter, maxNb = newSize, nIterMax = 0, lastSize = 0, nIter = 0;
        if (threadIdx.x == 0) {
            S.lens[0] = S.nOuter;
            for (int k = 0; k < 5; ++k) S.ells[0][k] = S.e[k];
        }
        ++nIter;
        while (newSize - lastSize > 0) {
            if (nIter > kMaxGrowIters) {
                fail(kGrowHost);
                break;
            }
            lastSize = count_in_hull(S, width);
            if (!grow_pass(S, L, width, a.cap)) {
                fail(kGrowHost);
                break;
            }
            if (threadIdx.x == 0) {
                S.lens[nIter] = S.nOuter;
                for (int k = 0; k < 5; ++k) S.ells[nIter][k] = S.e[k];
            }
            __syncthreads();
            if (!fit_outer(S, true) && threadIdx.x == 0) s_status = kGrowDrop;
            __syncthreads();
            if (s_status != kGrowKeep) break;
            newSize = count_in_hull(S, width);
            if (newSize > maxNb) {
                maxNb = newSize;
                nIterMax = nIter;
            }
            ++nIter;
        }
        if (s_status == kGrowKeep && threadIdx.x == 0) {
            // outer = sets[nIterMax] (a prefix of the list), ellipse = ells[nIterMax]
            S.nOuter = S.lens[nIterMax];
            const float* e = S.ells[nIterMax];
            set_ellipse(S, e[0], e[1], e[2], e[3], e[4]);
        }
        __syncthreads();
    }
    if (s_status == kGrowKeep) {
        // EllipseGrowing.cpp:508-550: ellipse fit, then grow while the list grows
        if (!fit_outer(S, false) && threadIdx.x == 0) s_status = kGrowDrop;
        __syncthreads();
        int lastSize = 0, iter = 0;
        while (s_status == kGrowKeep && S.nOuter > lastSize) {
            if (++iter > kMaxGrowIters) {
                fail(kGrowHost);
                break;
            }
            lastSize = S.nOuter;
            __syncthreads();
            if (!grow_pass(S, L, width, a.cap)) {
                fail(kGrowHost);
                break;
            }
            if (!fit_outer(S, false) && threadIdx.x == 0) s_status = kGrowDrop;
            __syncthreads();
        }
    }
    if (s_status == kGrowKeep) {
        // completeFlowComponent's checks (Detection.cpp:227-260)
        const float SmFinal = median_distance(S);
        if (threadIdx.x == 0) {
            if (SmFinal > a.thrMedian) s_status = kGrowDrop;
            const int per = geo::rasterize_perimeter_p(S.e[0], S.e[1], S.e[2], S.e[3], S.e[4]);
            const float quality = float(S.nOuter) / float(per);
            // the reference's literals are doubles
            if (double(quality) > 1.1) s_status = kGrowDrop;
            const float ratio = S.e[2] / S.e[3];
            if (double(ratio) < 0.05 || ratio > 20) s_status = kGrowDrop;
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < S.nOuter && s_status == kGrowKeep; i += kThreads) out[i] = S.pid[i];
    if (threadIdx.x == 0) {
        R->status = s_status;
        R->nOuter = s_status == kGrowKeep ? S.nOuter : 0;
        R->cx = S.e[0];
        R->cy = S.e[1];
        R->a = S.e[2];
        R->b = S.e[3];
        R->angle = S.e[4];
        for (int k = 0; k < 9; ++k) R->Q[k] = S.Q.m[k / 3][k % 3];
    }
}

}  // namespace

GrowGpu::GrowGpu(int spin_us, int max_points) : cap_(max_points)
{
    if (max_points < 16 || max_points > kGrowMaxOuter)
        throw Error{CCTAGB_BAD_ARG, "gpuGrowMaxPoints must be in [16, " + std::to_string(kGrowMaxOuter) + "]"};
    waiter_.init(spin_us);
    CCTAGB_CUDA(cudaFuncSetAttribute(k_grow, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sizeof(Smem))));
}

GrowGpu::~GrowGpu()
{
    for (void* p : {static_cast<void*>(d_tasks_), static_cast<void*>(d_pts_), static_cast<void*>(d_res_),
                    static_cast<void*>(d_outer_)})
        if (p) cudaFree(p);
    for (void* p : {static_cast<void*>(h_tasks_), static_cast<void*>(h_pts_), static_cast<void*>(h_res_),
                    static_cast<void*>(h_outer_)})
        if (p) cudaFreeHost(p);
}

void GrowGpu::ensure(int tasks, int pts)
{
    if (tasks > taskCap_) {
        for (void* p : {static_cast<void*>(d_tasks_), static_cast<void*>(d_res_), static_cast<void*>(d_outer_)})
            if (p) cudaFree(p);
        for (void* p : {static_cast<void*>(h_tasks_), static_cast<void*>(h_res_), static_cast<void*>(h_outer_)})
            if (p) cudaFreeHost(p);
        d_tasks_ = nullptr;
        d_res_ = nullptr;
        d_outer_ = nullptr;
        h_tasks_ = nullptr;
        h_res_ = nullptr;
        h_outer_ = nullptr;
        taskCap_ = 0;
        const int cap = std::max(tasks, 64);
        CCTAGB_CUDA(cudaMalloc(&d_tasks_, sizeof(GrowTask) * cap));
        CCTAGB_CUDA(cudaMalloc(&d_res_, sizeof(GrowResult) * cap));
        CCTAGB_CUDA(cudaMalloc(&d_outer_, sizeof(int32_t) * kGrowMaxOuter * size_t(cap)));
        CCTAGB_CUDA(cudaMallocHost(&h_tasks_, sizeof(GrowTask) * cap));
        CCTAGB_CUDA(cudaMallocHost(&h_res_, sizeof(GrowResult) * cap));
        CCTAGB_CUDA(cudaMallocHost(&h_outer_, sizeof(int32_t) * kGrowMaxOuter * size_t(cap)));
        taskCap_ = cap;
    }
    if (pts > ptsCap_) {
        if (d_pts_) cudaFree(d_pts_);
        if (h_pts_) cudaFreeHost(h_pts_);
        d_pts_ = nullptr;
        h_pts_ = nullptr;
        ptsCap_ = 0;
        const int cap = std::max(pts, 16384);
        CCTAGB_CUDA(cudaMalloc(&d_pts_, sizeof(int32_t) * cap));
        CCTAGB_CUDA(cudaMallocHost(&h_pts_, sizeof(int32_t) * cap));
        ptsCap_ = cap;
    }
}

void GrowGpu::run(const Levels& lv, const int* E, const std::vector<GrowTask>& tasks, const std::vector<int32_t>& pts,
                  float hullWidth, float thrMedian, cudaStream_t s, std::vector<GrowResult>& res,
                  std::vector<int32_t>& outer, int& stride)
{
    h2d_ = d2h_ = 0;
    launches_ = 0;
    const int n = int(tasks.size());
    res.assign(size_t(n), GrowResult{});
    outer.clear();
    stride = 0;
    if (n == 0) return;
    if (lv.n > kMaxLevels) throw Error{CCTAGB_INTERNAL, "grow: more levels than a frame has"};
    ensure(n, int(pts.size()));
    GrowArgs a{};
    for (int l = 0; l < lv.n; ++l) {
        const LevelView& v = lv.l[l];
        a.lv.l[l] = GrowLevel{v.W, v.H, v.WW, E[l], v.exy, v.grad, v.bitidx};
    }
    for (int t = 0; t < n; ++t) {
        const GrowTask& g = tasks[size_t(t)];
        if (g.level < 0 || g.level >= lv.n || g.first < 0 || g.count < 0 || size_t(g.first + g.count) > pts.size())
            throw Error{CCTAGB_INTERNAL, "grow: bad task"};
        for (int i = g.first; i < g.first + g.count; ++i)
            if (pts[size_t(i)] < 0 || pts[size_t(i)] >= E[g.level]) throw Error{CCTAGB_INTERNAL, "grow: bad point"};
    }
    std::memcpy(h_tasks_, tasks.data(), sizeof(GrowTask) * size_t(n));
    if (!pts.empty()) std::memcpy(h_pts_, pts.data(), sizeof(int32_t) * pts.size());
    CCTAGB_CUDA(cudaMemcpyAsync(d_tasks_, h_tasks_, sizeof(GrowTask) * size_t(n), cudaMemcpyHostToDevice, s));
    if (!pts.empty())
        CCTAGB_CUDA(cudaMemcpyAsync(d_pts_, h_pts_, sizeof(int32_t) * pts.size(), cudaMemcpyHostToDevice, s));
    a.tasks = d_tasks_;
    a.pts = d_pts_;
    a.res = d_res_;
    a.outer = d_outer_;
    a.width = hullWidth;
    a.thrMedian = thrMedian;
    a.cap = cap_;
    k_grow<<<n, kThreads, sizeof(Smem), s>>>(a);
    CCTAGB_CUDA(cudaGetLastError());
    CCTAGB_CUDA(cudaMemcpyAsync(h_res_, d_res_, sizeof(GrowResult) * size_t(n), cudaMemcpyDeviceToHost, s));
    waiter_.wait(s);
    // the outer lists: one copy of the used prefix of each task's row
    int maxOuter = 0;
    for (int t = 0; t < n; ++t) maxOuter = std::max(maxOuter, int(h_res_[t].nOuter));
    if (maxOuter > 0) {
        CCTAGB_CUDA(cudaMemcpy2DAsync(h_outer_, sizeof(int32_t) * maxOuter, d_outer_, sizeof(int32_t) * kGrowMaxOuter,
                                      sizeof(int32_t) * maxOuter, size_t(n), cudaMemcpyDeviceToHost, s));
        waiter_.wait(s);
    }
    res.assign(h_res_, h_res_ + n);
    outer.assign(h_outer_, h_outer_ + size_t(maxOuter) * size_t(n));
    stride = maxOuter;
    h2d_ = (long long)(sizeof(GrowTask) * n + sizeof(int32_t) * pts.size());
    d2h_ = (long long)(sizeof(GrowResult) * n + sizeof(int32_t) * size_t(maxOuter) * n);
    launches_ = 1;
}

}  // namespace cctagb
