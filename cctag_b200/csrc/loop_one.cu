// Loop 1 and the outlier removal of loop 2 of the candidate stage on the GPU
// (see loop_one.hpp).  Built with --fmad=false: every floating-point
// expression here and in cand_shared.hpp is then evaluated with the same IEEE
// operations as the host restatement, so the candidates are the same bits.
//
// k_point_records one thread per edge point: position, gradient angle,
//                 votes received and the 8 neighbouring edge points, so that
//                 a linking step is one dependent load;
// k_seed_slots    marks each seed's record with its processing slot;
// k_link_seeds    one thread per seed: the two edge-linking walks
//                 (Vote.cpp:255-394), independent of the other seeds since
//                 each walk only avoids its own points; also lists the later
//                 seeds its segment marks processed;
// k_link_resolve  one block per level: the seeds in processing order,
//                 skipping those an earlier segment marked (Detection.cpp:
//                 609-627), in shared memory; then the candidates ranked by
//                 averageReceivedVote;
// k_filter        one block per loop-two candidate: children (Vote.cpp:
//                 396-412) and the LMedS outlier removal (Vote.cpp:414-576),
//                 128 random draws evaluated at once and accepted in draw
//                 order; the draws' random stream is generated in parallel
//                 with the PCG jump-ahead;
// k_pack          the kept candidates' filtered children, packed for download.
#include "loop_one.hpp"

#include <algorithm>
#include <cstring>

#include "cand_shared.hpp"

namespace cctagb {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kVisitSlots = 512;  // > 2 * kSegSlot
constexpr int kResolveThreads = 256;
constexpr int kResolveSmemMarks = 12288;

// Record of edge point i: r0 = {x | y << 16, angle bits, votes received, seed
// slot or -1}, r1 / r2 = the edge points at the 8 neighbours in the order of
// Vote.cpp:283-286 for direction +1 (-1 where none).
struct PointRec {
    int4 r0, r1, r2;
};

__device__ __forceinline__ PointRec load_rec(const int4* rec, int i)
{
    PointRec r;
    r.r0 = rec[3 * i];
    r.r1 = rec[3 * i + 1];
    r.r2 = rec[3 * i + 2];
    return r;
}
__device__ __forceinline__ int nbr(const PointRec& r, int k)
{
    switch (k) {
    case 0: return r.r1.x;
    case 1: return r.r1.y;
    case 2: return r.r1.z;
    case 3: return r.r1.w;
    case 4: return r.r2.x;
    case 5: return r.r2.y;
    case 6: return r.r2.z;
    default: return r.r2.w;
    }
}

__device__ __forceinline__ int px_(const LoopOneLevel& L, int i) { return L.exy[i] & 0xffff; }
__device__ __forceinline__ int py_(const LoopOneLevel& L, int i) { return L.exy[i] >> 16; }
__device__ __forceinline__ float gdx(const LoopOneLevel& L, int i) { return float(int16_t(L.grad[i] & 0xffff)); }
__device__ __forceinline__ float gdy(const LoopOneLevel& L, int i) { return float(int16_t(L.grad[i] >> 16)); }
__device__ __forceinline__ int voters(const LoopOneLevel& L, int i) { return L.voff[i + 1] - L.voff[i]; }
__device__ __forceinline__ float gnorm(const LoopOneLevel& L, int i)
{
    const float dx = gdx(L, i), dy = gdy(L, i);
    return sqrtf(dx * dx + dy * dy);
}
// Edge point at pixel (x, y), -1 if none: the word's first index plus its
// set bits below x.
__device__ __forceinline__ int at(const LoopOneLevel& L, int x, int y)
{
    if (x < 0 || x >= L.W || y < 0 || y >= L.H) return -1;
    const uint2 v = L.bitidx[size_t(y) * L.WW + (x >> 5)];
    const uint32_t bit = 1u << (x & 31);
    const int i = int(v.y) + __popc(v.x & (bit - 1u));
    return (v.x & bit) && i < L.E ? i : -1;
}

__global__ void __launch_bounds__(256) k_point_records(LoopOneArgs a, int4 total)
{
    // total.x..w: cumulative point counts of levels 0..3
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int cum[4] = {total.x, total.y, total.z, total.w};
    int l = 0;
    while (l < a.nl - 1 && t >= cum[l]) ++l;
    if (t >= cum[a.nl - 1]) return;
    const int i = t - (l ? cum[l - 1] : 0);
    const LoopOneLevel& L = a.lv[l];
    const int x = px_(L, i), y = py_(L, i);
    const int xoff[8] = {1, 1, 0, -1, -1, -1, 0, 1};
    const int yoff[8] = {0, -1, -1, -1, 0, 1, 1, 1};
    int n[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) n[k] = at(L, x + xoff[k], y + yoff[k]);
    const float angle = cand::link_angle(gdx(L, i), gdy(L, i));
    int4* rec = L.rec + 3 * size_t(i);
    rec[0] = make_int4(L.exy[i], __float_as_int(angle), voters(L, i), -1);
    rec[1] = make_int4(n[0], n[1], n[2], n[3]);
    rec[2] = make_int4(n[4], n[5], n[6], n[7]);
}

__global__ void __launch_bounds__(256) k_seed_slots(LoopOneArgs a)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int l = t / a.maxSlotsPerLevel, s = t % a.maxSlotsPerLevel;
    if (l >= a.nl) return;
    const LoopOneLevel& L = a.lv[l];
    if (s >= L.nProc) return;
    L.rec[3 * size_t(L.order[s])].w = s;
}

// Points of one edge-linking call (the reference's set of visited positions),
// an open-addressing set in shared memory used by the 8 lanes of one seed.
constexpr int kLinkThreads = 128;
constexpr int kLinkGroups = kLinkThreads / 32;  // one seed per warp (lanes 0-7): seeds do not diverge each other

__device__ __forceinline__ uint32_t visit_slot(int v) { return (uint32_t(v) * 2654435761u) >> 23; }
__device__ __forceinline__ bool visit_has(const int32_t* set, int v)
{
    for (uint32_t h = visit_slot(v);; h = (h + 1) & (kVisitSlots - 1)) {
        const int k = set[h];
        if (k == v) return true;
        if (k == -1) return false;
    }
}
__device__ __forceinline__ void visit_add(int32_t* set, int v)
{
    for (uint32_t h = visit_slot(v);; h = (h + 1) & (kVisitSlots - 1)) {
        if (set[h] == v) return;
        if (set[h] == -1) {
            set[h] = v;
            return;
        }
    }
}

__device__ __forceinline__ int4 shfl_int4(unsigned mask, int4 v, int src)
{
    return make_int4(__shfl_sync(mask, v.x, src), __shfl_sync(mask, v.y, src), __shfl_sync(mask, v.z, src),
                     __shfl_sync(mask, v.w, src));
}

// cand::link_convexity_lost, decided from the fast sine and cosine where they
// are more than 1e-3 away from every threshold of the test (their error is
// below 1e-5 for |d| < 2 pi) and from the exact test elsewhere.
__device__ __forceinline__ bool convexity_lost(float front, float back, bool full, int dir)
{
    const float d = back - front;
    const float s = float(dir) * __sinf(d), c = __cosf(d);
    if (full) {
        if (fabsf(s) > 1e-3f) return s < 0.0f;
    } else if (fabsf(s) > 1e-3f && fabsf(s + 0.707f) > 1e-3f && fabsf(c) > 1e-3f) {
        return (s < -0.707f && c > 0.f) || (s < 0.f && c < 0.f);
    }
    return cand::link_convexity_lost(front, back, full, dir);
}

// cand::link_shift without a division where it is safe: the quotient by
// 2 pi through a float reciprocal is within 1e-6 of the exact one after the
// scaling by 8, so wherever that product is more than 1e-5 away from a
// rounding boundary (k + 1/2) both round to the same integer; elsewhere (and
// for a non-finite angle) the exact form decides.
__device__ __forceinline__ int link_shift_fast(float angle)
{
    const float a = __fadd_rn(angle, cand::kPiF / 4.0f);
    const float p = __fmul_rn(__fmul_rn(a, 0.159154943f), 8.0f);
    if (fabsf(__fsub_rn(__fsub_rn(p, floorf(p)), 0.5f)) > 1e-5f) return int(rintf(p)) - 1;
    return cand::link_shift(angle);
}

// cand::link_average_vote with the division by the segment size + 1 (an
// integer up to 2 kLinkMaxLength + 2) correctly rounded by div_small.
__device__ __forceinline__ float link_average_vote_fast(float average, int segSize, int voters)
{
    const float n = __fadd_rn(__fmul_rn(average, float(segSize)), float(voters));
    const float d = float(segSize) + 1.f;
    if (segSize + 1 > 256) return n / d;
    return pm::div_small(n, d, __frcp_rn(d));
}

// Vote.cpp:272-394 edgeLinkingDir from the seed in direction dir, by the 8
// lanes of a group: lane j examines the j-th neighbour of the search order,
// the first lane whose neighbour is an unvisited edge point decides the step.
// The segment is held around segc[0] = seed: the +1 walk appends at
// segc[1..], the -1 walk prepends at segc[-1..].  Returns how many points,
// counted from the front of the segment as it is when the walk ends, become
// processed.
__device__ int link_walk(const int4* recs, int seed, int dir, int32_t* segc, int& nf, int& nb, int32_t* vis,
                         float* ring, int window, float averageVoteMin, unsigned gmask, int j)
{
    int head = 0, count = 0;
    int i = 0;
    bool found = true;
    int stop = 0;
    PointRec r = load_rec(recs, seed);
    float averageVote = float(r.r0.z);
    const int gbase = __ffs(gmask) - 1;
    while (i < cand::kLinkMaxLength && found && averageVote >= averageVoteMin) {
        const float angle = __int_as_float(r.r0.y);
        // window of the last `window` angles (a ring of window + 1 entries)
        if (j == 0) ring[head + count > window ? head + count - window - 1 : head + count] = angle;
        if (++count > window) {
            head = head == window ? 0 : head + 1;
            --count;
        }
        __syncwarp(gmask);
        const int shifting = link_shift_fast(angle);
        const int k = dir == 1 ? (8 - shifting + j) % 8 : (shifting + j) % 8;
        // direction -1 mirrors the y offsets: neighbour (8 - k) % 8 of the +1 table
        const int q = nbr(r, dir == 1 ? k : (8 - k) % 8);
        // every lane fetches its neighbour's record now; the step keeps one
        PointRec rq = r;
        if (q >= 0) rq = load_rec(recs, q);
        const bool cand = q >= 0 && !visit_has(vis, q);
        const unsigned hits = (__ballot_sync(gmask, cand) >> gbase) & 0xffu;
        if (!hits) {
            stop = cand::kEdgeNotFound;
        } else {
            const int jj = __ffs(hits) - 1;
            const int qn = __shfl_sync(gmask, q, gbase + jj);
            const float front = ring[head];
            const float back = ring[head + count - 1 > window ? head + count - window - 2 : head + count - 1];
            if (convexity_lost(front, back, count == window, dir)) {
                stop = cand::kConvexityLost;
            } else {
                if (dir > 0) {
                    ++nb;
                    if (j == 0) segc[nb] = qn;
                } else {
                    ++nf;
                    if (j == 0) segc[-nf] = qn;
                }
                if (j == 0) visit_add(vis, qn);
                r.r0 = shfl_int4(gmask, rq.r0, gbase + jj);
                r.r1 = shfl_int4(gmask, rq.r1, gbase + jj);
                r.r2 = shfl_int4(gmask, rq.r2, gbase + jj);
                averageVote = link_average_vote_fast(averageVote, 1 + nf + nb, r.r0.z);
                stop = 1;
            }
        }
        __syncwarp(gmask);
        found = stop == 1;
        ++i;
    }
    const int size = 1 + nf + nb;
    if (i == cand::kLinkMaxLength || stop == cand::kConvexityLost) return size > window ? size - window : 0;
    if (stop == cand::kEdgeNotFound) return size;
    return 0;
}

__global__ void __launch_bounds__(kLinkThreads) k_link_seeds(LoopOneArgs a)
{
    __shared__ int32_t visAll[kLinkGroups][kVisitSlots];
    __shared__ float ringAll[kLinkGroups][cand::kLinkMaxWindow + 1];
    const int g = threadIdx.x >> 5, j = threadIdx.x & 31;
    if (j >= 8) return;
    const unsigned gmask = 0xffu;
    const int t = blockIdx.x * kLinkGroups + g;
    if (t >= a.totalSlots) return;
    const int l = t / a.maxSlotsPerLevel, s = t % a.maxSlotsPerLevel;
    if (l >= a.nl) return;
    const LoopOneLevel& L = a.lv[l];
    if (s >= L.nProc) return;
    const int seed = L.order[s];
    int32_t* segc = a.seg + size_t(t) * kSegSlot + kSegHalf;
    int32_t* vis = visAll[g];
    float* ring = ringAll[g];
    for (int k = j; k < kVisitSlots; k += 8) vis[k] = -1;
    __syncwarp(gmask);
    if (j == 0) {
        visit_add(vis, seed);
        segc[0] = seed;
    }
    __syncwarp(gmask);
    int nf = 0, nb = 0;
    const int m1 = link_walk(L.rec, seed, 1, segc, nf, nb, vis, ring, a.window, a.averageVoteMin, gmask, j);
    const int m2 = link_walk(L.rec, seed, -1, segc, nf, nb, vis, ring, a.window, a.averageVoteMin, gmask, j);
    __syncwarp(gmask);
    if (j != 0) return;
    int nReceived = 0, nVoted = 0;
    for (int k = -nf; k <= nb; ++k) {
        const int v = L.rec[3 * size_t(segc[k])].z;
        nReceived += v;
        if (v > 0) ++nVoted;
    }
    // later seeds the marks reach: points [0, m1) of (seed, back...) after the
    // +1 walk, points [0, m2) of the whole segment after the -1 walk
    int32_t* ml = a.mlist + size_t(t) * kMarkCap;
    int nm = 0;
    for (int k = 0; k < m1; ++k) {
        const int sl = L.rec[3 * size_t(segc[k])].w;
        if (sl > s) ml[nm++] = sl;
    }
    for (int k = 0; k < m2; ++k) {
        const int sl = L.rec[3 * size_t(segc[-nf + k])].w;
        if (sl > s) ml[nm++] = sl;
    }
    int32_t* info = a.sinfo + size_t(t) * 4;
    info[0] = nf;
    info[1] = nb;
    info[2] = nm;
    info[3] = 0;
    a.skey[t] = cand::received_vote_key(nReceived, nVoted);
}

__global__ void __launch_bounds__(kResolveThreads) k_link_resolve(LoopOneArgs a)
{
    const int l = blockIdx.x;
    const LoopOneLevel& L = a.lv[l];
    const int tid = threadIdx.x;
    extern __shared__ int smem[];
    // [flags: maxSlots][marks offsets: maxSlots + 1][marks: kResolveSmemMarks][keys: maxSlots]
    int* flags = smem;
    int* moff = flags + a.maxSlotsPerLevel;
    int* marks = moff + a.maxSlotsPerLevel + 1;
    float* keys = reinterpret_cast<float*>(marks + kResolveSmemMarks);
    __shared__ int sM, sInSmem;
    const int n = L.nProc;
    for (int s = tid; s < n; s += blockDim.x) flags[s] = 0;
    for (int s = tid; s < n; s += blockDim.x) moff[s + 1] = a.sinfo[size_t(L.slot0 + s) * 4 + 2];
    __syncthreads();
    if (tid == 0) {
        moff[0] = 0;
        for (int s = 0; s < n; ++s) moff[s + 1] += moff[s];
        sInSmem = moff[n] <= kResolveSmemMarks;
    }
    __syncthreads();
    if (sInSmem)
        for (int s = tid; s < n; s += blockDim.x) {
            const int32_t* ml = a.mlist + size_t(L.slot0 + s) * kMarkCap;
            for (int k = 0; k < moff[s + 1] - moff[s]; ++k) marks[moff[s] + k] = ml[k];
        }
    __syncthreads();
    int32_t* made = a.made + size_t(l) * a.maxSlotsPerLevel;
    if (tid == 0) {
        int m = 0;
        for (int s = 0; s < n; ++s) {
            if (flags[s]) continue;
            made[m++] = s;
            const int cnt = moff[s + 1] - moff[s];
            const int32_t* ml = sInSmem ? marks + moff[s] : a.mlist + size_t(L.slot0 + s) * kMarkCap;
            for (int k = 0; k < cnt; ++k) flags[ml[k]] = 1;
        }
        sM = m;
        a.meta[size_t(a.nl) * a.n2max * 4 + l] = m;
    }
    __syncthreads();
    const int m = sM;
    for (int i = tid; i < m; i += blockDim.x) keys[i] = a.skey[L.slot0 + made[i]];
    __syncthreads();
    // Loop-1 order: averageReceivedVote descending, the newer candidate first
    // on equal keys (Detection.cpp:619-622).
    const int n2 = min(m, a.n2max);
    int32_t* meta = a.meta + size_t(l) * a.n2max * 4;
    for (int i = tid; i < m; i += blockDim.x) {
        const float ki = keys[i];
        int rank = 0;
        for (int j = 0; j < m; ++j) {
            const float kj = keys[j];
            rank += (kj > ki || (!(ki > kj) && j > i)) ? 1 : 0;
        }
        if (rank < n2) meta[rank * 4] = made[i];
    }
}

// Ascending bitonic sort of 64 keys held by a warp, key `lane` in a and key
// `lane + 32` in b.
__device__ __forceinline__ void bitonic64(uint32_t& a, uint32_t& b, int lane)
{
#pragma unroll
    for (int k = 2; k <= 64; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j == 32) {  // partners lane and lane + 32, both ascending at k = 64
                const uint32_t lo = min(a, b), hi = max(a, b);
                a = lo;
                b = hi;
            } else {
                const uint32_t ya = __shfl_xor_sync(kFull, a, j), yb = __shfl_xor_sync(kFull, b, j);
                const int ea = lane, eb = lane + 32;
                const bool keepLowA = ((ea & j) == 0) == ((ea & k) == 0);
                const bool keepLowB = ((eb & j) == 0) == ((eb & k) == 0);
                a = keepLowA ? min(a, ya) : max(a, ya);
                b = keepLowB ? min(b, yb) : max(b, yb);
            }
        }
    }
}

__device__ __forceinline__ float key_value(uint32_t k)
{
    if (k == 0xffffffffu) return __int_as_float(0x7fffffff);
    const uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    return __uint_as_float(u);
}

// Draw kinds after evaluation
constexpr int kDrawFail = 0;      // counted: no usable ellipse
constexpr int kDrawUsable = 1;    // S holds its median
constexpr int kDrawNotReal = 2;   // the reference's exception: not counted
constexpr int kDrawNoGain = 3;    // counted: its median cannot beat the best so far

// Five distinct residues read from mods[p0...] (rand_5_k without rejected
// outputs); returns the position after the last one read, or -1 when the
// pool ends first.  Registers only.
__device__ __forceinline__ int draw_from(const uint8_t* mods, int p0, int g[5])
{
    int n = 0, q = p0;
    int g0 = -1, g1 = -1, g2 = -1, g3 = -1, g4 = -1;
    while (n < 5) {
        if (q >= kRawPool) return -1;
        const int r = mods[q++];
        const bool seen = r == g0 || r == g1 || r == g2 || r == g3;
        if (seen) continue;
        if (n == 0) g0 = r;
        else if (n == 1) g1 = r;
        else if (n == 2) g2 = r;
        else if (n == 3) g3 = r;
        else g4 = r;
        ++n;
    }
    g[0] = g0;
    g[1] = g1;
    g[2] = g2;
    g[3] = g3;
    g[4] = g4;
    return q;
}

// Whether the (weighted) distance d(Q, p) * w of dist_point_ellipse is below
// S, decided exactly: an estimate with the fast reciprocal settles the cases
// that are more than 2^-16 (relative) away from S; the rest are computed with
// the IEEE expression.
__device__ __forceinline__ bool dist_below(const geo::Mat3& Q, float x, float y, bool weighted, float w, float S)
{
    const float aux0 = x * x, aux1 = 2 * x * y, aux2 = 2 * x, aux3 = y * y, aux4 = 2 * y;
    const float t1 = x * Q.m[0][0] + y * Q.m[0][1] + Q.m[0][2];
    const float t2 = x * Q.m[0][1] + y * Q.m[1][1] + Q.m[1][2];
    const float denom = t1 * t1 + t2 * t2;
    const float dot = aux0 * Q.m[0][0] + aux1 * Q.m[0][1] + aux2 * Q.m[0][2] + aux3 * Q.m[1][1] + aux4 * Q.m[1][2] +
                      Q.m[2][2];
    const float dd = dot * dot;
    float v = dd * __frcp_rn(denom);
    if (weighted) v *= w;
    if (v < S * 0.99998f) return true;
    if (v > S * 1.00002f && v <= 3.4e38f) return false;  // an infinite estimate is settled exactly
    float d = dd / denom;
    if (weighted) d *= w;
    return d < S;
}

// Block-wide outlierRemoval (Vote.cpp:414-576) with maxSize 60 over the n
// edge points idx[0, n) of level L: LMedS ellipse from random 5-point subsets
// of a regular subsample, drawn from `rng`, kDrawsPerBatch at a time and
// accepted in draw order; then idx is compacted in place (order kept) to the
// points whose distance (times 255 / |gradient| when weighted) is below
// threshold * the best median.  Returns their number (0 when fewer than 5
// points are subsampled).  Every thread of the block must call it.
__device__ int lmeds_outliers(const LoopOneLevel& L, int32_t* idx, int n, bool weighted, float threshold,
                              const geo::Pcg32 rng0, int32_t* err)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    __shared__ geo::Pt pts[kLmedsMaxPts];
    __shared__ float wts[kLmedsMaxPts];
    __shared__ uint32_t raws[kRawPool];
    __shared__ uint8_t mods[kRawPool];
    __shared__ int16_t lens[kRawPool];
    __shared__ uint32_t keysAll[kLmedsMaxPts * kFilterThreads];
    __shared__ int16_t starts[kFilterThreads];
    __shared__ int8_t perms[kFilterThreads][5];
    __shared__ int kinds[kFilterThreads];
    __shared__ float svals[kFilterThreads];
    __shared__ float sQ[kFilterThreads][9];
    __shared__ float bestQ[9];
    __shared__ int sNpts, sDone, sNd, sCounter, sDraws, sWarpCnt[kFilterThreads / 32];
    __shared__ float sSm;
    __shared__ unsigned long long sState, sInc;
    const int nchild = n;
    int32_t* children = idx;
    // The reference scans the children and takes child i when i equals
    // size_t(float(k) * step) for the next k: the taken indices are those
    // targets while they increase strictly and stay below nchild.
    const int nSub = min(nchild, 60);
    __shared__ long long sTarget[kLmedsMaxPts + 1];
    if (nSub >= 5 && tid <= kLmedsMaxPts) {
        const float step = float(nchild) / float(nSub);
        sTarget[tid] = (long long)size_t(float(size_t(tid)) * step);
    }
    __syncthreads();
    if (tid == 0) {
        int np = 0;
        if (nSub >= 5) {
            while (np <= kLmedsMaxPts && sTarget[np] < nchild && (np == 0 || sTarget[np] > sTarget[np - 1])) ++np;
            if (np > kLmedsMaxPts) atomicOr(err, kLoopOneErrPoints);
        }
        sNpts = np;
        for (int k = 0; k < 9; ++k) bestQ[k] = 0.f;
        sSm = 10000000.0f;
        sDone = 0;
        sCounter = 0;
        sDraws = 0;
        sState = rng0.state;
        sInc = rng0.inc;
    }
    __syncthreads();
    const int np = sNpts;
    if (np <= kLmedsMaxPts && tid < np) {
        const int e = children[sTarget[tid]];
        pts[tid] = {float(px_(L, e)), float(py_(L, e))};
        wts[tid] = 255.f / gnorm(L, e);
    }
    __syncthreads();
    if (nSub < 5 || np > kLmedsMaxPts) return 0;
    // ... then random 5-point conics, 128 draws at a time, accepted in order.
    const uint32_t rejectBelow = uint32_t(-uint32_t(np)) % uint32_t(np);
    while (!sDone) {
        // the next kRawPool outputs of the candidate's stream, 8 per thread
        {
            geo::Pcg32 g;
            g.state = sState;
            g.inc = sInc;
            g.advance(uint64_t(tid) * (kRawPool / kFilterThreads));
            for (int k = 0; k < kRawPool / kFilterThreads; ++k) {
                const uint32_t r = g.next();
                raws[tid * (kRawPool / kFilterThreads) + k] = r;
                mods[tid * (kRawPool / kFilterThreads) + k] = uint8_t(r % uint32_t(np));
            }
        }
        // Statistic.cpp:16-29 rand_5_k on that stream, as many whole draws as
        // it holds.  A bounded draw rejects an output only below 2^32 mod np
        // (< 64 of 2^32 values): when the pool holds none, a draw consumes
        // outputs until it has 5 distinct residues, so each position's draw
        // length is found in parallel and the draws chained from position 0.
        bool rejects = false;
        for (int k = 0; k < kRawPool / kFilterThreads; ++k)
            rejects = rejects || raws[tid * (kRawPool / kFilterThreads) + k] < rejectBelow;
        rejects = __syncthreads_or(rejects);
        if (!rejects) {
            for (int k = 0; k < kRawPool / kFilterThreads; ++k) {
                const int p0 = tid * (kRawPool / kFilterThreads) + k;
                int g[5];
                const int q = draw_from(mods, p0, g);
                lens[p0] = int16_t(q > 0 ? q - p0 : -1);
            }
            __syncthreads();
            if (tid == 0) {
                int ptr = 0, nd = 0;
                while (nd < kFilterThreads && ptr < kRawPool && lens[ptr] > 0) {
                    starts[nd++] = int16_t(ptr);
                    ptr += lens[ptr];
                }
                if (nd == 0) atomicOr(err, kLoopOneErrRandom);
                sNd = nd;
                geo::Pcg32 g;
                g.state = sState;
                g.inc = sInc;
                g.advance(uint64_t(ptr));
                sState = g.state;
            }
            __syncthreads();
            if (tid < sNd) {
                int g[5];
                draw_from(mods, starts[tid], g);
#pragma unroll
                for (int i = 0; i < 5; ++i) perms[tid][i] = int8_t(g[i]);
            }
        } else if (tid == 0) {
            int ptr = 0, nd = 0;
            while (nd < kFilterThreads) {
                int perm[5] = {-1, -1, -1, -1, -1};
                const int start = ptr;
                bool complete = true;
                for (int i = 0; i < 5 && complete; ++i) {
                    for (;;) {
                        if (ptr >= kRawPool) {
                            complete = false;
                            break;
                        }
                        const uint32_t raw = raws[ptr];
                        const int r = mods[ptr];
                        ++ptr;
                        if (raw < rejectBelow) continue;
                        bool seen = false;
                        for (int q = 0; q < i; ++q) seen = seen || perm[q] == r;
                        if (seen) continue;
                        perm[i] = r;
                        break;
                    }
                }
                if (!complete) {
                    ptr = start;
                    break;
                }
                for (int i = 0; i < 5; ++i) perms[nd][i] = int8_t(perm[i]);
                ++nd;
            }
            if (nd == 0) atomicOr(err, kLoopOneErrRandom);
            sNd = nd;
            geo::Pcg32 g;
            g.state = sState;
            g.inc = sInc;
            g.advance(uint64_t(ptr));
            sState = g.state;
        }
        __syncthreads();
        const int nd = sNd;
        if (nd == 0) break;
        const float SmStart = sSm;
        {
            const bool valid = tid < nd;
            geo::Mat3 Q = geo::Mat3::zero();
            int kind = kDrawNotReal;
            bool needS = false;
            if (valid) {
                int perm[5];
                for (int i = 0; i < 5; ++i) perm[i] = perms[tid][i];
                kind = cand::lmeds_conic(pts, perm, Q);
                if (kind == kDrawUsable) {
                    int below = 0;
#pragma unroll 4
                    for (int i = 0; i < np; ++i) below += dist_below(Q, pts[i].x, pts[i].y, weighted, wts[i], SmStart);
                    // no median below the best so far: it cannot improve (Sm only decreases)
                    if (below >= np / 2 + 1) {
                        needS = true;
                        uint32_t* keys = keysAll + tid;  // column tid of a [kLmedsMaxPts][kFilterThreads] array
                        for (int i = 0; i < np; ++i) {
                            float d = geo::dist_point_ellipse(Q, pts[i].x, pts[i].y);
                            if (weighted) d *= wts[i];
                            keys[i * kFilterThreads] = geo::order_key(d);
                        }
                    } else {
                        kind = kDrawNoGain;
                    }
                }
            }
            // medians (rank np / 2, NaN last) of the draws that need one, a draw at
            // a time by the whole warp: a 64-key bitonic sort of its column
            __syncwarp();
            float S = 0.f;
            for (unsigned m = __ballot_sync(kFull, needS); m; m &= m - 1) {
                const int src = __ffs(m) - 1;
                const uint32_t* col = keysAll + (warp * 32 + src);
                uint32_t ka = lane < np ? col[lane * kFilterThreads] : 0xffffffffu;
                uint32_t kb = lane + 32 < np ? col[(lane + 32) * kFilterThreads] : 0xffffffffu;
                bitonic64(ka, kb, lane);
                const int r = np / 2;
                const uint32_t v = __shfl_sync(kFull, r < 32 ? ka : kb, r & 31);
                if (lane == src) S = key_value(v);
            }
            if (valid) {
                kinds[tid] = kind;
                svals[tid] = S;
                for (int k = 0; k < 9; ++k) sQ[tid][k] = Q.m[k / 3][k % 3];
            }
        }
        __syncthreads();
        // Acceptance in draw order (Vote.cpp:478-545) by warp 0, 32 draws at a
        // time: draw j improves when its median is below the best before it,
        // which is the minimum of the carried best and every usable median
        // before j; the no-gain counter restarts at each improvement, and the
        // loop stops before the first draw at which it has reached 70 (or the
        // draws 7000).
        if (warp == 0) {
            int counter = sCounter, draws = sDraws, best = -1;
            float Sm = sSm;
            bool stopped = false;
            for (int c0 = 0; c0 < nd && !stopped; c0 += 32) {
                const int j = c0 + lane;
                const bool valid = j < nd;
                const int kind = valid ? kinds[j] : kDrawNotReal;
                const bool usable = valid && kind == kDrawUsable;
                const float Sj = usable ? svals[j] : __int_as_float(0x7f800000);
                float incl = Sj;
                for (int o = 1; o < 32; o <<= 1) {
                    const float v = __shfl_up_sync(kFull, incl, o);
                    if (lane >= o) incl = fminf(incl, v);
                }
                float excl = __shfl_up_sync(kFull, incl, 1);
                if (lane == 0) excl = __int_as_float(0x7f800000);
                const bool improving = usable && Sj < fminf(Sm, excl);
                const bool counted = valid && (kind == kDrawFail || kind == kDrawNoGain || (usable && !improving));
                const unsigned impM = __ballot_sync(kFull, improving);
                const unsigned cntM = __ballot_sync(kFull, counted);
                const unsigned lower = (1u << lane) - 1u;
                const unsigned impBefore = impM & lower;
                int cb;
                if (impBefore) {
                    const int last = 31 - __clz(impBefore);
                    cb = __popc(cntM & lower & ~((2u << last) - 1u));
                } else {
                    cb = counter + __popc(cntM & lower);
                }
                const bool stopHere = valid && !(cb < 70 && draws + lane < 7000);
                const unsigned stopM = __ballot_sync(kFull, stopHere);
                const int n = min(nd - c0, 32);
                const int js = stopM ? __ffs(stopM) - 1 : n;
                const unsigned proc = js >= 32 ? 0xffffffffu : ((1u << js) - 1u);
                const unsigned impP = impM & proc;
                if (impP) {
                    const int last = 31 - __clz(impP);
                    best = c0 + last;
                    Sm = __shfl_sync(kFull, Sj, last);
                    counter = __popc(cntM & proc & ~((2u << last) - 1u));
                } else {
                    counter += __popc(cntM & proc);
                }
                draws += js;
                stopped = stopM != 0;
            }
            if (lane == 0) {
                if (best >= 0)
                    for (int k = 0; k < 9; ++k) bestQ[k] = sQ[best][k];
                sCounter = counter;
                sDraws = draws;
                sSm = Sm;
                if (stopped || !(counter < 70 && draws < 7000)) sDone = 1;
            }
        }
        __syncthreads();
    }
    // the children whose weighted distance is below threshold * median, in order
    geo::Mat3 Q;
    for (int k = 0; k < 9; ++k) Q.m[k / 3][k % 3] = bestQ[k];
    const float thr = threshold * sSm;
    int nflt = 0;
    for (int c0 = 0; c0 < nchild; c0 += kFilterThreads) {
        const int i = c0 + tid;
        int e = -1;
        if (i < nchild) e = children[i];
        __syncthreads();  // every element of the chunk read before any is overwritten
        bool pass = false;
        if (e >= 0) {
            float d = geo::dist_point_ellipse(Q, float(px_(L, e)), float(py_(L, e)));
            if (weighted) d = d * 255 / gnorm(L, e);
            pass = d < thr;
        }
        const unsigned mask = __ballot_sync(kFull, pass);
        if (lane == 0) sWarpCnt[warp] = __popc(mask);
        __syncthreads();
        int off = nflt;
        for (int w = 0; w < warp; ++w) off += sWarpCnt[w];
        if (pass) children[off + __popc(mask & ((1u << lane) - 1u))] = e;
        for (int w = 0; w < kFilterThreads / 32; ++w) nflt += sWarpCnt[w];
        __syncthreads();
    }
    return nflt;
}


__global__ void __launch_bounds__(kFilterThreads) k_filter(LoopOneArgs a)
{
    const int l = blockIdx.x / a.n2max, rank = blockIdx.x % a.n2max;
    const LoopOneLevel& L = a.lv[l];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int madeCount = a.meta[size_t(a.nl) * a.n2max * 4 + l];
    if (rank >= min(madeCount, a.n2max)) return;
    int32_t* meta = a.meta + (size_t(l) * a.n2max + rank) * 4;
    const int s = meta[0];
    const int t = L.slot0 + s;
    const int32_t* info = a.sinfo + size_t(t) * 4;
    const int nf = info[0], nb = info[1];
    const int32_t* segc = a.seg + size_t(t) * kSegSlot + kSegHalf;
    const int len = nf + 1 + nb;
    int32_t* children = a.children + size_t(blockIdx.x) * a.childCap;
    if (threadIdx.x == 0) a.cflow[blockIdx.x] = L.flow[L.order[s]];

    __shared__ int sNchild;

    // children (Vote.cpp:396-412): voters of the points with >= voteMax/14 votes
    if (warp == 0) {
        int vmax = 1;
        for (int k = lane; k < len; k += 32) vmax = max(vmax, voters(L, segc[-nf + k]));
        for (int o = 16; o; o >>= 1) vmax = max(vmax, __shfl_xor_sync(kFull, vmax, o));
        int nchild = 0;
        for (int c0 = 0; c0 < len; c0 += 32) {
            const int pos = c0 + lane;
            const int e = pos < len ? segc[-nf + pos] : -1;
            const int n = e >= 0 ? voters(L, e) : 0;
            const int cnt = (n > 0 && n >= vmax / 14) ? n : 0;
            int incl = cnt;
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(kFull, incl, o);
                if (lane >= o) incl += v;
            }
            const int excl = incl - cnt;
            const int base = cnt ? L.voff[e] : 0;
            const int tot = __shfl_sync(kFull, incl, 31);
            // the chunk's voter lists, 32 entries at a time: entry o belongs to
            // the first lane whose inclusive count exceeds o
            for (int o0 = 0; o0 < tot; o0 += 32) {
                const int o = o0 + lane;
                int w = 0;
                for (int b = 16; b > 0; b >>= 1)
                    if (__shfl_sync(kFull, incl, w + b - 1) <= o) w += b;
                const int wbase = __shfl_sync(kFull, base, w & 31);
                const int wexcl = __shfl_sync(kFull, excl, w & 31);
                if (o < tot && nchild + o < a.childCap) children[nchild + o] = L.vlist[wbase + (o - wexcl)];
            }
            nchild += tot;
        }
        if (lane == 0) sNchild = nchild;
    }
    __syncthreads();
    const int nchild = sNchild;
    if (nchild > a.childCap) {
        if (tid == 0) {
            atomicOr(a.err, kLoopOneErrChildren);
            meta[0] = L.order[s];
            meta[1] = nchild;
            meta[2] = 0;
            meta[3] = 0;
        }
        return;
    }
    if (nchild < a.minPoints) {
        if (tid == 0) {
            meta[0] = L.order[s];
            meta[1] = 0;
            meta[2] = 0;
            meta[3] = 0;
        }
        return;
    }

    // outlierRemoval with inverse-gradient weights (Detection.cpp:131-133)
    const int nflt = lmeds_outliers(L, children, nchild, true, a.threshold,
                                    cand::candidate_rng(L.level, uint64_t(rank), 0), a.err);
    if (tid == 0) {
        meta[0] = L.order[s];
        meta[1] = nchild;
        meta[2] = nflt >= 5 ? 1 : 0;
        meta[3] = nflt;
    }
}

// float -> int as the host's conversion does it on x86-64: out of range and
// NaN give INT_MIN (the device instruction would saturate instead).
__device__ __forceinline__ int host_int(float f)
{
    return (f >= -2147483648.0f && f < 2147483648.0f) ? int(f) : int(0x80000000u);
}

// Multiresolution.cpp:43-142 intersectLineToTwoEllipses for row y: whether the
// row counts, and up to two x ranges to scan.
__device__ bool refit_row(const geo::Mat3& Qi, const geo::Mat3& Qo, int W, int y, int& nr, int xb[2], int xe[2])
{
    float io[2], ii[2];
    const int no = geo::intersect_line_q(Qo, float(y), true, io);
    const int ni = geo::intersect_line_q(Qi, float(y), true, ii);
    nr = 0;
    if (no == 2 && ni == 2) {
        nr = 2;
        xb[0] = max(0, host_int(io[0]));
        xe[0] = min(W - 1, host_int(ii[0]));
        xb[1] = max(0, host_int(ii[1]));
        xe[1] = min(W - 1, host_int(io[1]));
    } else if (no == 2 && ni <= 1) {
        nr = 1;
        xb[0] = max(0, host_int(io[0]));
        xe[0] = min(W - 1, host_int(io[1]));
    } else if (no == 1 && ni == 0) {
        if (io[0] >= 0 && io[0] < float(W)) {
            nr = 1;
            xb[0] = xe[0] = host_int(io[0]);
        }
    } else {
        return false;
    }
    return true;
}

// Edge points of row y taken into the hull, in x order: written at out[]
// when out is not null; returns their number.
__device__ int refit_row_takes(const LoopOneLevel& L, const geo::Mat3& Qi, const geo::Mat3& Qo, float inCx,
                               float inCy, int y, int32_t* out)
{
    int nr, xb[2], xe[2];
    if (!refit_row(Qi, Qo, L.W, y, nr, xb, xe)) return 0;
    int n = 0;
    // the edge pixels of each x range, a bitmap word at a time, in x order
    const uint2* row = L.bitidx + size_t(y) * L.WW;
    for (int r = 0; r < nr; ++r) {
        if (xb[r] > xe[r]) continue;
        for (int wx = xb[r] >> 5; wx <= xe[r] >> 5; ++wx) {
            const int lo = wx << 5;
            const uint2 word = row[wx];
            uint32_t w = word.x;
            if (xb[r] > lo) w &= 0xffffffffu << (xb[r] - lo);
            if (xe[r] < lo + 31) w &= 0xffffffffu >> (31 - (xe[r] - lo));
            while (w) {
                const int b = __ffs(w) - 1;
                w &= w - 1;
                const int e = int(word.y) + __popc(word.x & ((1u << b) - 1u));
                if (e >= L.E) break;  // past a clamped edge count
                const float cx = inCx - float(px_(L, e)), cy = inCy - float(py_(L, e));
                if (gdx(L, e) * cx + gdy(L, e) * cy < 0) {
                    if (out) out[n] = e;
                    ++n;
                }
            }
        }
    }
    return n;
}

// Multiresolution.cpp:319-401: level-0 hull of one coarse-level marker (rows
// from the center row down the image until one misses the hull, then from
// the center row up), then the outlier removal without weights.
__global__ void __launch_bounds__(kFilterThreads) k_refit(LoopOneLevel L, const RefitTask* tasks, int32_t* hullAll,
                                                        int hullCap, int32_t* rowsAll, int rowStride, int32_t* counts)
{
    const int b = blockIdx.x, tid = threadIdx.x;
    const RefitTask& T = tasks[b];
    int32_t* hull = hullAll + size_t(b) * hullCap;
    int32_t* rowOff = rowsAll + size_t(b) * rowStride;
    int32_t* err = counts + gridDim.x;
    geo::Mat3 Qi, Qo;
    for (int k = 0; k < 9; ++k) {
        Qi.m[k / 3][k % 3] = T.qin[k];
        Qo.m[k / 3][k % 3] = T.qout[k];
    }
    const int maxY = max(host_int(T.yc), 0);
    const int minY = min(host_int(T.yc), L.H - 1);
    __shared__ int sUpEnd, sDownEnd, sTotal;
    __shared__ int sPart[kFilterThreads];
    if (tid == 0) {
        sUpEnd = L.H;
        sDownEnd = -1;
    }
    __syncthreads();
    int nr, xb[2], xe[2];
    for (int y = maxY + tid; y < L.H; y += blockDim.x)
        if (!refit_row(Qi, Qo, L.W, y, nr, xb, xe)) atomicMin(&sUpEnd, y);
    for (int y = minY - tid; y >= 0; y -= blockDim.x)
        if (!refit_row(Qi, Qo, L.W, y, nr, xb, xe)) atomicMax(&sDownEnd, y);
    __syncthreads();
    const int rUp = max(sUpEnd - maxY, 0), rDown = max(minY - sDownEnd, 0);
    const int R = rUp + rDown;
    auto row_y = [&](int r) { return r < rUp ? maxY + r : minY - (r - rUp); };
    // per-row counts in processing order, contiguous chunks per thread
    const int chunk = (R + blockDim.x - 1) / blockDim.x;
    const int r0 = min(R, tid * chunk), r1 = min(R, r0 + chunk);
    int part = 0;
    for (int r = r0; r < r1; ++r) {
        const int c = refit_row_takes(L, Qi, Qo, T.inCx, T.inCy, row_y(r), nullptr);
        rowOff[r] = c;
        part += c;
    }
    sPart[tid] = part;
    __syncthreads();
    if (tid == 0) {
        int acc = 0;
        for (int k = 0; k < int(blockDim.x); ++k) {
            const int v = sPart[k];
            sPart[k] = acc;
            acc += v;
        }
        sTotal = acc;
    }
    __syncthreads();
    const int total = sTotal;
    if (total > hullCap) {
        if (tid == 0) {
            atomicOr(err, kLoopOneErrChildren);
            counts[b] = -1;
        }
        return;
    }
    int off = sPart[tid];
    for (int r = r0; r < r1; ++r) {
        const int c = rowOff[r];
        refit_row_takes(L, Qi, Qo, T.inCx, T.inCy, row_y(r), hull + off);
        off += c;
    }
    __syncthreads();
    if (total < 5) {
        if (tid == 0) counts[b] = -1;
        return;
    }
    const geo::Pcg32 rng(271828, (uint64_t(1) << 62) | uint64_t(T.marker));
    const int nflt = lmeds_outliers(L, hull, total, false, 20.0f, rng, err);
    if (tid == 0) counts[b] = nflt;
}

__global__ void __launch_bounds__(256) k_refit_pack(const int32_t* hullAll, int hullCap, const int32_t* counts,
                                                    int32_t* packed)
{
    const int b = blockIdx.x;
    __shared__ int sOff;
    const int n = counts[b];
    if (n <= 0) return;
    if (threadIdx.x == 0) {
        int off = 0;
        for (int q = 0; q < b; ++q) off += max(counts[q], 0);
        sOff = off;
    }
    __syncthreads();
    const int32_t* src = hullAll + size_t(b) * hullCap;
    for (int i = threadIdx.x; i < n; i += blockDim.x) packed[sOff + i] = src[i];
}

// Kept candidates' filtered children, in candidate order, into one array.
// The link chains of the packed filtered children: point i of level l (the
// levels' entries are contiguous, from first[l]) walks len alternating
// before / after links, as addCandidateFlowtoCCTag does (EllipseGrowing.cpp:
// 63-178).
struct ChainLevels {
    const int32_t* before[kMaxLevels];
    const int32_t* after[kMaxLevels];
    int first[kMaxLevels + 1];
};

__global__ void __launch_bounds__(256) k_chains(const int32_t* __restrict__ packed, int total, int len,
                                                ChainLevels cl, int nl, int32_t* __restrict__ chain)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    int l = 0;
    while (l < nl - 1 && i >= cl.first[l + 1]) ++l;
    int q = packed[i];
    for (int j = 0; j < len; ++j) {
        q = q < 0 ? -1 : (j & 1) ? cl.after[l][q] : cl.before[l][q];
        chain[size_t(i) * len + j] = q;
    }
}

__global__ void __launch_bounds__(256) k_pack(LoopOneArgs a, int32_t* packed)
{
    const int b = blockIdx.x;
    const int l = b / a.n2max, rank = b % a.n2max;
    __shared__ int sOff;
    const int n2 = min(a.meta[size_t(a.nl) * a.n2max * 4 + l], a.n2max);
    if (rank >= n2) return;
    const int32_t* meta = a.meta + size_t(b) * 4;
    if (!meta[2]) return;
    if (threadIdx.x == 0) {
        int off = 0;
        for (int q = 0; q < b; ++q) {
            const int lq = q / a.n2max, rq = q % a.n2max;
            const int n2q = min(a.meta[size_t(a.nl) * a.n2max * 4 + lq], a.n2max);
            if (rq < n2q && a.meta[size_t(q) * 4 + 2]) off += a.meta[size_t(q) * 4 + 3];
        }
        sOff = off;
    }
    __syncthreads();
    const int32_t* src = a.children + size_t(b) * a.childCap;
    for (int i = threadIdx.x; i < meta[3]; i += blockDim.x) packed[sOff + i] = src[i];
}

template <class T>
T* dev_alloc(std::vector<void*>& list, size_t n)
{
    void* p = nullptr;
    CCTAGB_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
    list.push_back(p);
    return static_cast<T*>(p);
}

}  // namespace

LoopOneGpu::LoopOneGpu(const cctagb_params& p, int max_h, const std::vector<int>& caps) : p_(p)
{
    if (p.windowSizeOnInnerEllipticSegment < 1 || p.windowSizeOnInnerEllipticSegment > cand::kLinkMaxWindow)
        throw Error{CCTAGB_BAD_ARG, "windowSizeOnInnerEllipticSegment must be in [1, 64]"};
    if (p.maximumNbCandidatesLoopTwo < 1 || p.maximumNbCandidatesLoopTwo > 1024)
        throw Error{CCTAGB_BAD_ARG, "maximumNbCandidatesLoopTwo must be in [1, 1024]"};
    nl_ = int(caps.size());
    n2max_ = p.maximumNbCandidatesLoopTwo;
    waiter_.init(p.hostSpinMicros);
    // seeds processed per level: max(rows / 2, maximumNbSeeds) (Detection.cpp:603-605);
    // level 0 has the most rows
    maxSlotsPerLevel_ = std::max(max_h / 2, p.maximumNbSeeds);
    maxH_ = max_h;
    totalSlots_ = nl_ * maxSlotsPerLevel_;
    size_t nrec = 0;
    for (int l = 0; l < nl_; ++l) {
        caps_.push_back(caps[size_t(l)]);
        nrec += size_t(caps[size_t(l)]);
    }
    args_.seg = dev_alloc<int32_t>(allocs_, size_t(totalSlots_) * kSegSlot);
    args_.sinfo = dev_alloc<int32_t>(allocs_, size_t(totalSlots_) * 4);
    args_.mlist = dev_alloc<int32_t>(allocs_, size_t(totalSlots_) * kMarkCap);
    args_.skey = dev_alloc<float>(allocs_, size_t(totalSlots_));
    args_.made = dev_alloc<int32_t>(allocs_, size_t(totalSlots_));
    const size_t metaN = size_t(nl_) * n2max_ * 4 + nl_ + 1;
    args_.meta = dev_alloc<int32_t>(allocs_, metaN);
    args_.cflow = dev_alloc<float>(allocs_, size_t(nl_) * n2max_);
    args_.err = args_.meta + size_t(nl_) * n2max_ * 4 + nl_;

    d_order_ = dev_alloc<int32_t>(allocs_, size_t(totalSlots_));
    d_rec_ = dev_alloc<int4>(allocs_, nrec * 3);
    for (int l = 0; l < nl_; ++l) maxCap_ = std::max(maxCap_, size_t(caps[size_t(l)]));
    grow_children(std::min<size_t>(kChildCap, maxCap_ + 1));
    CCTAGB_CUDA(cudaMallocHost(&h_order_, sizeof(int32_t) * std::max(totalSlots_, 1)));
    CCTAGB_CUDA(cudaMallocHost(&h_meta_, sizeof(int32_t) * metaN));
    CCTAGB_CUDA(cudaMallocHost(&h_cflow_, sizeof(float) * size_t(nl_) * n2max_));
    h_flt_cap_ = size_t(nl_) * n2max_ * 512;
    CCTAGB_CUDA(cudaMallocHost(&h_flt_, sizeof(int32_t) * h_flt_cap_));
    args_.maxSlotsPerLevel = maxSlotsPerLevel_;
    args_.totalSlots = totalSlots_;
    args_.nl = nl_;
    args_.window = p.windowSizeOnInnerEllipticSegment;
    args_.averageVoteMin = p.averageVoteMin;
    args_.n2max = n2max_;
    args_.minPoints = p.minPointsSegmentCandidate;
    args_.threshold = p.threshRobustEstimationOfOuterEllipse;
    // The attribute is per kernel and shared by every handle: set it to what
    // the device allows, so that no handle lowers it below another's need.
    int dev = 0, optin = 0;
    CCTAGB_CUDA(cudaGetDevice(&dev));
    CCTAGB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const int maxSmem = optin - 1024;  // room for the kernel's static shared memory
    if (resolve_smem() > maxSmem)
        throw Error{CCTAGB_BAD_ARG, "maximumNbSeeds / frame height too large for the loop-one resolve kernel"};
    CCTAGB_CUDA(cudaFuncSetAttribute(k_link_resolve, cudaFuncAttributeMaxDynamicSharedMemorySize, maxSmem));
}

int LoopOneGpu::resolve_smem() const
{
    return int(sizeof(int) * (3 * size_t(maxSlotsPerLevel_) + 1 + kResolveSmemMarks));
}

LoopOneGpu::~LoopOneGpu()
{
    for (void* q : allocs_) cudaFree(q);
    if (args_.children) cudaFree(args_.children);
    if (d_packed_) cudaFree(d_packed_);
    for (void* q : {static_cast<void*>(d_rtask_), static_cast<void*>(d_rhull_), static_cast<void*>(d_rrows_),
                    static_cast<void*>(d_rcount_), static_cast<void*>(d_rpacked_)})
        if (q) cudaFree(q);
    if (h_rtask_) cudaFreeHost(h_rtask_);
    if (h_rcount_) cudaFreeHost(h_rcount_);
    if (h_rpacked_) cudaFreeHost(h_rpacked_);
    if (h_order_) cudaFreeHost(h_order_);
    if (h_meta_) cudaFreeHost(h_meta_);
    if (h_cflow_) cudaFreeHost(h_cflow_);
    if (h_flt_) cudaFreeHost(h_flt_);
    if (d_chain_) cudaFree(d_chain_);
    if (h_chain_) cudaFreeHost(h_chain_);
}

void LoopOneGpu::launch(const Levels& lv, const int* E, const std::vector<const std::vector<int32_t>*>& seeds,
                        cudaStream_t s)
{
    if (lv.n != nl_ || int(seeds.size()) != nl_) throw Error{CCTAGB_BAD_ARG, "loop one: level count changed"};
    h2d_ = d2h_ = 0;
    size_t roff = 0;
    int cum[kMaxLevels] = {};
    for (int l = 0; l < nl_; ++l) {
        const LevelView& v = lv.l[l];
        LoopOneLevel& L = args_.lv[l];
        L.W = v.W;
        L.H = v.H;
        L.WW = v.WW;
        L.E = E[l];
        L.exy = v.exy;
        L.grad = v.grad;
        L.voff = v.voff;
        L.vlist = v.vlist;
        L.bitidx = v.bitidx;
        L.before = v.before;
        L.after = v.after;
        L.flow = v.flow;
        L.level = l;
        L.slot0 = l * maxSlotsPerLevel_;
        const size_t nMax = size_t(std::max(v.H / 2, p_.maximumNbSeeds));
        L.nProc = int(std::min(seeds[l]->size(), nMax));
        L.order = d_order_ + L.slot0;
        std::copy(seeds[l]->begin(), seeds[l]->begin() + L.nProc, h_order_ + L.slot0);
        if (v.cap > caps_[size_t(l)]) throw Error{CCTAGB_INTERNAL, "loop one: level capacity changed"};
        if (E[l] > caps_[size_t(l)]) throw Error{CCTAGB_INTERNAL, "loop one: more edge points than capacity"};
        L.rec = d_rec_ + 3 * roff;
        roff += size_t(caps_[size_t(l)]);
        cum[l] = (l ? cum[l - 1] : 0) + E[l];
        if (L.nProc)
            CCTAGB_CUDA(cudaMemcpyAsync(d_order_ + L.slot0, h_order_ + L.slot0, sizeof(int32_t) * L.nProc,
                                        cudaMemcpyHostToDevice, s));
        h2d_ += 4LL * L.nProc;
    }
    for (int l = nl_; l < kMaxLevels; ++l) cum[l] = cum[nl_ - 1];
    cum_ = make_int4(cum[0], cum[1], cum[2], cum[3]);
    run_kernels(s);
}

void LoopOneGpu::grow_children(size_t cap)
{
    if (args_.children) cudaFree(args_.children);
    if (d_packed_) cudaFree(d_packed_);
    args_.children = nullptr;
    d_packed_ = nullptr;
    args_.childCap = 0;
    const size_t n = size_t(nl_) * n2max_ * cap;
    CCTAGB_CUDA(cudaMalloc(&args_.children, sizeof(int32_t) * n));
    CCTAGB_CUDA(cudaMalloc(&d_packed_, sizeof(int32_t) * n));
    args_.childCap = int(cap);
}

void LoopOneGpu::run_kernels(cudaStream_t s)
{
    const size_t metaN = size_t(nl_) * n2max_ * 4 + nl_ + 1;
    CCTAGB_CUDA(cudaMemsetAsync(args_.meta, 0, sizeof(int32_t) * metaN, s));
    const int cumv[kMaxLevels] = {cum_.x, cum_.y, cum_.z, cum_.w};
    const int npts = nl_ > 0 ? cumv[nl_ - 1] : 0;
    if (npts > 0) {
        k_point_records<<<(npts + 255) / 256, 256, 0, s>>>(args_, cum_);
        CCTAGB_CUDA(cudaGetLastError());
    }
    k_seed_slots<<<(totalSlots_ + 255) / 256, 256, 0, s>>>(args_);
    CCTAGB_CUDA(cudaGetLastError());
    k_link_seeds<<<(totalSlots_ + kLinkGroups - 1) / kLinkGroups, kLinkThreads, 0, s>>>(args_);
    CCTAGB_CUDA(cudaGetLastError());
    k_link_resolve<<<nl_, kResolveThreads, resolve_smem(), s>>>(args_);
    CCTAGB_CUDA(cudaGetLastError());
    k_filter<<<nl_ * n2max_, kFilterThreads, 0, s>>>(args_);
    CCTAGB_CUDA(cudaGetLastError());
    k_pack<<<nl_ * n2max_, 256, 0, s>>>(args_, d_packed_);
    CCTAGB_CUDA(cudaGetLastError());
    CCTAGB_CUDA(cudaMemcpyAsync(h_meta_, args_.meta, sizeof(int32_t) * metaN, cudaMemcpyDeviceToHost, s));
    CCTAGB_CUDA(cudaMemcpyAsync(h_cflow_, args_.cflow, sizeof(float) * size_t(nl_) * n2max_,
                                cudaMemcpyDeviceToHost, s));
    d2h_ += 4LL * metaN + 4LL * nl_ * n2max_;
}

void LoopOneGpu::collect(cudaStream_t s, std::vector<LoopTwoIn>& out)
{
    chainLaunches_ = 0;
    waiter_.wait(s);
    const int32_t* made = h_meta_ + size_t(nl_) * n2max_ * 4;
    // a candidate with more voters than the room: more room, same kernels
    // (no list can hold more points than its level)
    while ((made[nl_] & kLoopOneErrChildren) && size_t(args_.childCap) <= maxCap_) {
        grow_children(std::min(size_t(args_.childCap) * 4, maxCap_ + 1));
        run_kernels(s);
        waiter_.wait(s);
    }
    const int err = made[nl_];
    if (err & kLoopOneErrChildren)
        throw Error{CCTAGB_OVERFLOW_VOTERS, "a loop-two candidate gathers more voters than its level has points"};
    if (err) throw Error{CCTAGB_INTERNAL, "loop one: error bits " + std::to_string(err)};
    size_t total = 0;
    for (int l = 0; l < nl_; ++l) {
        const int n2 = std::min(made[l], n2max_);
        for (int r = 0; r < n2; ++r) {
            const int32_t* m = h_meta_ + (size_t(l) * n2max_ + r) * 4;
            if (m[2]) total += size_t(m[3]);
        }
    }
    if (total > h_flt_cap_) {
        cudaFreeHost(h_flt_);
        h_flt_ = nullptr;
        h_flt_cap_ = 0;
        CCTAGB_CUDA(cudaMallocHost(&h_flt_, sizeof(int32_t) * total));
        h_flt_cap_ = total;
    }
    // the link chains of the filtered children (the host's flow assembling
    // walks them; the links themselves stay on the device)
    const int len = 2 * p_.nCrowns - 1;
    ChainLevels cl{};
    {
        size_t off = 0;
        for (int l = 0; l < nl_; ++l) {
            cl.before[l] = args_.lv[l].before;
            cl.after[l] = args_.lv[l].after;
            cl.first[l] = int(off);
            const int n2 = std::min(made[l], n2max_);
            for (int r = 0; r < n2; ++r) {
                const int32_t* m = h_meta_ + (size_t(l) * n2max_ + r) * 4;
                if (m[2]) off += size_t(m[3]);
            }
        }
        cl.first[nl_] = int(off);
    }
    if (total * len > chain_cap_) {
        if (d_chain_) cudaFree(d_chain_);
        if (h_chain_) cudaFreeHost(h_chain_);
        d_chain_ = nullptr;
        h_chain_ = nullptr;
        chain_cap_ = 0;
        const size_t cap = std::max(total * len, size_t(65536));
        CCTAGB_CUDA(cudaMalloc(&d_chain_, sizeof(int32_t) * cap));
        CCTAGB_CUDA(cudaMallocHost(&h_chain_, sizeof(int32_t) * cap));
        chain_cap_ = cap;
    }
    if (total) {
        k_chains<<<int((total + 255) / 256), 256, 0, s>>>(d_packed_, int(total), len, cl, nl_, d_chain_);
        CCTAGB_CUDA(cudaGetLastError());
        ++chainLaunches_;
        CCTAGB_CUDA(cudaMemcpyAsync(h_flt_, d_packed_, sizeof(int32_t) * total, cudaMemcpyDeviceToHost, s));
        CCTAGB_CUDA(cudaMemcpyAsync(h_chain_, d_chain_, sizeof(int32_t) * total * len, cudaMemcpyDeviceToHost, s));
        waiter_.wait(s);
    }
    d2h_ += 4LL * total * (1 + len);
    out.assign(size_t(nl_), {});
    size_t off = 0;
    for (int l = 0; l < nl_; ++l) {
        LoopTwoIn& o = out[size_t(l)];
        const int n2 = std::min(made[l], n2max_);
        o.chainLen = len;
        o.foff.push_back(0);
        for (int r = 0; r < n2; ++r) {
            const int32_t* m = h_meta_ + (size_t(l) * n2max_ + r) * 4;
            o.seed.push_back(m[0]);
            o.flow.push_back(h_cflow_[size_t(l) * n2max_ + r]);
            o.score.push_back(m[1]);
            o.keep.push_back(uint8_t(m[2]));
            if (m[2]) {
                o.flt.insert(o.flt.end(), h_flt_ + off, h_flt_ + off + m[3]);
                o.chain.insert(o.chain.end(), h_chain_ + off * len, h_chain_ + (off + m[3]) * len);
                off += size_t(m[3]);
            }
            o.foff.push_back(int32_t(o.flt.size()));
        }
    }
}

void LoopOneGpu::ensure_refit_capacity(int n)
{
    if (n <= refitCap_) return;
    for (void* q : {static_cast<void*>(d_rtask_), static_cast<void*>(d_rhull_), static_cast<void*>(d_rrows_),
                    static_cast<void*>(d_rcount_), static_cast<void*>(d_rpacked_)})
        if (q) cudaFree(q);
    if (h_rtask_) cudaFreeHost(h_rtask_);
    if (h_rcount_) cudaFreeHost(h_rcount_);
    d_rtask_ = nullptr;
    d_rhull_ = d_rrows_ = d_rcount_ = d_rpacked_ = nullptr;
    h_rtask_ = nullptr;
    h_rcount_ = nullptr;
    refitCap_ = 0;
    const int cap = std::max(n, 64);
    CCTAGB_CUDA(cudaMalloc(&d_rtask_, sizeof(RefitTask) * cap));
    CCTAGB_CUDA(cudaMalloc(&d_rhull_, sizeof(int32_t) * size_t(cap) * hullCap_));
    CCTAGB_CUDA(cudaMalloc(&d_rrows_, sizeof(int32_t) * size_t(cap) * (maxH_ + 2)));
    CCTAGB_CUDA(cudaMalloc(&d_rcount_, sizeof(int32_t) * (cap + 1)));
    CCTAGB_CUDA(cudaMalloc(&d_rpacked_, sizeof(int32_t) * size_t(cap) * hullCap_));
    CCTAGB_CUDA(cudaMallocHost(&h_rtask_, sizeof(RefitTask) * cap));
    CCTAGB_CUDA(cudaMallocHost(&h_rcount_, sizeof(int32_t) * (cap + 1)));
    refitCap_ = cap;
}

void LoopOneGpu::refit(const Levels& lv, const std::vector<RefitTask>& tasks, cudaStream_t s,
                       std::vector<std::vector<int32_t>>& filtered)
{
    const int n = int(tasks.size());
    filtered.assign(size_t(n), {});
    if (n == 0) return;
    ensure_refit_capacity(n);
    const LevelView& v = lv.l[0];
    if (v.H > maxH_) throw Error{CCTAGB_INTERNAL, "refit: frame taller than the handle"};
    LoopOneLevel L = args_.lv[0];  // level-0 view of the frame loop one ran on
    std::copy(tasks.begin(), tasks.end(), h_rtask_);
    CCTAGB_CUDA(cudaMemcpyAsync(d_rtask_, h_rtask_, sizeof(RefitTask) * n, cudaMemcpyHostToDevice, s));
    // the hull of one marker holds at most every level-0 point and a row twice
    const size_t hullMax = size_t(L.E) + size_t(L.W) + 1;
    for (;;) {
        CCTAGB_CUDA(cudaMemsetAsync(d_rcount_ + n, 0, sizeof(int32_t), s));
        k_refit<<<n, kFilterThreads, 0, s>>>(L, d_rtask_, d_rhull_, hullCap_, d_rrows_, maxH_ + 2, d_rcount_);
        CCTAGB_CUDA(cudaGetLastError());
        k_refit_pack<<<n, 256, 0, s>>>(d_rhull_, hullCap_, d_rcount_, d_rpacked_);
        CCTAGB_CUDA(cudaGetLastError());
        CCTAGB_CUDA(cudaMemcpyAsync(h_rcount_, d_rcount_, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToHost, s));
        waiter_.wait(s);
        if (!(h_rcount_[n] & kLoopOneErrChildren) || size_t(hullCap_) > hullMax) break;
        // more room for the hulls, same kernels
        hullCap_ = int(std::min(size_t(hullCap_) * 4, hullMax + 1));
        const int keep = refitCap_;
        refitCap_ = 0;
        ensure_refit_capacity(keep);
        std::copy(tasks.begin(), tasks.end(), h_rtask_);
        CCTAGB_CUDA(cudaMemcpyAsync(d_rtask_, h_rtask_, sizeof(RefitTask) * n, cudaMemcpyHostToDevice, s));
    }
    const int err = h_rcount_[n];
    if (err & kLoopOneErrChildren)
        throw Error{CCTAGB_OVERFLOW_VOTERS, "a re-fit hull holds more points than level 0"};
    if (err) throw Error{CCTAGB_INTERNAL, "refit: error bits " + std::to_string(err)};
    size_t total = 0;
    for (int i = 0; i < n; ++i) total += size_t(std::max(h_rcount_[i], 0));
    if (total > h_rpacked_cap_) {
        if (h_rpacked_) cudaFreeHost(h_rpacked_);
        h_rpacked_ = nullptr;
        h_rpacked_cap_ = 0;
        CCTAGB_CUDA(cudaMallocHost(&h_rpacked_, sizeof(int32_t) * std::max<size_t>(total, 4096)));
        h_rpacked_cap_ = std::max<size_t>(total, 4096);
    }
    if (total) {
        CCTAGB_CUDA(cudaMemcpyAsync(h_rpacked_, d_rpacked_, sizeof(int32_t) * total, cudaMemcpyDeviceToHost, s));
        waiter_.wait(s);
    }
    h2d_ += (long long)sizeof(RefitTask) * n;
    d2h_ += 4LL * (n + 1) + 4LL * (long long)total;
    size_t off = 0;
    for (int i = 0; i < n; ++i) {
        const int c = std::max(h_rcount_[i], 0);
        filtered[size_t(i)].assign(h_rpacked_ + off, h_rpacked_ + off + c);
        off += size_t(c);
    }
}

}  // namespace cctagb
