// Loop 1 and the outlier removal of loop 2 of the candidate stage on the GPU
// (see loop_one.hpp).  Built with --fmad=false: every floating-point
// expression here and in cand_shared.hpp is then evaluated with the same IEEE
// operations as the host restatement, so the candidates are the same bits.
//
// k_link_seeds   one thread per seed: the two edge-linking walks
//                (Vote.cpp:255-394), independent of the other seeds since
//                each walk only avoids its own points;
// k_link_resolve one warp per level: the seeds in processing order, skipping
//                those an earlier segment marked processed (Detection.cpp:
//                609-627), then the candidates ranked by averageReceivedVote;
// k_filter       one warp per loop-two candidate: children (Vote.cpp:
//                396-412) and the LMedS outlier removal (Vote.cpp:414-576),
//                32 random draws evaluated at once and accepted in draw order;
// k_pack         the kept candidates' filtered children, packed for download.
#include "loop_one.hpp"

#include <algorithm>
#include <cstring>

#include "cand_shared.hpp"

namespace cctagb {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kVisitSlots = 512;  // > 2 * kSegSlot

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
// Edge point at pixel (x, y), -1 if none (the index map is valid only where
// the edge bitmap is set).
__device__ __forceinline__ int at(const LoopOneLevel& L, int x, int y)
{
    const uint32_t w = L.bitmap[size_t(y) * L.WW + (x >> 5)];
    return ((w >> (x & 31)) & 1u) ? L.idxmap[size_t(y) * L.W + x] : -1;
}

// Points of one edge-linking call (the reference's set of visited positions).
struct VisitSet {
    int32_t k[kVisitSlots];
    __device__ void clear()
    {
        for (int i = 0; i < kVisitSlots; ++i) k[i] = -1;
    }
    __device__ static uint32_t slot(int v) { return (uint32_t(v) * 2654435761u) >> 23; }
    __device__ bool has(int v) const
    {
        for (uint32_t h = slot(v);; h = (h + 1) & (kVisitSlots - 1)) {
            if (k[h] == v) return true;
            if (k[h] == -1) return false;
        }
    }
    __device__ void add(int v)
    {
        for (uint32_t h = slot(v);; h = (h + 1) & (kVisitSlots - 1)) {
            if (k[h] == v) return;
            if (k[h] == -1) {
                k[h] = v;
                return;
            }
        }
    }
};

// Vote.cpp:272-394 edgeLinkingDir from the seed in direction dir.  The segment
// is held around segc[0] = seed: the +1 walk appends at segc[1..], the -1 walk
// prepends at segc[-1..].  Returns how many points, counted from the front of
// the segment as it is when the walk ends, become processed.
__device__ int link_walk(const LoopOneLevel& L, int seed, int dir, int32_t* segc, int& nf, int& nb, VisitSet& vis,
                         int window, float averageVoteMin)
{
    float ring[cand::kLinkMaxWindow + 1];
    int head = 0, count = 0;
    int i = 0;
    bool found = true;
    int stop = 0;
    int p = seed;
    float averageVote = float(voters(L, p));
    const int xoff[8] = {1, 1, 0, -1, -1, -1, 0, 1};
    const int yoff[8] = {0, -dir, -dir, -dir, 0, dir, dir, dir};
    while (i < cand::kLinkMaxLength && found && averageVote >= averageVoteMin) {
        const float angle = cand::link_angle(gdx(L, p), gdy(L, p));
        ring[(head + count) % (window + 1)] = angle;
        if (++count > window) {
            head = (head + 1) % (window + 1);
            --count;
        }
        const int shifting = cand::link_shift(angle);
        int j = 0;
        stop = 0;
        while (!stop) {
            if (j >= 8) {
                stop = cand::kEdgeNotFound;
            } else {
                const int k = dir == 1 ? (8 - shifting + j) % 8 : (shifting + j) % 8;
                const int sx = px_(L, p) + xoff[k];
                const int sy = py_(L, p) + yoff[k];
                if (sx >= 0 && sx < L.W && sy >= 0 && sy < L.H) {
                    const int q = at(L, sx, sy);
                    if (q >= 0 && !vis.has(q)) {
                        const float front = ring[head], back = ring[(head + count - 1) % (window + 1)];
                        if (cand::link_convexity_lost(front, back, count == window, dir)) stop = cand::kConvexityLost;
                        if (stop == 0) {
                            p = q;
                            if (dir > 0) segc[++nb] = p;
                            else segc[-(++nf)] = p;
                            averageVote = cand::link_average_vote(averageVote, 1 + nf + nb, voters(L, p));
                            stop = 1;
                        }
                        vis.add(p);
                    }
                }
            }
            ++j;
        }
        found = stop == 1;
        ++i;
    }
    const int size = 1 + nf + nb;
    if (i == cand::kLinkMaxLength || stop == cand::kConvexityLost) return size > window ? size - window : 0;
    if (stop == cand::kEdgeNotFound) return size;
    return 0;
}

__global__ void __launch_bounds__(128) k_link_seeds(LoopOneArgs a)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.totalSlots) return;
    const int l = t / a.maxSlotsPerLevel, s = t % a.maxSlotsPerLevel;
    if (l >= a.nl) return;
    const LoopOneLevel& L = a.lv[l];
    if (s >= L.nProc) return;
    const int seed = L.order[s];
    int32_t* segc = a.seg + size_t(t) * kSegSlot + kSegHalf;
    VisitSet vis;
    vis.clear();
    vis.add(seed);
    segc[0] = seed;
    int nf = 0, nb = 0;
    const int m1 = link_walk(L, seed, 1, segc, nf, nb, vis, a.window, a.averageVoteMin);
    const int m2 = link_walk(L, seed, -1, segc, nf, nb, vis, a.window, a.averageVoteMin);
    int nReceived = 0, nVoted = 0;
    for (int k = -nf; k <= nb; ++k) {
        const int v = voters(L, segc[k]);
        nReceived += v;
        if (v > 0) ++nVoted;
    }
    int32_t* info = a.sinfo + size_t(t) * 4;
    info[0] = nf;
    info[1] = nb;
    info[2] = m1;
    info[3] = m2;
    a.skey[t] = cand::received_vote_key(nReceived, nVoted);
}

__global__ void __launch_bounds__(32) k_link_resolve(LoopOneArgs a)
{
    const int l = blockIdx.x;
    const LoopOneLevel& L = a.lv[l];
    const int lane = threadIdx.x;
    int32_t* made = a.made + size_t(l) * a.maxSlotsPerLevel;
    int m = 0;
    for (int s = 0; s < L.nProc; ++s) {
        const int seed = L.order[s];
        int flag = lane == 0 ? L.processed[seed] : 0;
        flag = __shfl_sync(kFull, flag, 0);
        if (flag) continue;
        const int t = L.slot0 + s;
        if (lane == 0) {
            made[m] = s;
            L.processed[seed] = 1;
        }
        ++m;
        const int32_t* info = a.sinfo + size_t(t) * 4;
        const int nf = info[0], m1 = info[2], m2 = info[3];
        const int32_t* segc = a.seg + size_t(t) * kSegSlot + kSegHalf;
        for (int k = lane; k < m1; k += 32) L.processed[segc[k]] = 1;
        for (int k = lane; k < m2; k += 32) L.processed[segc[-nf + k]] = 1;
        __syncwarp();
    }
    __syncwarp();
    // Loop-1 order: averageReceivedVote descending, the newer candidate first
    // on equal keys (Detection.cpp:619-622).
    const int n2 = min(m, a.n2max);
    int32_t* meta = a.meta + size_t(l) * a.n2max * 4;
    for (int i = lane; i < m; i += 32) {
        const float ki = a.skey[L.slot0 + made[i]];
        int rank = 0;
        for (int j = 0; j < m; ++j) {
            const float kj = a.skey[L.slot0 + made[j]];
            rank += (kj > ki || (!(ki > kj) && j > i)) ? 1 : 0;
        }
        if (rank < n2) meta[rank * 4] = made[i];
    }
    if (lane == 0) a.meta[size_t(a.nl) * a.n2max * 4 + l] = m;
}

// Value of rank k (NaN last) of n order keys, reordering them.
__device__ uint32_t select_key(uint32_t* v, int n, int k)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const uint32_t pivot = v[(lo + hi) >> 1];
        int i = lo, j = hi;
        while (i <= j) {
            while (v[i] < pivot) ++i;
            while (v[j] > pivot) --j;
            if (i <= j) {
                const uint32_t t = v[i];
                v[i] = v[j];
                v[j] = t;
                ++i;
                --j;
            }
        }
        if (k <= j) hi = j;
        else if (k >= i) lo = i;
        else break;
    }
    return v[k];
}

__device__ __forceinline__ float key_value(uint32_t k)
{
    if (k == 0xffffffffu) return __int_as_float(0x7fffffff);
    const uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    return __uint_as_float(u);
}

__global__ void __launch_bounds__(32) k_filter(LoopOneArgs a)
{
    const int l = blockIdx.x / a.n2max, rank = blockIdx.x % a.n2max;
    const LoopOneLevel& L = a.lv[l];
    const int lane = threadIdx.x;
    const int madeCount = a.meta[size_t(a.nl) * a.n2max * 4 + l];
    if (rank >= min(madeCount, a.n2max)) return;
    int32_t* meta = a.meta + (size_t(l) * a.n2max + rank) * 4;
    const int s = meta[0];
    const int t = L.slot0 + s;
    const int32_t* info = a.sinfo + size_t(t) * 4;
    const int nf = info[0], nb = info[1];
    const int32_t* segc = a.seg + size_t(t) * kSegSlot + kSegHalf;
    const int len = nf + 1 + nb;
    int32_t* children = a.children + size_t(blockIdx.x) * kChildCap;
    __syncwarp();
    if (lane == 0) meta[0] = L.order[s];

    // children (Vote.cpp:396-412): voters of the points with >= voteMax/14 votes
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
        if (cnt && nchild + incl <= kChildCap) {
            const int32_t* src = L.vlist + L.voff[e];
            for (int k = 0; k < cnt; ++k) children[nchild + excl + k] = src[k];
        }
        nchild += __shfl_sync(kFull, incl, 31);
    }
    if (nchild > kChildCap) {
        if (lane == 0) {
            atomicOr(a.err, kLoopOneErrChildren);
            meta[1] = nchild;
            meta[2] = 0;
            meta[3] = 0;
        }
        return;
    }
    if (nchild < a.minPoints) {
        if (lane == 0) {
            meta[1] = 0;
            meta[2] = 0;
            meta[3] = 0;
        }
        return;
    }
    __syncwarp();

    // outlierRemoval (Vote.cpp:414-576) with maxSize 60 and inverse-gradient
    // weights: a regular subsample of the children ...
    __shared__ geo::Pt pts[kLmedsMaxPts];
    __shared__ float wts[kLmedsMaxPts];
    __shared__ int sPerm[32][5];
    __shared__ int sKind[32];
    __shared__ float sS[32];
    __shared__ float sQ[32][9];
    __shared__ float bestQ[9];
    __shared__ int sNpts, sDone;
    __shared__ float sSm;
    const int nSub = min(nchild, 60);
    if (lane == 0) {
        int np = 0;
        if (nSub >= 5) {
            const float step = float(nchild) / float(nSub);
            size_t k = 0;
            for (int i = 0; i < nchild; ++i) {
                if (size_t(i) == size_t(float(k) * step)) {
                    ++k;
                    const int e = children[i];
                    if (np < kLmedsMaxPts) {
                        pts[np] = {float(px_(L, e)), float(py_(L, e))};
                        wts[np] = 255.f / gnorm(L, e);
                    }
                    ++np;
                }
            }
            if (np > kLmedsMaxPts) atomicOr(a.err, kLoopOneErrPoints);
        }
        sNpts = np;
        for (int k = 0; k < 9; ++k) bestQ[k] = 0.f;
        sSm = 10000000.0f;
        sDone = 0;
    }
    __syncwarp();
    const int np = sNpts;
    if (nSub < 5 || np > kLmedsMaxPts) {
        if (lane == 0) {
            meta[1] = nchild;
            meta[2] = 0;
            meta[3] = 0;
        }
        return;
    }
    // ... then random 5-point conics, 32 draws at a time, accepted in order.
    geo::Pcg32 rng = cand::candidate_rng(L.level, uint64_t(rank), 0);
    int counter = 0, draws = 0;
    float Sm = 10000000.0f;
    uint32_t keys[kLmedsMaxPts];
    while (!sDone) {
        if (lane == 0)
            for (int j = 0; j < 32; ++j) rng.rand5(sPerm[j], size_t(np));
        __syncwarp();
        {
            geo::Mat3 Q;
            const int kind = cand::lmeds_conic(pts, sPerm[lane], Q);
            float S = 0.f;
            if (kind == 1) {
                for (int i = 0; i < np; ++i) {
                    const float d = geo::dist_point_ellipse(Q, pts[i].x, pts[i].y) * wts[i];
                    keys[i] = geo::order_key(d);
                }
                S = key_value(select_key(keys, np, np / 2));
            }
            sKind[lane] = kind;
            sS[lane] = S;
            for (int k = 0; k < 9; ++k) sQ[lane][k] = Q.m[k / 3][k % 3];
        }
        __syncwarp();
        if (lane == 0) {
            for (int j = 0; j < 32; ++j) {
                if (!(counter < 70 && draws < 7000)) break;
                ++draws;
                if (sKind[j] == 0) {
                    ++counter;
                } else if (sKind[j] == 1) {
                    if (sS[j] < Sm) {
                        counter = 0;
                        Sm = sS[j];
                        for (int k = 0; k < 9; ++k) bestQ[k] = sQ[j][k];
                    } else {
                        ++counter;
                    }
                }
            }
            if (!(counter < 70 && draws < 7000)) sDone = 1;
            sSm = Sm;
        }
        __syncwarp();
    }
    // the children whose weighted distance is below threshold * median
    geo::Mat3 Q;
    for (int k = 0; k < 9; ++k) Q.m[k / 3][k % 3] = bestQ[k];
    const float thr = a.threshold * sSm;
    int nflt = 0;
    for (int c0 = 0; c0 < nchild; c0 += 32) {
        const int i = c0 + lane;
        bool pass = false;
        int e = -1;
        if (i < nchild) {
            e = children[i];
            float d = geo::dist_point_ellipse(Q, float(px_(L, e)), float(py_(L, e)));
            d = d * 255 / gnorm(L, e);
            pass = d < thr;
        }
        const unsigned mask = __ballot_sync(kFull, pass);
        if (pass) children[nflt + __popc(mask & ((1u << lane) - 1u))] = e;
        nflt += __popc(mask);
        __syncwarp();
    }
    if (lane == 0) {
        meta[1] = nchild;
        meta[2] = nflt >= 5 ? 1 : 0;
        meta[3] = nflt;
    }
}

// Kept candidates' filtered children, in candidate order, into one array.
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
    const int32_t* src = a.children + size_t(b) * kChildCap;
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
    // seeds processed per level: max(rows / 2, maximumNbSeeds) (Detection.cpp:603-605);
    // level 0 has the most rows
    maxSlotsPerLevel_ = std::max(max_h / 2, p.maximumNbSeeds);
    totalSlots_ = nl_ * maxSlotsPerLevel_;
    for (int l = 0; l < nl_; ++l) {
        caps_.push_back(caps[size_t(l)]);
        processed_bytes_ += size_t(caps[size_t(l)]);
    }
    args_.seg = dev_alloc<int32_t>(allocs_, size_t(totalSlots_) * kSegSlot);
    args_.sinfo = dev_alloc<int32_t>(allocs_, size_t(totalSlots_) * 4);
    args_.skey = dev_alloc<float>(allocs_, size_t(totalSlots_));
    args_.made = dev_alloc<int32_t>(allocs_, size_t(totalSlots_));
    const size_t metaN = size_t(nl_) * n2max_ * 4 + nl_ + 1;
    args_.meta = dev_alloc<int32_t>(allocs_, metaN);
    args_.err = args_.meta + size_t(nl_) * n2max_ * 4 + nl_;
    args_.children = dev_alloc<int32_t>(allocs_, size_t(nl_) * n2max_ * kChildCap);
    d_order_ = dev_alloc<int32_t>(allocs_, size_t(totalSlots_));
    d_processed_ = dev_alloc<uint8_t>(allocs_, processed_bytes_);
    d_packed_ = dev_alloc<int32_t>(allocs_, size_t(nl_) * n2max_ * kChildCap);
    CCTAGB_CUDA(cudaMallocHost(&h_order_, sizeof(int32_t) * std::max(totalSlots_, 1)));
    CCTAGB_CUDA(cudaMallocHost(&h_meta_, sizeof(int32_t) * metaN));
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
}

LoopOneGpu::~LoopOneGpu()
{
    for (void* q : allocs_) cudaFree(q);
    if (h_order_) cudaFreeHost(h_order_);
    if (h_meta_) cudaFreeHost(h_meta_);
    if (h_flt_) cudaFreeHost(h_flt_);
}

void LoopOneGpu::launch(const Levels& lv, const int* E, const std::vector<const std::vector<int32_t>*>& seeds,
                        cudaStream_t s)
{
    if (lv.n != nl_ || int(seeds.size()) != nl_) throw Error{CCTAGB_BAD_ARG, "loop one: level count changed"};
    h2d_ = d2h_ = 0;
    size_t poff = 0;
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
        L.bitmap = v.bitmap;
        L.idxmap = v.idxmap;
        L.level = l;
        L.slot0 = l * maxSlotsPerLevel_;
        const size_t nMax = size_t(std::max(v.H / 2, p_.maximumNbSeeds));
        L.nProc = int(std::min(seeds[l]->size(), nMax));
        L.order = d_order_ + L.slot0;
        std::copy(seeds[l]->begin(), seeds[l]->begin() + L.nProc, h_order_ + L.slot0);
        if (v.cap > caps_[size_t(l)]) throw Error{CCTAGB_INTERNAL, "loop one: level capacity changed"};
        L.processed = d_processed_ + poff;
        poff += size_t(caps_[size_t(l)]);
        if (L.nProc)
            CCTAGB_CUDA(cudaMemcpyAsync(d_order_ + L.slot0, h_order_ + L.slot0, sizeof(int32_t) * L.nProc,
                                        cudaMemcpyHostToDevice, s));
        h2d_ += 4LL * L.nProc;
    }
    CCTAGB_CUDA(cudaMemsetAsync(d_processed_, 0, processed_bytes_, s));
    const size_t metaN = size_t(nl_) * n2max_ * 4 + nl_ + 1;
    CCTAGB_CUDA(cudaMemsetAsync(args_.meta, 0, sizeof(int32_t) * metaN, s));
    k_link_seeds<<<(totalSlots_ + 127) / 128, 128, 0, s>>>(args_);
    CCTAGB_CUDA(cudaGetLastError());
    k_link_resolve<<<nl_, 32, 0, s>>>(args_);
    CCTAGB_CUDA(cudaGetLastError());
    k_filter<<<nl_ * n2max_, 32, 0, s>>>(args_);
    CCTAGB_CUDA(cudaGetLastError());
    k_pack<<<nl_ * n2max_, 256, 0, s>>>(args_, d_packed_);
    CCTAGB_CUDA(cudaGetLastError());
    CCTAGB_CUDA(cudaMemcpyAsync(h_meta_, args_.meta, sizeof(int32_t) * metaN, cudaMemcpyDeviceToHost, s));
    d2h_ += 4LL * metaN;
}

void LoopOneGpu::collect(cudaStream_t s, std::vector<LoopTwoIn>& out)
{
    CCTAGB_CUDA(cudaStreamSynchronize(s));
    const int32_t* made = h_meta_ + size_t(nl_) * n2max_ * 4;
    const int err = made[nl_];
    if (err & kLoopOneErrChildren)
        throw Error{CCTAGB_OVERFLOW_VOTERS, "a loop-two candidate gathers more than 32768 voters"};
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
    if (total) {
        CCTAGB_CUDA(cudaMemcpyAsync(h_flt_, d_packed_, sizeof(int32_t) * total, cudaMemcpyDeviceToHost, s));
        CCTAGB_CUDA(cudaStreamSynchronize(s));
    }
    d2h_ += 4LL * total;
    out.assign(size_t(nl_), {});
    size_t off = 0;
    for (int l = 0; l < nl_; ++l) {
        LoopTwoIn& o = out[size_t(l)];
        const int n2 = std::min(made[l], n2max_);
        o.foff.push_back(0);
        for (int r = 0; r < n2; ++r) {
            const int32_t* m = h_meta_ + (size_t(l) * n2max_ + r) * 4;
            o.seed.push_back(m[0]);
            o.score.push_back(m[1]);
            o.keep.push_back(uint8_t(m[2]));
            if (m[2]) {
                o.flt.insert(o.flt.end(), h_flt_ + off, h_flt_ + off + m[3]);
                off += size_t(m[3]);
            }
            o.foff.push_back(int32_t(o.flt.size()));
        }
    }
}

}  // namespace cctagb
