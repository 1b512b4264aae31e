// Shared definitions of the B200 CCTag library (host and device).
#pragma once

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <string>

#include <cuda_runtime.h>

#include "cctag_b200.h"

namespace cctagb {

constexpr int kMaxLevels = 4;         // pyramid levels of one frame
constexpr int kMaxBatchFrames = 16;   // frames whose image stages share one launch per kernel
constexpr int kMaxLaunchLevels = kMaxLevels * kMaxBatchFrames;
constexpr int kScanBlocksPerLevel = 148;  // blocks of the voter-count scan (its partial sums per level)

// One pyramid level as the kernels see it.  All pointers are device memory.
struct LevelView {
    int W, H, WW;            // size; WW = 32-pixel words per bitmap row
    uint8_t* src;            // W*H gray
    int16_t* dx;             // W*H
    int16_t* dy;             // W*H
    uint8_t* map;            // W*H: 0 no edge, 1 weak candidate, 2 strong candidate
    uint32_t* hbits;         // 3 * WW*H: hysteresis planes C (candidates), R (tile-local strong closure), H (result)
    uint8_t* blab;           // uf_tiles * 128: border-position -> tile component (0xff none)
    int32_t* tcomp;          // uf_tiles * 64: union-find parents over (tile, component) ids
    int32_t* tflag;          // uf_tiles * 64: bit 0 holds a strong pixel, bit 1 (at roots) its set does
    uint32_t* bitmap;        // WW*H final thinned edges, bit x&31 of word x>>5
    uint2* bitidx;           // WW*H: (bitmap word, edge index of the word's first set bit)
    int32_t* row_count;      // H
    int32_t* row_off;        // H+1
    int cap;                 // edge-point capacity
    int32_t* exy;            // cap: x | y << 16
    int32_t* grad;           // cap: (uint16)dx | dy << 16
    int32_t* before;         // cap
    int32_t* after;          // cap
    int32_t* chosen;         // cap
    float* total;            // cap: field-line length of a successful vote
    int32_t* nvotes;         // cap: votes received
    int32_t* fill;           // cap: fill cursors of the voter lists
    int32_t* voff;           // cap+1: voter list offsets (CSR)
    int32_t* vlist;          // cap: voter lists, ascending voter index
    float* flow;             // cap: running-mean flow length (Vote.cpp:232)
    int seedcap;
    int32_t* seed_idx;       // seedcap
    int32_t* seed_key;       // seedcap: index of the voter that made it a seed
    int32_t* seed_votes;     // seedcap: votes the seed received
    int32_t* bigq;           // cap: points whose voter list needs a block sort
    // launch geometry of the tiled kernels
    int nms_tx, nms_tiles;   // 30x30 output tiles
    int thin_tx, thin_tiles; // thinning: 32-pixel word columns x 28-row strips
    int pix_blocks;          // 256-pixel blocks
    int uf_tx, uf_tiles;     // 32x32 hysteresis tiles
};

struct LevelCounters {
    int32_t E;       // edge points
    int32_t V;       // votes cast (= voters)
    int32_t S;       // seeds
    int32_t err;     // error bits (kErr*)
    int32_t bigq;    // long voter lists queued for the block sort
    int32_t pad[3];
};

constexpr int kErrEdgeOverflow = 1;
constexpr int kErrSeedOverflow = 2;
constexpr int kErrUnionFind = 4;

// The levels one launch of the image-stage kernels covers: the pyramid of one
// frame, or those of several frames back to back (frame f's level k is
// l[f * (n / frames) + k]).  Every kernel maps its blocks over all of them.
struct Levels {
    int n;
    int frames;              // frames in the launch; n / frames levels each
    LevelView l[kMaxLaunchLevels];
    LevelCounters* cnt;      // device, n entries
    int32_t* partial;        // device, n * kScanBlocksPerLevel: voter-count scan partial sums
};

struct VoteParamsDev {
    int distSearch;
    int thrGradient;
    float angleVoting;
    float ratioVoting;
    int nCrowns;
    int minVotes;
    int low, high;  // Canny thresholds after cvFloor
};

// Error type carried by host code; converted to cctagb_status at the ABI.
struct Error {
    cctagb_status status;
    std::string msg;
};

#define CCTAGB_CUDA(call)                                                                   \
    do {                                                                                    \
        cudaError_t e__ = (call);                                                           \
        if (e__ != cudaSuccess)                                                             \
            throw ::cctagb::Error{CCTAGB_CUDA_ERROR, std::string(#call) + ": " +             \
                                                         cudaGetErrorString(e__)};          \
    } while (0)

// A host thread's waits on its stream: a spin on an event for at most
// spin_us microseconds, then a blocking wait (the event is created with
// cudaEventBlockingSync), so that a thread whose frame waits on the GPU gives
// its core to the host stages of other frames.  spin_us < 0 spins throughout.
class HostWaiter {
public:
    HostWaiter() = default;
    ~HostWaiter()
    {
        if (ev_) cudaEventDestroy(ev_);
    }
    HostWaiter(const HostWaiter&) = delete;
    HostWaiter& operator=(const HostWaiter&) = delete;
    void init(int spin_us)
    {
        spin_us_ = spin_us;
        if (!ev_) CCTAGB_CUDA(cudaEventCreateWithFlags(&ev_, cudaEventBlockingSync | cudaEventDisableTiming));
    }
    void wait(cudaStream_t s) const
    {
        CCTAGB_CUDA(cudaEventRecord(ev_, s));
        const auto t0 = std::chrono::steady_clock::now();
        for (;;) {
            const cudaError_t q = cudaEventQuery(ev_);
            if (q == cudaSuccess) return;
            if (q != cudaErrorNotReady) CCTAGB_CUDA(q);
            if (spin_us_ >= 0 && std::chrono::steady_clock::now() - t0 >= std::chrono::microseconds(spin_us_)) break;
        }
        CCTAGB_CUDA(cudaEventSynchronize(ev_));
    }

private:
    cudaEvent_t ev_ = nullptr;
    int spin_us_ = -1;
};

// Optional per-stage timing: when `ev` is non-null the launcher records
// ev[k] after stage k (ev[0] before the first stage), kStageCount+1 events.
enum Stage {
    kStPyramid = 0, kStDerivNms, kStHystMerge, kStHystCompress, kStFinalThin, kStRowScan, kStEmit,
    kStWalk, kStVote, kStVoterScan, kStVoterFill, kStVoterSort, kStageCount
};
const char* stage_name(int k);

// Host launchers (image_stage.cu).
void upload_constants(const float* bank, int n_ids, int n_ratios);
void launch_image_stage(const Levels& lv, const VoteParamsDev& vp, cudaStream_t s, bool fused_pyramid,
                        cudaEvent_t* ev = nullptr);
void launch_canny_only(const Levels& lv, const VoteParamsDev& vp, cudaStream_t s);
void launch_gate(cudaStream_t s, int us);

// Device arrays of 32-bit words copied back to back into one buffer, so that
// a download is one copy instead of one per array (seeds and edge points of
// every level: 7 arrays per level).
constexpr int kMaxPackSegs = 7 * kMaxLevels;
struct PackSegs {
    const int32_t* src[kMaxPackSegs];
    long long off[kMaxPackSegs + 1];  // word offsets in dst; off[n] = total
    int n;
};
// Returns the number of kernels launched (0 when every segment is empty).
int launch_pack(const PackSegs& p, int32_t* dst, cudaStream_t s);
void launch_edge_level(const Levels& lv, const VoteParamsDev& vp, cudaStream_t s, uint8_t* edges_out,
                       int32_t* status_out);
// Copies counters src[0, n) of a batched launch to each level's own (dst[i]).
struct CounterTargets {
    LevelCounters* dst[kMaxLaunchLevels];
    int n;
};
void launch_scatter_counters(const LevelCounters* src, const CounterTargets& t, cudaStream_t s);

}  // namespace cctagb
