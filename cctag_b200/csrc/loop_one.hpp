// Loop 1 of the candidate stage (edge linking from the seeds,
// Detection.cpp:69-113, 609-627, Vote.cpp:255-394) and the first half of
// loop 2 (children collection and LMedS outlier removal, Detection.cpp:
// 115-156, Vote.cpp:396-576) on the GPU, with the same results as the host
// restatement in candidates.cpp (shared arithmetic in cand_shared.hpp).
#pragma once

#include <cstdint>
#include <vector>

#include "candidates.hpp"
#include "common.hpp"

namespace cctagb {

constexpr int kSegHalf = 100;                 // points per linking direction (maxLength)
constexpr int kSegSlot = 2 * kSegHalf + 1;    // one segment: front, seed, back
constexpr int kChildCap = 32768;              // initial room for the children of one loop-two candidate
constexpr int kLmedsMaxPts = 64;              // subsampled points of one outlier removal
constexpr int kMarkCap = 2 * kSegSlot;        // later seeds one segment can mark processed
constexpr int kFilterThreads = 128;           // LMedS draws evaluated at once per candidate
constexpr int kRawPool = 1024;                // random outputs generated per batch of draws

// One level as the loop-one kernels see it (device pointers).
struct LoopOneLevel {
    int W, H, WW, E;
    const int32_t* exy;
    const int32_t* grad;
    const int32_t* voff;
    const int32_t* vlist;
    const uint2* bitidx;     // WW*H: (edge bitmap word, edge index of its first set bit)
    const int32_t* before;  // E: the walks' links
    const int32_t* after;
    const int32_t* order;   // seeds in processing order, nProc of them
    int nProc, slot0;       // seed slots [slot0, slot0 + nProc)
    int4* rec;              // E point records (3 int4 each): xy, angle, voters, seed slot; 8 neighbours
    const float* flow;      // E flow lengths (Vote.cpp:232)
    int level;
};

struct LoopOneArgs {
    int nl;
    LoopOneLevel lv[kMaxLevels];
    int window;             // windowSizeOnInnerEllipticSegment
    float averageVoteMin;
    int n2max;              // maximumNbCandidatesLoopTwo
    int minPoints;          // minPointsSegmentCandidate
    float threshold;        // threshRobustEstimationOfOuterEllipse
    int totalSlots;
    int32_t* seg;           // totalSlots * kSegSlot: segment of each seed slot, seed at kSegHalf
    int32_t* sinfo;         // totalSlots * 4: front length, back length, number of marked later seeds
    int32_t* mlist;         // totalSlots * kMarkCap: later seed slots the segment marks processed
    float* skey;            // totalSlots: averageReceivedVote
    int32_t* made;          // nl * maxSlotsPerLevel: made candidates (seed slots), per level
    int maxSlotsPerLevel;
    int32_t* meta;          // nl * n2max * 4: seed slot, score, keep, filtered count; then nl: made count
    float* cflow;           // nl * n2max: flow length of each loop-two candidate's seed
    int32_t* children;      // nl * n2max * childCap: children, then filtered in place
    int childCap;           // room per candidate (grown and re-run on overflow)
    int32_t* err;           // error bits
};

constexpr int kLoopOneErrChildren = 1;
constexpr int kLoopOneErrWindow = 2;
constexpr int kLoopOneErrPoints = 4;
constexpr int kLoopOneErrRandom = 8;

// One coarse-level marker to re-fit on level 0 (Multiresolution.cpp:319-401):
// the hull's inner and outer conics, the inner center, the center row, and
// the marker's index in the frame (its random stream).
struct RefitTask {
    float qin[9], qout[9];
    float inCx, inCy, yc;
    int marker;
};

void launch_loop_one(const LoopOneArgs& a, cudaStream_t s);

// Device buffers of loop 1 / loop 2 (first half) for one detection slot.
class LoopOneGpu {
public:
    // max_h: largest frame height; caps: edge-point capacity of each level.
    LoopOneGpu(const cctagb_params& p, int max_h, const std::vector<int>& caps);
    ~LoopOneGpu();
    LoopOneGpu(const LoopOneGpu&) = delete;
    LoopOneGpu& operator=(const LoopOneGpu&) = delete;

    // Uploads the seeds (processing order), launches the kernels on `s` and
    // queues the download of the per-candidate counts.  `E` = edge points per
    // level.  Returns immediately.
    void launch(const Levels& lv, const int* E, const std::vector<const std::vector<int32_t>*>& seeds,
                cudaStream_t s);
    // Waits for launch()'s work and fills `out` (one LoopTwoIn per level).
    void collect(cudaStream_t s, std::vector<LoopTwoIn>& out);
    // Level-0 hull collection and outlier removal of the re-fit of `tasks`
    // on level 0 of `lv` (synchronous): per task, the filtered hull points
    // (fewer than 5 when the marker keeps its coarse-level ellipse).
    void refit(const Levels& lv, const std::vector<RefitTask>& tasks, cudaStream_t s,
               std::vector<std::vector<int32_t>>& filtered);
    int launches() const { return 6 + chainLaunches_; }
    int refit_launches() const { return 2; }
    long long h2d_bytes() const { return h2d_; }
    long long d2h_bytes() const { return d2h_; }

private:
    int resolve_smem() const;
    void run_kernels(cudaStream_t s);    // the loop-one kernels and the count download
    void grow_children(size_t cap);     // children / packed buffers for `cap` per candidate
    void ensure_refit_capacity(int n);
    cctagb_params p_;
    HostWaiter waiter_;            // waits of the calling thread on its stream
    int nl_ = 0, n2max_ = 0, maxSlotsPerLevel_ = 0, totalSlots_ = 0;
    LoopOneArgs args_{};
    int4 cum_{};                   // cumulative edge points of the levels (last launch)
    int32_t* d_order_ = nullptr;   // all levels' seed slots
    int32_t* h_order_ = nullptr;   // pinned staging
    int4* d_rec_ = nullptr;        // point records of all levels
    int32_t* d_packed_ = nullptr;  // kept candidates' filtered children
    std::vector<int> caps_;
    int maxH_ = 0;
    size_t maxCap_ = 0;             // largest level capacity: no list can exceed it
    int refitCap_ = 0;
    RefitTask* d_rtask_ = nullptr;
    RefitTask* h_rtask_ = nullptr;
    int hullCap_ = kChildCap;       // room for one marker's hull points
    int32_t* d_rhull_ = nullptr;    // refitCap_ * hullCap_
    int32_t* d_rrows_ = nullptr;    // refitCap_ * (maxH_ + 2) per-row offsets
    int32_t* d_rcount_ = nullptr;   // refitCap_ + 1 (last: error bits)
    int32_t* h_rcount_ = nullptr;
    int32_t* d_rpacked_ = nullptr;  // refitCap_ * hullCap_
    int32_t* h_rpacked_ = nullptr;
    size_t h_rpacked_cap_ = 0;
    int32_t* h_meta_ = nullptr;    // pinned: meta + made counts + err
    float* h_cflow_ = nullptr;     // pinned: seeds' flow lengths
    int32_t* h_flt_ = nullptr;     // pinned: filtered children, all candidates
    size_t h_flt_cap_ = 0;
    int32_t* d_chain_ = nullptr;   // link chains of the filtered children (k_chains)
    int32_t* h_chain_ = nullptr;   // pinned
    size_t chain_cap_ = 0;
    int chainLaunches_ = 0;        // k_chains launches of the last collect
    std::vector<void*> allocs_;
    long long h2d_ = 0, d2h_ = 0;
};

}  // namespace cctagb
