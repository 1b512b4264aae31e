// Host orchestration of one detection pipeline (one handle).
#pragma once

#include <mutex>
#include <memory>
#include <cstdint>
#include <string>
#include <vector>

#include "common.hpp"

namespace cctagb {

// Host copy of one level's edge-point collection, the interchange format of
// the reference (EdgePointCollection, Types.hpp:19-158): raster-ordered edge
// points with gradients, before/after links, CSR voter lists, vote-derived
// per-point state and the seeds in processing order.
// The arrays live in pinned host memory owned by the Pipeline and stay valid
// until the next download of the same level.
struct HostLevel {
    int W = 0, H = 0;
    int E = 0, V = 0;
    const int32_t* exy = nullptr;
    const int32_t* grad = nullptr;
    const int32_t* before = nullptr;
    const int32_t* after = nullptr;
    const int32_t* bidx = nullptr;   // WW * H (word, first index) pairs, or null
    int WW = 0;
    const int32_t* voff = nullptr;   // E + 1
    const int32_t* vlist = nullptr;  // V
    const float* flow = nullptr;
    std::vector<int32_t> seeds;  // processing order (Multiresolution.cpp:239-242)
};

// Orders the image stages of the detectors of one handle on the GPU: each
// stage waits for the one submitted before it, so that the full-GPU stages
// run one after the other in submission order.  The first frames of a batch
// then leave their image stage early and their latency-bound kernels and host
// phases overlap the later frames' stages, instead of every stage
// interleaving with the others and all finishing together.
struct StageOrder {
    StageOrder();
    ~StageOrder();
    StageOrder(const StageOrder&) = delete;
    StageOrder& operator=(const StageOrder&) = delete;
    std::mutex m;
    cudaEvent_t last = nullptr;  // end of the last submitted image stage
};

class Pipeline {
public:
    Pipeline(const cctagb_params& p, int max_w, int max_h, int max_batch);
    ~Pipeline();
    Pipeline(const Pipeline&) = delete;
    Pipeline& operator=(const Pipeline&) = delete;

    const cctagb_params& params() const { return params_; }
    cudaStream_t stream() const { return stream_; }
    // Shares the image-stage order of the other detectors of a handle.
    void set_stage_order(std::shared_ptr<StageOrder> o) { order_ = std::move(o); }

    // Pyramid .. seeds for one frame; results stay on the device.
    void image_stage(const uint8_t* gray, int w, int h, size_t pitch, bool is_device);
    // The batched form of image_stage (see BatchStage): the views of a w x h
    // frame and its upload on the batch stream s ...
    void prepare_batched(const uint8_t* gray, int w, int h, size_t pitch, bool is_device, cudaStream_t s);
    // ... and, once the batched launch has recorded `done`, this frame's
    // counters on the host (stage_ms and launches go to the statistics).
    void finish_batched(cudaEvent_t done, float stage_ms, int launches);
    // Waits for the work queued on s (this pipeline's streams).
    void host_wait(cudaStream_t s) const { waiter_.wait(s); }
    LevelCounters* device_counters() const { return d_cnt_; }
    const VoteParamsDev& vote_params() const { return vp_; }
    // Canny + thinning from caller derivatives (level 0 buffers).
    void canny_only(const int16_t* dx, const int16_t* dy, int w, int h, uint8_t* edges_out);

    int levels() const { return lv_.n; }
    // Device views of the levels of the last image_stage().
    const Levels& level_views() const { return lv_; }
    // Edge-point capacity of level l (fixed at construction).
    int level_capacity(int l) const { return la_[l].v.cap; }
    const uint8_t* level0_src() const { return lv_.l[0].src; }
    void level_size(int l, int* w, int* h) const;
    void copy_planes(int l, uint8_t* src, int16_t* dx, int16_t* dy, uint8_t* edges);
    const LevelCounters& counters(int l) const { return h_cnt_[l]; }
    // Downloads one level's edge-point collection (after image_stage).
    void download_level(int l, HostLevel& out);
    // Downloads every level with one synchronisation; without `voters` the
    // voter lists, their offsets and the flow lengths stay on the device
    // (out.voff / vlist / flow null: the GPU's loop one is their only reader
    // in a detection, and it hands the seeds' flow lengths over itself).
    void download_levels(std::vector<HostLevel>& out, bool voters = true);
    // The detection's form: the seeds (sorted, returned once they are on the
    // host) on the pipeline stream, and the edge points' positions,
    // gradients and links on a copy stream, so that they travel while the
    // GPU's loop one runs; wait_points() waits for them and sets
    // out.exy / grad / before / after.
    void download_seeds_then_points(std::vector<HostLevel>& out);
    void wait_points(std::vector<HostLevel>& out);
    float last_image_stage_ms() const { return last_ms_; }
    // Transfers and kernel launches since the last image_stage() began.
    long long h2d_bytes() const { return h2d_bytes_; }
    long long d2h_bytes() const { return d2h_bytes_; }
    int kernel_launches() const { return launches_; }
    void add_io(long long h2d, long long d2h, int launches)
    {
        h2d_bytes_ += h2d;
        d2h_bytes_ += d2h;
        launches_ += launches;
    }
    // Per-stage device times of the last frame (events captured into the graph).
    void set_stage_timing(bool on);
    const float* stage_ms() const { return stage_ms_; }

private:
    void alloc(int max_w, int max_h);
    void set_views(int w, int h, int nlevels);
    void sync_counters(cudaStream_t s);  // counters to the host; s synchronised

    cctagb_params params_;
    VoteParamsDev vp_{};
    int max_w_ = 0, max_h_ = 0;
    cudaStream_t stream_ = nullptr;
    cudaStream_t stage_stream_ = nullptr; // upload + image stage, lowest priority
    cudaStream_t copy_stream_ = nullptr;  // edge-point downloads of a detection
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    HostWaiter waiter_;                   // waits of the calling thread on stream_ / copy_stream_
    cudaEvent_t ev_in_ = nullptr;         // orders the stage stream after stream_
    std::shared_ptr<StageOrder> order_;
    std::vector<void*> allocs_;
    struct LevelAlloc {
        size_t px = 0;  // pixel capacity
        int cap = 0, seedcap = 0;
        LevelView v{};
        // pinned staging of the downloads
        int32_t* h_exy = nullptr;
        int32_t* h_grad = nullptr;
        int32_t* h_before = nullptr;
        int32_t* h_after = nullptr;
        int32_t* h_voff = nullptr;
        int32_t* h_vlist = nullptr;
        float* h_flow = nullptr;
        int32_t* h_sidx = nullptr;
        int32_t* h_skey = nullptr;
        int32_t* h_svotes = nullptr;
    } la_[kMaxLevels];
    std::vector<void*> host_allocs_;
    void issue_level_download(int l, bool voters);
    void finish_level_download(int l, HostLevel& out, bool voters);
    // Fills out from the counters and the downloaded seed arrays (sorted into
    // processing order); the point pointers are the per-level staging's.
    void finish_level(int l, HostLevel& out, bool voters, const int32_t* sidx, const int32_t* skey,
                      const int32_t* svotes);
    // compact staging of download_seeds_then_points and its per-level views
    int32_t* d_pack_ = nullptr;
    int32_t* h_pack_ = nullptr;  // pinned
    long long pack_words_ = 0;
    struct Packed {
        const int32_t *sidx, *skey, *svotes, *exy, *grad, *before, *after, *bidx;
    } pk_[kMaxLevels] = {};
    cudaEvent_t ev_pack_ = nullptr;  // the pack launch, for the copy stream
    Levels lv_{};
    LevelCounters* d_cnt_ = nullptr;  // + scan partials
    LevelCounters* h_cnt_ = nullptr;  // pinned
    cudaGraphExec_t graph_ = nullptr;
    int graph_w_ = -1, graph_h_ = -1;
    float last_ms_ = 0.f;
    long long h2d_bytes_ = 0, d2h_bytes_ = 0;
    int launches_ = 0;
    bool timing_ = false;
    cudaEvent_t st_ev_[kStageCount + 1] = {};
    float stage_ms_[kStageCount] = {};
};

// The image stages of several frames (each prepared in its own Pipeline's
// buffers) with one launch per kernel: the kernels map their blocks over the
// levels of all the frames, so a batch of 1080p frames fills the GPU where
// one frame's stage leaves it latency-bound.  The launches are captured into
// a CUDA graph, re-captured when the frames' pipelines or sizes change.
class BatchStage {
public:
    BatchStage();
    ~BatchStage();
    BatchStage(const BatchStage&) = delete;
    BatchStage& operator=(const BatchStage&) = delete;

    // Queues the stages of the prepared frames of `pipes` (at most
    // kMaxBatchFrames) on s; afterwards each pipeline's device counters hold
    // its frame's.  Record an event on s to hand the frames on.
    void run(const std::vector<Pipeline*>& pipes, cudaStream_t s);
    // Device time of the last run (waits for it) ...
    float finish_ms();
    // ... or, once the run is known complete, without waiting or writing.
    float elapsed_ms() const
    {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ev0_, ev1_) != cudaSuccess) cudaGetLastError();
        return ms;
    }
    int launches() const { return launches_; }
    // Per-stage timing of the batched launch (eager, events between kernels).
    void set_stage_timing(bool on);
    bool stage_timing() const { return timing_; }
    const float* stage_ms() const { return stage_ms_; }

private:
    struct Key {
        const Pipeline* p;
        int w, h;
        bool operator==(const Key& o) const { return p == o.p && w == o.w && h == o.h; }
        bool operator!=(const Key& o) const { return !(*this == o); }
    };
    Levels lv_{};
    LevelCounters* d_cnt_ = nullptr;
    int32_t* d_partial_ = nullptr;
    cudaGraphExec_t graph_ = nullptr;
    std::vector<Key> key_;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    cudaEvent_t st_ev_[kStageCount + 1] = {};
    bool timing_ = false;
    float stage_ms_[kStageCount] = {};
    float last_ms_ = 0.f;
    int launches_ = 0;
};

}  // namespace cctagb
