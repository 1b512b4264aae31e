// Host orchestration: device arena, per-resolution CUDA graph of the image
// stage, downloads of the per-level edge-point collections.
#include "pipeline.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace cctagb {

namespace {

template <class T>
T* dev_alloc(std::vector<void*>& list, size_t n)
{
    void* p = nullptr;
    CCTAGB_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
    list.push_back(p);
    return static_cast<T*>(p);
}

}  // namespace

Pipeline::Pipeline(const cctagb_params& p, int max_w, int max_h, int max_batch) : params_(p)
{
    (void)max_batch;
    int dev = 0;
    CCTAGB_CUDA(cudaGetDevice(&dev));
    cudaDeviceProp prop{};
    CCTAGB_CUDA(cudaGetDeviceProperties(&prop, dev));
    if (prop.major < 10) throw Error{CCTAGB_NO_DEVICE, "device is not sm_100 (compute capability " +
                                                           std::to_string(prop.major) + "." +
                                                           std::to_string(prop.minor) + ")"};
    if (p.numberOfProcessedMultiresLayers < 1 || p.numberOfProcessedMultiresLayers > kMaxLevels)
        throw Error{CCTAGB_BAD_ARG, "numberOfProcessedMultiresLayers must be in [1, 4]"};
    if (p.nCrowns < 1 || 2 * p.nCrowns - 1 > 16) throw Error{CCTAGB_BAD_ARG, "nCrowns out of range"};
    if (p.edgeCapacityDivisor < 1) throw Error{CCTAGB_BAD_ARG, "edgeCapacityDivisor must be >= 1"};
    // a walk that does not move (zero gradient) runs distSearch steps
    if (p.distSearch < 0 || p.distSearch > 16384) throw Error{CCTAGB_BAD_ARG, "distSearch must be in [0, 16384]"};
    vp_.distSearch = p.distSearch;
    vp_.thrGradient = p.thrGradientMagInVote;
    vp_.angleVoting = p.angleVoting;
    vp_.ratioVoting = p.ratioVoting;
    vp_.nCrowns = p.nCrowns;
    vp_.minVotes = p.minVotesToSelectCandidate;
    float lo = p.cannyThrLow * 256.f, hi = p.cannyThrHigh * 256.f;
    if (lo > hi) std::swap(lo, hi);
    vp_.low = int(std::floor(lo));
    vp_.high = int(std::floor(hi));
    // The image stage (full-GPU, bandwidth-bound grids) runs at the lowest
    // stream priority and the later latency-bound kernels of a detection at
    // the highest, so that with several detections in flight a frame past its
    // image stage gets SMs ahead of the next frame's image stage.
    int least = 0, greatest = 0;
    CCTAGB_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    CCTAGB_CUDA(cudaStreamCreateWithPriority(&stream_, cudaStreamNonBlocking, greatest));
    CCTAGB_CUDA(cudaStreamCreateWithPriority(&stage_stream_, cudaStreamNonBlocking, least));
    CCTAGB_CUDA(cudaStreamCreateWithPriority(&copy_stream_, cudaStreamNonBlocking, greatest));
    CCTAGB_CUDA(cudaEventCreate(&ev0_));
    CCTAGB_CUDA(cudaEventCreate(&ev1_));
    CCTAGB_CUDA(cudaEventCreateWithFlags(&ev_in_, cudaEventDisableTiming));
    CCTAGB_CUDA(cudaEventCreateWithFlags(&ev_pack_, cudaEventDisableTiming));
    upload_constants(nullptr, 0, 0);
    waiter_.init(p.hostSpinMicros);
    alloc(max_w, max_h);
}

Pipeline::~Pipeline()
{
    if (graph_) cudaGraphExecDestroy(graph_);
    for (cudaEvent_t e : st_ev_)
        if (e) cudaEventDestroy(e);
    for (void* p : allocs_) cudaFree(p);
    for (void* p : host_allocs_) cudaFreeHost(p);
    if (h_cnt_) cudaFreeHost(h_cnt_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (ev_in_) cudaEventDestroy(ev_in_);
    if (ev_pack_) cudaEventDestroy(ev_pack_);
    if (stream_) cudaStreamDestroy(stream_);
    if (stage_stream_) cudaStreamDestroy(stage_stream_);
    if (copy_stream_) cudaStreamDestroy(copy_stream_);
}

StageOrder::StageOrder() { CCTAGB_CUDA(cudaEventCreateWithFlags(&last, cudaEventDisableTiming)); }

StageOrder::~StageOrder()
{
    if (last) cudaEventDestroy(last);
}

void Pipeline::alloc(int max_w, int max_h)
{
    if (max_w < 1 || max_h < 1 || max_w > 16384 || max_h > 16384)
        throw Error{CCTAGB_BAD_ARG, "max frame size must be in [1, 16384]"};
    max_w_ = max_w;
    max_h_ = max_h;
    int w = max_w, h = max_h;
    const int nl = params_.numberOfProcessedMultiresLayers;
    for (int l = 0; l < nl; ++l) {
        LevelAlloc& a = la_[l];
        // Level buffers are sized for the largest frame; +8 rows/cols of slack
        // lets a smaller frame use its own width as the row stride.
        const size_t px = size_t(w) * h;
        a.px = px;
        a.cap = int(std::max<size_t>(px / params_.edgeCapacityDivisor, 1024));
        a.seedcap = a.cap;
        LevelView& v = a.v;
        v.src = dev_alloc<uint8_t>(allocs_, px + 16);
        v.dx = dev_alloc<int16_t>(allocs_, px);
        v.dy = dev_alloc<int16_t>(allocs_, px);
        v.map = dev_alloc<uint8_t>(allocs_, px);
        const size_t tiles = size_t((w + 31) / 32) * size_t((h + 31) / 32);
        v.hbits = dev_alloc<uint32_t>(allocs_, 3 * size_t((w + 31) / 32) * h);
        v.blab = dev_alloc<uint8_t>(allocs_, tiles * 128);
        v.tcomp = dev_alloc<int32_t>(allocs_, tiles * 64);
        v.tflag = dev_alloc<int32_t>(allocs_, tiles * 64);
        v.bitmap = dev_alloc<uint32_t>(allocs_, size_t((w + 31) / 32) * h);
        v.bitidx = dev_alloc<uint2>(allocs_, size_t((w + 31) / 32) * h);
        v.row_count = dev_alloc<int32_t>(allocs_, h);
        v.row_off = dev_alloc<int32_t>(allocs_, h + 1);
        CCTAGB_CUDA(cudaMemset(v.row_count, 0, sizeof(int32_t) * h));
        v.cap = a.cap;
        v.exy = dev_alloc<int32_t>(allocs_, a.cap);
        v.grad = dev_alloc<int32_t>(allocs_, a.cap);
        v.before = dev_alloc<int32_t>(allocs_, a.cap);
        v.after = dev_alloc<int32_t>(allocs_, a.cap);
        v.chosen = dev_alloc<int32_t>(allocs_, a.cap);
        v.total = dev_alloc<float>(allocs_, a.cap);
        v.nvotes = dev_alloc<int32_t>(allocs_, a.cap);
        v.fill = dev_alloc<int32_t>(allocs_, a.cap);
        v.voff = dev_alloc<int32_t>(allocs_, a.cap + 1);
        v.vlist = dev_alloc<int32_t>(allocs_, a.cap);
        v.flow = dev_alloc<float>(allocs_, a.cap);
        v.seedcap = a.seedcap;
        v.seed_idx = dev_alloc<int32_t>(allocs_, a.seedcap);
        v.seed_key = dev_alloc<int32_t>(allocs_, a.seedcap);
        v.seed_votes = dev_alloc<int32_t>(allocs_, a.seedcap);
        v.bigq = dev_alloc<int32_t>(allocs_, a.cap);
        auto pinned = [&](size_t n) {
            void* q = nullptr;
            CCTAGB_CUDA(cudaMallocHost(&q, std::max<size_t>(n, 1) * 4));
            host_allocs_.push_back(q);
            return q;
        };
        a.h_exy = static_cast<int32_t*>(pinned(a.cap));
        a.h_grad = static_cast<int32_t*>(pinned(a.cap));
        a.h_before = static_cast<int32_t*>(pinned(a.cap));
        a.h_after = static_cast<int32_t*>(pinned(a.cap));
        a.h_voff = static_cast<int32_t*>(pinned(size_t(a.cap) + 1));
        a.h_vlist = static_cast<int32_t*>(pinned(a.cap));
        a.h_flow = static_cast<float*>(pinned(a.cap));
        a.h_sidx = static_cast<int32_t*>(pinned(a.seedcap));
        a.h_skey = static_cast<int32_t*>(pinned(a.seedcap));
        a.h_svotes = static_cast<int32_t*>(pinned(a.seedcap));
        w /= 2;
        h /= 2;
        if (w < 1 || h < 1) throw Error{CCTAGB_BAD_ARG, "frame too small for the number of pyramid levels"};
    }
    // Compact download staging: seeds, edge points and word index planes of
    // every level.
    pack_words_ = 0;
    for (int l = 0, lw = max_w, lh = max_h; l < nl; ++l, lw /= 2, lh /= 2)
        pack_words_ += 3LL * la_[l].seedcap + 2LL * la_[l].cap + 2LL * ((lw + 31) / 32) * lh;
    d_pack_ = dev_alloc<int32_t>(allocs_, size_t(pack_words_));
    CCTAGB_CUDA(cudaMallocHost(&h_pack_, size_t(pack_words_) * 4));
    host_allocs_.push_back(h_pack_);
    // Counters followed by the partial sums of the voter-count scan.
    const size_t cnt_bytes = sizeof(LevelCounters) * kMaxLevels + sizeof(int32_t) * kMaxLevels * kScanBlocksPerLevel;
    d_cnt_ = reinterpret_cast<LevelCounters*>(dev_alloc<uint8_t>(allocs_, cnt_bytes));
    CCTAGB_CUDA(cudaMemset(d_cnt_, 0, cnt_bytes));
    CCTAGB_CUDA(cudaMallocHost(&h_cnt_, sizeof(LevelCounters) * kMaxLevels));
    std::memset(h_cnt_, 0, sizeof(LevelCounters) * kMaxLevels);
}

void Pipeline::set_views(int w, int h, int nl)
{
    if (w > max_w_ || h > max_h_) throw Error{CCTAGB_TOO_LARGE, "frame larger than the handle's maximum"};
    lv_.n = nl;
    lv_.frames = 1;
    lv_.cnt = d_cnt_;
    lv_.partial = reinterpret_cast<int32_t*>(d_cnt_ + kMaxLevels);
    for (int l = 0; l < nl; ++l) {
        if (w < 1 || h < 1) throw Error{CCTAGB_BAD_ARG, "frame too small for the number of pyramid levels"};
        LevelView v = la_[l].v;
        v.W = w;
        v.H = h;
        v.WW = (w + 31) / 32;
        v.nms_tx = (w + 29) / 30;
        v.nms_tiles = v.nms_tx * ((h + 29) / 30);
        v.thin_tx = (w + 31) / 32;
        v.thin_tiles = v.thin_tx * ((h + 27) / 28);  // word columns x 28-row strips
        v.pix_blocks = int((size_t(w) * h + 255) / 256);
        v.uf_tx = (w + 31) / 32;
        v.uf_tiles = v.uf_tx * ((h + 31) / 32);
        lv_.l[l] = v;
        w /= 2;
        h /= 2;
    }
}

void Pipeline::image_stage(const uint8_t* gray, int w, int h, size_t pitch, bool is_device)
{
    if (!gray || w < 1 || h < 1 || pitch < size_t(w)) throw Error{CCTAGB_BAD_ARG, "bad frame arguments"};
    set_views(w, h, params_.numberOfProcessedMultiresLayers);
    // the stage stream starts after all earlier work of the pipeline stream
    cudaStream_t st = stage_stream_;
    CCTAGB_CUDA(cudaEventRecord(ev_in_, stream_));
    CCTAGB_CUDA(cudaStreamWaitEvent(st, ev_in_, 0));
    CCTAGB_CUDA(cudaMemcpy2DAsync(lv_.l[0].src, w, gray, pitch, w, h,
                                  is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    const bool fused = (w % 8 == 0) && (h % 8 == 0) && lv_.n == 4;
    h2d_bytes_ = is_device ? 0 : (long long)w * h;
    d2h_bytes_ = 0;
    // kernels of one image stage: pyramid (1 fused or one per level), 15 others
    launches_ = (fused ? 1 : lv_.n - 1) + 15;
    if (timing_) {
        // Per-stage timing: eager launches queued behind a ~2 ms gate so the
        // GPU never waits for the host between two stage events.
        launch_gate(st, 2000);
        CCTAGB_CUDA(cudaEventRecord(ev0_, st));
        launch_image_stage(lv_, vp_, st, fused, st_ev_);
        CCTAGB_CUDA(cudaEventRecord(ev1_, st));
        sync_counters(st);
        CCTAGB_CUDA(cudaEventElapsedTime(&last_ms_, ev0_, ev1_));
        for (int k = 0; k < kStageCount; ++k) CCTAGB_CUDA(cudaEventElapsedTime(&stage_ms_[k], st_ev_[k], st_ev_[k + 1]));
        return;
    }
    if (!graph_ || graph_w_ != w || graph_h_ != h) {
        if (graph_) {
            cudaGraphExecDestroy(graph_);
            graph_ = nullptr;
        }
        cudaGraph_t g = nullptr;
        CCTAGB_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        try {
            launch_image_stage(lv_, vp_, st, fused, nullptr);
        } catch (...) {
            cudaStreamEndCapture(st, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        CCTAGB_CUDA(cudaStreamEndCapture(st, &g));
        const cudaError_t e = cudaGraphInstantiate(&graph_, g, 0);
        cudaGraphDestroy(g);
        CCTAGB_CUDA(e);
        graph_w_ = w;
        graph_h_ = h;
    }
    if (order_) {
        std::lock_guard<std::mutex> lock(order_->m);
        CCTAGB_CUDA(cudaStreamWaitEvent(st, order_->last, 0));
        CCTAGB_CUDA(cudaEventRecord(ev0_, st));
        CCTAGB_CUDA(cudaGraphLaunch(graph_, st));
        CCTAGB_CUDA(cudaEventRecord(ev1_, st));
        CCTAGB_CUDA(cudaEventRecord(order_->last, st));
    } else {
        CCTAGB_CUDA(cudaEventRecord(ev0_, st));
        CCTAGB_CUDA(cudaGraphLaunch(graph_, st));
        CCTAGB_CUDA(cudaEventRecord(ev1_, st));
    }
    sync_counters(st);
    CCTAGB_CUDA(cudaEventElapsedTime(&last_ms_, ev0_, ev1_));
}

void Pipeline::prepare_batched(const uint8_t* gray, int w, int h, size_t pitch, bool is_device, cudaStream_t s)
{
    if (!gray || w < 1 || h < 1 || pitch < size_t(w)) throw Error{CCTAGB_BAD_ARG, "bad frame arguments"};
    set_views(w, h, params_.numberOfProcessedMultiresLayers);
    // the batch stream starts after all earlier work of this pipeline
    CCTAGB_CUDA(cudaEventRecord(ev_in_, stream_));
    CCTAGB_CUDA(cudaStreamWaitEvent(s, ev_in_, 0));
    CCTAGB_CUDA(cudaMemcpy2DAsync(lv_.l[0].src, w, gray, pitch, w, h,
                                  is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    h2d_bytes_ = is_device ? 0 : (long long)w * h;
    d2h_bytes_ = 0;
    launches_ = 0;
}

void Pipeline::finish_batched(cudaEvent_t done, float stage_ms, int launches)
{
    CCTAGB_CUDA(cudaStreamWaitEvent(stream_, done, 0));
    sync_counters(stream_);
    last_ms_ = stage_ms;
    launches_ = launches;
}

// ---------------------------------------------------------------- batches --
BatchStage::BatchStage()
{
    CCTAGB_CUDA(cudaMalloc(&d_cnt_, sizeof(LevelCounters) * kMaxLaunchLevels));
    CCTAGB_CUDA(cudaMalloc(&d_partial_, sizeof(int32_t) * kMaxLaunchLevels * kScanBlocksPerLevel));
    CCTAGB_CUDA(cudaEventCreate(&ev0_));
    CCTAGB_CUDA(cudaEventCreate(&ev1_));
}

BatchStage::~BatchStage()
{
    if (graph_) cudaGraphExecDestroy(graph_);
    for (cudaEvent_t e : st_ev_)
        if (e) cudaEventDestroy(e);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (d_cnt_) cudaFree(d_cnt_);
    if (d_partial_) cudaFree(d_partial_);
}

void BatchStage::set_stage_timing(bool on)
{
    if (on && !st_ev_[0])
        for (cudaEvent_t& e : st_ev_) CCTAGB_CUDA(cudaEventCreate(&e));
    timing_ = on;
    std::fill(stage_ms_, stage_ms_ + kStageCount, 0.f);
}

void BatchStage::run(const std::vector<Pipeline*>& pipes, cudaStream_t s)
{
    const int nf = int(pipes.size());
    if (nf < 1 || nf > kMaxBatchFrames) throw Error{CCTAGB_INTERNAL, "batched image stage: bad frame count"};
    lv_.n = 0;
    lv_.frames = nf;
    lv_.cnt = d_cnt_;
    lv_.partial = d_partial_;
    CounterTargets tg{};
    bool fused = true;
    std::vector<Key> key;
    for (Pipeline* p : pipes) {
        const Levels& v = p->level_views();
        if (v.n != pipes[0]->level_views().n) throw Error{CCTAGB_INTERNAL, "batched frames differ in level count"};
        fused = fused && v.n == 4 && v.l[0].W % 8 == 0 && v.l[0].H % 8 == 0;
        for (int l = 0; l < v.n; ++l) {
            tg.dst[lv_.n] = p->device_counters() + l;
            lv_.l[lv_.n++] = v.l[l];
        }
        key.push_back({p, v.l[0].W, v.l[0].H});
    }
    tg.n = lv_.n;
    const VoteParamsDev& vp = pipes[0]->vote_params();
    // kernels: pyramid (1 fused or one per level), 15 image-stage kernels, the counter scatter
    launches_ = (fused ? 1 : lv_.n - nf) + 15 + 1;
    if (timing_) {
        launch_gate(s, 2000);
        CCTAGB_CUDA(cudaEventRecord(ev0_, s));
        launch_image_stage(lv_, vp, s, fused, st_ev_);
        launch_scatter_counters(d_cnt_, tg, s);
        CCTAGB_CUDA(cudaEventRecord(ev1_, s));
        CCTAGB_CUDA(cudaEventSynchronize(ev1_));
        CCTAGB_CUDA(cudaEventElapsedTime(&last_ms_, ev0_, ev1_));
        for (int k = 0; k < kStageCount; ++k) CCTAGB_CUDA(cudaEventElapsedTime(&stage_ms_[k], st_ev_[k], st_ev_[k + 1]));
        return;
    }
    if (!graph_ || key != key_) {
        if (graph_) {
            cudaGraphExecDestroy(graph_);
            graph_ = nullptr;
        }
        cudaGraph_t g = nullptr;
        CCTAGB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        try {
            launch_image_stage(lv_, vp, s, fused, nullptr);
            launch_scatter_counters(d_cnt_, tg, s);
        } catch (...) {
            cudaStreamEndCapture(s, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        CCTAGB_CUDA(cudaStreamEndCapture(s, &g));
        const cudaError_t e = cudaGraphInstantiate(&graph_, g, 0);
        cudaGraphDestroy(g);
        CCTAGB_CUDA(e);
        key_ = key;
    }
    CCTAGB_CUDA(cudaEventRecord(ev0_, s));
    CCTAGB_CUDA(cudaGraphLaunch(graph_, s));
    CCTAGB_CUDA(cudaEventRecord(ev1_, s));
}

float BatchStage::finish_ms()
{
    if (!timing_) {
        CCTAGB_CUDA(cudaEventSynchronize(ev1_));
        CCTAGB_CUDA(cudaEventElapsedTime(&last_ms_, ev0_, ev1_));
    }
    return last_ms_;
}

void Pipeline::set_stage_timing(bool on)
{
    if (on == timing_) return;
    if (on && !st_ev_[0])
        for (cudaEvent_t& e : st_ev_) CCTAGB_CUDA(cudaEventCreate(&e));
    timing_ = on;
    std::fill(stage_ms_, stage_ms_ + kStageCount, 0.f);
}

void Pipeline::sync_counters(cudaStream_t s)
{
    CCTAGB_CUDA(cudaMemcpyAsync(h_cnt_, d_cnt_, sizeof(LevelCounters) * kMaxLevels, cudaMemcpyDeviceToHost, s));
    d2h_bytes_ += sizeof(LevelCounters) * kMaxLevels;
    waiter_.wait(s);
    for (int l = 0; l < lv_.n; ++l) {
        const int err = h_cnt_[l].err;
        if (err & kErrUnionFind) throw Error{CCTAGB_HYST_NO_CONVERGE, "hysteresis union-find exceeded its cap"};
        if (err & kErrEdgeOverflow)
            throw Error{CCTAGB_OVERFLOW_EDGES, "level " + std::to_string(l) + ": edge points exceed capacity " +
                                                   std::to_string(lv_.l[l].cap)};
        if (err & kErrSeedOverflow) throw Error{CCTAGB_OVERFLOW_SEEDS, "seed capacity exceeded"};
    }
}

void Pipeline::canny_only(const int16_t* dx, const int16_t* dy, int w, int h, uint8_t* edges_out)
{
    if (!dx || !dy || !edges_out || w < 1 || h < 1) throw Error{CCTAGB_BAD_ARG, "bad arguments"};
    set_views(w, h, 1);
    const size_t px = size_t(w) * h;
    CCTAGB_CUDA(cudaMemcpyAsync(lv_.l[0].dx, dx, px * 2, cudaMemcpyHostToDevice, stream_));
    CCTAGB_CUDA(cudaMemcpyAsync(lv_.l[0].dy, dy, px * 2, cudaMemcpyHostToDevice, stream_));
    launch_canny_only(lv_, vp_, stream_);
    sync_counters(stream_);
    copy_planes(0, nullptr, nullptr, nullptr, edges_out);
    graph_w_ = graph_h_ = -1;  // views were narrowed; force a fresh capture next frame
}

void Pipeline::level_size(int l, int* w, int* h) const
{
    if (l < 0 || l >= lv_.n) throw Error{CCTAGB_BAD_ARG, "level out of range"};
    *w = lv_.l[l].W;
    *h = lv_.l[l].H;
}

void Pipeline::copy_planes(int l, uint8_t* src, int16_t* dx, int16_t* dy, uint8_t* edges)
{
    if (l < 0 || l >= lv_.n) throw Error{CCTAGB_BAD_ARG, "level out of range"};
    const LevelView& v = lv_.l[l];
    const size_t px = size_t(v.W) * v.H;
    if (src) CCTAGB_CUDA(cudaMemcpyAsync(src, v.src, px, cudaMemcpyDeviceToHost, stream_));
    if (dx) CCTAGB_CUDA(cudaMemcpyAsync(dx, v.dx, px * 2, cudaMemcpyDeviceToHost, stream_));
    if (dy) CCTAGB_CUDA(cudaMemcpyAsync(dy, v.dy, px * 2, cudaMemcpyDeviceToHost, stream_));
    std::vector<uint32_t> bits;
    if (edges) {
        bits.resize(size_t(v.WW) * v.H);
        CCTAGB_CUDA(cudaMemcpyAsync(bits.data(), v.bitmap, bits.size() * 4, cudaMemcpyDeviceToHost, stream_));
    }
    waiter_.wait(stream_);
    if (edges) {
        for (int y = 0; y < v.H; ++y)
            for (int x = 0; x < v.W; ++x)
                edges[size_t(y) * v.W + x] = ((bits[size_t(y) * v.WW + (x >> 5)] >> (x & 31)) & 1u) ? 255 : 0;
    }
}

void Pipeline::issue_level_download(int l, bool voters)
{
    const LevelView& v = lv_.l[l];
    const LevelCounters& c = h_cnt_[l];
    LevelAlloc& a = la_[l];
    const int E = c.E;
    const int S = std::min(c.S, v.seedcap);
    auto d2h = [&](void* dst, const void* src, size_t bytes) {
        if (bytes) CCTAGB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream_));
    };
    d2h(a.h_exy, v.exy, size_t(E) * 4);
    d2h(a.h_grad, v.grad, size_t(E) * 4);
    d2h(a.h_before, v.before, size_t(E) * 4);
    d2h(a.h_after, v.after, size_t(E) * 4);
    if (voters) {
        d2h(a.h_voff, v.voff, size_t(E + 1) * 4);
        d2h(a.h_vlist, v.vlist, size_t(c.V) * 4);
        d2h(a.h_flow, v.flow, size_t(E) * 4);
    }
    d2h(a.h_sidx, v.seed_idx, size_t(S) * 4);
    d2h(a.h_skey, v.seed_key, size_t(S) * 4);
    d2h(a.h_svotes, v.seed_votes, size_t(S) * 4);
    d2h_bytes_ += (long long)E * 16 + (voters ? (long long)E * 8 + 4 + (long long)c.V * 4 : 0) + (long long)S * 12;
}

void Pipeline::finish_level_download(int l, HostLevel& out, bool voters)
{
    const LevelAlloc& a = la_[l];
    finish_level(l, out, voters, a.h_sidx, a.h_skey, a.h_svotes);
}

void Pipeline::finish_level(int l, HostLevel& out, bool voters, const int32_t* sidx, const int32_t* skey,
                            const int32_t* svotes)
{
    const LevelView& v = lv_.l[l];
    const LevelCounters& c = h_cnt_[l];
    const LevelAlloc& a = la_[l];
    out.W = v.W;
    out.H = v.H;
    out.E = c.E;
    out.V = c.V;
    out.exy = a.h_exy;
    out.grad = a.h_grad;
    out.before = a.h_before;
    out.after = a.h_after;
    out.voff = voters ? a.h_voff : nullptr;
    out.vlist = voters ? a.h_vlist : nullptr;
    out.flow = voters ? a.h_flow : nullptr;
    const int S = std::min(c.S, v.seedcap);
    // Seeds in the order vote() appends them (the voter that brings a point to
    // minVotes, Vote.cpp:236-241), then std::sort by votes received, as
    // Multiresolution.cpp:239-242 does (same comparator, same libstdc++ sort).
    // (The element sorted second carries its vote count along; std::sort's
    // permutation depends only on the comparisons, so it is the one of
    // sorting the indices with a vote-count comparator.)
    struct SeedRec {
        int32_t key, idx, votes;
    };
    std::vector<SeedRec> ks(static_cast<size_t>(S));
    for (int i = 0; i < S; ++i) ks[size_t(i)] = {skey[i], sidx[i], svotes[i]};
    std::sort(ks.begin(), ks.end(),
              [](const SeedRec& x, const SeedRec& y) { return x.key < y.key || (x.key == y.key && x.idx < y.idx); });
    std::vector<std::pair<int32_t, int32_t>> sv(static_cast<size_t>(S));
    for (int i = 0; i < S; ++i) sv[size_t(i)] = {ks[size_t(i)].idx, ks[size_t(i)].votes};
    if (S > 1)
        std::sort(sv.begin(), sv.end(),
                  [](const std::pair<int32_t, int32_t>& x, const std::pair<int32_t, int32_t>& y) {
                      return x.second > y.second;
                  });
    out.seeds.resize(S);
    for (int i = 0; i < S; ++i) out.seeds[size_t(i)] = sv[size_t(i)].first;
}

void Pipeline::download_level(int l, HostLevel& out)
{
    if (l < 0 || l >= lv_.n) throw Error{CCTAGB_BAD_ARG, "level out of range"};
    issue_level_download(l, true);
    waiter_.wait(stream_);
    finish_level_download(l, out, true);
}

void Pipeline::download_seeds_then_points(std::vector<HostLevel>& out)
{
    out.resize(lv_.n);
    // One compacting launch and two copies: the seeds of every level (index,
    // key, votes) on the pipeline stream, then the edge points' positions and
    // gradients on the copy stream.  The links stay on the device: the host
    // reads them only as the link chains of the loop-two candidates' points,
    // which loop one computes and downloads (LoopOneGpu::collect).
    PackSegs ps{};
    long long off = 0;
    auto seg = [&](const int32_t* src, long long n) {
        ps.src[ps.n] = src;
        ps.off[ps.n] = off;
        ++ps.n;
        off += n;
    };
    for (int l = 0; l < lv_.n; ++l) {
        const LevelView& v = lv_.l[l];
        const long long S = std::min(h_cnt_[l].S, v.seedcap);
        seg(v.seed_idx, S);
        seg(v.seed_key, S);
        seg(v.seed_votes, S);
    }
    const long long nseed = off;
    for (int l = 0; l < lv_.n; ++l) {
        const LevelView& v = lv_.l[l];
        const long long E = h_cnt_[l].E;
        seg(v.exy, E);
        seg(v.grad, E);
        seg(reinterpret_cast<const int32_t*>(v.bitidx), 2LL * v.WW * v.H);
    }
    ps.off[ps.n] = off;
    if (off > pack_words_) throw Error{CCTAGB_INTERNAL, "download staging too small"};
    launches_ += launch_pack(ps, d_pack_, stream_);
    CCTAGB_CUDA(cudaEventRecord(ev_pack_, stream_));
    if (nseed)
        CCTAGB_CUDA(cudaMemcpyAsync(h_pack_, d_pack_, size_t(nseed) * 4, cudaMemcpyDeviceToHost, stream_));
    CCTAGB_CUDA(cudaStreamWaitEvent(copy_stream_, ev_pack_, 0));
    if (off > nseed)
        CCTAGB_CUDA(cudaMemcpyAsync(h_pack_ + nseed, d_pack_ + nseed, size_t(off - nseed) * 4,
                                    cudaMemcpyDeviceToHost, copy_stream_));
    d2h_bytes_ += off * 4;
    for (int l = 0; l < lv_.n; ++l) {
        Packed& k = pk_[l];
        k.sidx = h_pack_ + ps.off[3 * l];
        k.skey = h_pack_ + ps.off[3 * l + 1];
        k.svotes = h_pack_ + ps.off[3 * l + 2];
        const int p = 3 * lv_.n + 3 * l;
        k.exy = h_pack_ + ps.off[p];
        k.grad = h_pack_ + ps.off[p + 1];
        k.bidx = h_pack_ + ps.off[p + 2];
        k.before = nullptr;
        k.after = nullptr;
    }
    waiter_.wait(stream_);
    for (int l = 0; l < lv_.n; ++l) {
        const Packed& k = pk_[l];
        finish_level(l, out[l], false, k.sidx, k.skey, k.svotes);
        out[l].exy = out[l].grad = out[l].before = out[l].after = nullptr;  // until wait_points()
    }
}

void Pipeline::wait_points(std::vector<HostLevel>& out)
{
    waiter_.wait(copy_stream_);
    for (int l = 0; l < lv_.n; ++l) {
        const Packed& k = pk_[l];
        out[l].exy = k.exy;
        out[l].grad = k.grad;
        out[l].before = k.before;
        out[l].after = k.after;
        out[l].bidx = k.bidx;
        out[l].WW = lv_.l[l].WW;
    }
}

void Pipeline::download_levels(std::vector<HostLevel>& out, bool voters)
{
    out.resize(lv_.n);
    for (int l = 0; l < lv_.n; ++l) issue_level_download(l, voters);
    waiter_.wait(stream_);
    for (int l = 0; l < lv_.n; ++l) finish_level_download(l, out[l], voters);
}

}  // namespace cctagb
