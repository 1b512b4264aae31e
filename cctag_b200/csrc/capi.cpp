// C ABI of the library (include/cctag_b200.h).  Converts exceptions into
// status codes; nothing crosses the ABI as a C++ exception.
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "autotune.hpp"
#include "cctag_b200.h"
#include "detector.hpp"
#include "pipeline.hpp"

namespace {

// One frame handed to cctagb_submit, and what its detection returned.
struct Ticket {
    const uint8_t* gray = nullptr;
    int w = 0, h = 0;
    size_t pitch = 0;
    int is_device = 0, frame_id = 0;
    bool done = false;
    cctagb_status status = CCTAGB_OK;
    std::string msg;
    std::vector<cctagb_marker> markers;
    int n = 0;
    cctagb_stats stats{};
};

}  // namespace

struct cctagb_handle {
    std::shared_ptr<cctagb::ThreadPool> pool;     // host workers shared by every slot
    std::shared_ptr<cctagb::StageOrder> order;    // image stages of the slots, in submission order
    std::unique_ptr<cctagb::Detector> det;        // slot 0: every single-frame call
    std::vector<std::unique_ptr<cctagb::Detector>> extra;  // slots 1..: cctagb_detect_batch
    cctagb_params params{};
    int max_w = 0, max_h = 0, max_batch = 1, device = 0;
    int pool_threads = 0;                         // the host pool's size, counting the caller
    std::string last_error;

    int slots() const { return std::max(1, std::min(max_batch, kMaxSlots)); }
    static constexpr int kMaxSlots = 32;
    // Detection slots for a batch: own device buffers and stream, the host
    // pool shared.
    void ensure_slots(int n)
    {
        while (int(extra.size()) + 1 < n) {
            extra.emplace_back(new cctagb::Detector(params, max_w, max_h, 1, pool));
            extra.back()->pipeline().set_stage_order(order);
            copy_bank(*extra.back());
        }
    }
    void copy_bank(cctagb::Detector& d) const
    {
        const auto& b = det->bank();
        if (b.empty()) return;
        std::vector<float> flat;
        for (const auto& row : b) flat.insert(flat.end(), row.begin(), row.end());
        d.set_bank(flat.data(), int(b.size()), int(b[0].size()));
    }
    cctagb::Detector& slot(int i) { return i == 0 ? *det : *extra[size_t(i - 1)]; }
    // Batch configuration (cctagb_autotune): on the handle's parameters and
    // on every slot made so far (later slots copy the parameters).
    void set_batch_config(int wave, int layout, int threads)
    {
        params.batchWaveFrames = wave;
        params.identLayout = layout;
        det->set_ident_layout(layout);
        for (auto& d : extra) d->set_ident_layout(layout);
        const int t = threads > 0 ? threads : default_pool_threads();
        if (t != pool_threads) {
            pool = cctagb::make_host_pool(t);
            det->set_pool(pool);
            for (auto& d : extra) d->set_pool(pool);
            pool_threads = t;
        }
        params.hostThreads = threads;
    }
    // One thread per physical core, less one per detection slot beyond the
    // first -- a slot's own thread works in its frame's parallel loops and
    // spins while it waits on the GPU (measured on a 16-core host with 8
    // slots: 8 pool threads 1.09-1.13 k frames/s, 16 threads 0.99 k).
    int default_pool_threads() const { return std::max(2, cctagb::physical_cores() - (slots() - 1)); }

    // Streaming ingest (cctagb_submit / cctagb_wait): one worker thread per
    // slot takes queued tickets in order.
    std::vector<uint8_t*> host_frames;            // pinned, max_w * max_h bytes each
    std::mutex smu;
    std::condition_variable scv, sdone;
    std::deque<int> queue;
    std::map<int, std::shared_ptr<Ticket>> tickets;
    std::vector<std::thread> sworkers;
    int next_ticket = 1;
    bool sstop = false;

    void stream_worker(int s)
    {
        cudaSetDevice(device);
        cctagb::Detector& d = slot(s);
        for (;;) {
            std::shared_ptr<Ticket> t;
            {
                std::unique_lock<std::mutex> l(smu);
                scv.wait(l, [&] { return sstop || !queue.empty(); });
                if (sstop) return;
                t = tickets.at(queue.front());
                queue.pop_front();
            }
            cctagb_status st = CCTAGB_OK;
            std::string msg;
            t->markers.resize(256);
            for (int attempt = 0; attempt < 2; ++attempt) {
                try {
                    d.detect(t->gray, t->w, t->h, t->pitch, t->is_device != 0, t->frame_id, t->markers.data(),
                             int(t->markers.size()), &t->n, &t->stats);
                    st = CCTAGB_OK;
                    msg.clear();
                    break;
                } catch (const cctagb::Error& e) {
                    st = e.status;
                    msg = e.msg;
                    // more markers than the buffer holds: once more with room
                    if (st != CCTAGB_BAD_ARG || t->n <= int(t->markers.size())) break;
                    t->markers.resize(size_t(t->n));
                } catch (const std::exception& e) {
                    st = CCTAGB_INTERNAL;
                    msg = e.what();
                    break;
                }
            }
            {
                std::lock_guard<std::mutex> l(smu);
                t->status = st;
                t->msg = msg;
                t->done = true;
            }
            sdone.notify_all();
        }
    }
    void start_stream()
    {
        if (!sworkers.empty()) return;
        const int S = slots();
        ensure_slots(S);
        for (int s = 0; s < S; ++s) sworkers.emplace_back([this, s] { stream_worker(s); });
    }
    bool streaming() const { return !tickets.empty(); }

    // Batched image stage of cctagb_detect_batch: one launch per kernel for
    // the frames of a wave, on its own (lowest-priority) stream.
    // One batch-stage state and completion event per wave in flight.
    std::vector<std::unique_ptr<cctagb::BatchStage>> batch;
    std::vector<cudaEvent_t> bdone;
    cudaStream_t bstream = nullptr;
    bool batch_timing = false;
    bool last_timed_batch = false;  // stage times: of the last batch, else of the last single frame
    int last_batch = 0;             // the wave state whose stage times are the last batch's
    void ensure_batch(int d)
    {
        if (!bstream) {
            int least = 0, greatest = 0;
            CCTAGB_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
            CCTAGB_CUDA(cudaStreamCreateWithPriority(&bstream, cudaStreamNonBlocking, least));
        }
        while (int(batch.size()) < d) {
            cudaEvent_t e = nullptr;
            CCTAGB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            bdone.push_back(e);
            batch.push_back(std::make_unique<cctagb::BatchStage>());
            batch.back()->set_stage_timing(batch_timing);
        }
    }

    ~cctagb_handle()
    {
        {
            std::lock_guard<std::mutex> l(smu);
            sstop = true;
        }
        scv.notify_all();
        for (auto& t : sworkers) t.join();
        if (det) cudaStreamSynchronize(det->pipeline().stream());
        for (auto& d : extra) cudaStreamSynchronize(d->pipeline().stream());
        if (bstream) cudaStreamSynchronize(bstream);
        batch.clear();
        for (cudaEvent_t e : bdone) cudaEventDestroy(e);
        if (bstream) cudaStreamDestroy(bstream);
        for (uint8_t* p : host_frames) cudaFreeHost(p);
    }
};

namespace {

template <class F>
cctagb_status guarded(cctagb_handle* h, F&& f)
{
    try {
        f();
        if (h) h->last_error.clear();
        return CCTAGB_OK;
    } catch (const cctagb::Error& e) {
        if (h) h->last_error = e.msg;
        return e.status;
    } catch (const std::bad_alloc&) {
        if (h) h->last_error = "host allocation failed";
        return CCTAGB_INTERNAL;
    } catch (const std::exception& e) {
        if (h) h->last_error = e.what();
        return CCTAGB_INTERNAL;
    } catch (...) {
        if (h) h->last_error = "unknown error";
        return CCTAGB_INTERNAL;
    }
}

// Slot 0 belongs to the streaming workers while tickets are outstanding.
bool refuse_if_streaming(cctagb_handle* h)
{
    if (!h->streaming()) return false;
    h->last_error = "tickets outstanding: wait for them first";
    return true;
}

}  // namespace

extern "C" {

void cctagb_params_default(cctagb_params* p, int nCrowns)
{
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->cannyThrLow = 0.01f;
    p->cannyThrHigh = 0.04f;
    p->distSearch = 30;
    p->thrGradientMagInVote = 2500;
    p->angleVoting = 0.f;
    p->ratioVoting = 4.f;
    p->averageVoteMin = 0.f;
    p->thrMedianDistanceEllipse = 3.f;
    p->maximumNbSeeds = 500;
    p->maximumNbCandidatesLoopTwo = 40;
    p->nCrowns = nCrowns;
    p->nCircles = 2 * nCrowns;
    p->minPointsSegmentCandidate = 10;
    p->minVotesToSelectCandidate = 3;
    p->threshRobustEstimationOfOuterEllipse = 30.f;
    p->ellipseGrowingEllipticHullWidth = 2.3f;
    p->windowSizeOnInnerEllipticSegment = 20;
    p->numberOfMultiresLayers = 4;
    p->numberOfProcessedMultiresLayers = 4;
    p->nSamplesOuterEllipse = 150;
    p->numCutsInIdentStep = 22;
    p->numSamplesOuterEdgePointsRefinement = 20;
    p->cutsSelectionTrials = 500;
    p->sampleCutLength = 100;
    p->imagedCenterNGridSample = 5;
    p->imagedCenterNeighbourSize = 0.20f;
    p->minIdentProba = 1e-6f;
    p->useLMDif = 1;
    p->searchForAnotherSegment = 1;
    p->writeOutput = 0;
    p->doIdentification = 1;
    p->maxEdges = 20000;
    p->refineMode = CCTAGB_REFINE_GRID;
    p->gnIterations = 12;
    p->gnCoarseRounds = 1;
    p->edgeCapacityDivisor = 4;
    p->gnCoarseGrid = 3;
    p->gnCoarseNeighbourSize = 0.1f;
    p->batchWaveFrames = 4;
    p->identLayout = CCTAGB_IDENT_AUTO;
    p->hostSpinMicros = -1;
    p->gpuEllipseGrowing = 0;
    p->gpuGrowMaxPoints = 2048;
}

const char* cctagb_status_string(cctagb_status s)
{
    switch (s) {
    case CCTAGB_OK: return "ok";
    case CCTAGB_BAD_ARG: return "bad argument";
    case CCTAGB_CUDA_ERROR: return "CUDA error";
    case CCTAGB_NO_DEVICE: return "no sm_100 CUDA device";
    case CCTAGB_OVERFLOW_EDGES: return "edge-point capacity exceeded";
    case CCTAGB_OVERFLOW_SEEDS: return "seed capacity exceeded";
    case CCTAGB_OVERFLOW_VOTERS: return "voter capacity exceeded";
    case CCTAGB_HYST_NO_CONVERGE: return "hysteresis did not converge";
    case CCTAGB_TOO_LARGE: return "frame larger than the handle";
    case CCTAGB_BANK_ERROR: return "bad marker bank";
    case CCTAGB_INTERNAL: return "internal error";
    }
    return "unknown status";
}

cctagb_status cctagb_create(const cctagb_params* p, int max_w, int max_h, int max_batch, cctagb_handle** out)
{
    if (!out) return CCTAGB_BAD_ARG;
    *out = nullptr;
    cctagb_params def;
    if (!p) {
        cctagb_params_default(&def, 3);
        p = &def;
    }
    std::unique_ptr<cctagb_handle> h(new (std::nothrow) cctagb_handle);
    if (!h) return CCTAGB_INTERNAL;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return CCTAGB_NO_DEVICE;
    }
    if (p->identLayout != CCTAGB_IDENT_AUTO && p->identLayout != CCTAGB_IDENT_BLOCK) return CCTAGB_BAD_ARG;
    h->params = *p;
    h->max_w = max_w;
    h->max_h = max_h;
    h->max_batch = max_batch;
    cudaGetDevice(&h->device);
    const cctagb_status s = guarded(h.get(), [&] {
        const int threads = p->hostThreads > 0 ? p->hostThreads : h->default_pool_threads();
        h->pool = cctagb::make_host_pool(threads);
        h->pool_threads = threads;
        h->det.reset(new cctagb::Detector(*p, max_w, max_h, max_batch, h->pool));
        h->order = std::make_shared<cctagb::StageOrder>();
        h->det->pipeline().set_stage_order(h->order);
    });
    if (s != CCTAGB_OK) return s;
    *out = h.release();
    return CCTAGB_OK;
}

cctagb_status cctagb_destroy(cctagb_handle* h)
{
    if (!h) return CCTAGB_BAD_ARG;
    delete h;
    return CCTAGB_OK;
}

const char* cctagb_last_error_string(const cctagb_handle* h) { return h ? h->last_error.c_str() : "null handle"; }

cctagb_status cctagb_set_bank(cctagb_handle* h, const float* ratios, int n_ids, int n_ratios)
{
    if (!h) return CCTAGB_BAD_ARG;
    if (refuse_if_streaming(h)) return CCTAGB_BAD_ARG;
    return guarded(h, [&] {
        h->det->set_bank(ratios, n_ids, n_ratios);
        for (auto& d : h->extra) d->set_bank(ratios, n_ids, n_ratios);
    });
}

cctagb_status cctagb_image_stage(cctagb_handle* h, const uint8_t* gray, int w, int hgt, size_t pitch, int is_device)
{
    if (!h) return CCTAGB_BAD_ARG;
    if (refuse_if_streaming(h)) return CCTAGB_BAD_ARG;
    return guarded(h, [&] { h->det->pipeline().image_stage(gray, w, hgt, pitch, is_device != 0); });
}

cctagb_status cctagb_level_size(cctagb_handle* h, int level, int* w, int* hgt)
{
    if (!h || !w || !hgt) return CCTAGB_BAD_ARG;
    return guarded(h, [&] { h->det->pipeline().level_size(level, w, hgt); });
}

cctagb_status cctagb_level_planes(cctagb_handle* h, int level, uint8_t* src, int16_t* dx, int16_t* dy, uint8_t* edges)
{
    if (!h) return CCTAGB_BAD_ARG;
    return guarded(h, [&] { h->det->pipeline().copy_planes(level, src, dx, dy, edges); });
}

cctagb_status cctagb_level_edge_points(cctagb_handle* h, int level, int cap, int* n, int32_t* x, int32_t* y)
{
    if (!h || !n) return CCTAGB_BAD_ARG;
    return guarded(h, [&] {
        cctagb::HostLevel hl;
        h->det->pipeline().download_level(level, hl);
        *n = hl.E;
        if (hl.E > cap) throw cctagb::Error{CCTAGB_BAD_ARG, "output capacity too small"};
        for (int i = 0; i < hl.E; ++i) {
            if (x) x[i] = hl.exy[i] & 0xffff;
            if (y) y[i] = hl.exy[i] >> 16;
        }
    });
}

cctagb_status cctagb_level_links(cctagb_handle* h, int level, int cap, int32_t* before, int32_t* after)
{
    if (!h) return CCTAGB_BAD_ARG;
    return guarded(h, [&] {
        cctagb::HostLevel hl;
        h->det->pipeline().download_level(level, hl);
        if (hl.E > cap) throw cctagb::Error{CCTAGB_BAD_ARG, "output capacity too small"};
        if (before) std::copy(hl.before, hl.before + hl.E, before);
        if (after) std::copy(hl.after, hl.after + hl.E, after);
    });
}

cctagb_status cctagb_level_votes(cctagb_handle* h, int level, int cap, int32_t* chosen, int32_t* nvotes,
                                 float* flow_length, int32_t* voter_off, int32_t* voter_list, int voter_cap,
                                 int32_t* n_voters)
{
    if (!h) return CCTAGB_BAD_ARG;
    return guarded(h, [&] {
        cctagb::HostLevel hl;
        h->det->pipeline().download_level(level, hl);
        if (hl.E > cap || hl.V > voter_cap) throw cctagb::Error{CCTAGB_BAD_ARG, "output capacity too small"};
        if (n_voters) *n_voters = hl.V;
        if (chosen) {
            std::fill(chosen, chosen + hl.E, -1);
            for (int c = 0; c < hl.E; ++c)
                for (int k = hl.voff[c]; k < hl.voff[c + 1]; ++k) chosen[hl.vlist[k]] = c;
        }
        for (int c = 0; c < hl.E; ++c) {
            if (nvotes) nvotes[c] = hl.voff[c + 1] - hl.voff[c];
            if (flow_length) flow_length[c] = hl.flow[c];
        }
        if (voter_off) std::copy(hl.voff, hl.voff + hl.E + 1, voter_off);
        if (voter_list) std::copy(hl.vlist, hl.vlist + hl.V, voter_list);
    });
}

cctagb_status cctagb_level_seeds(cctagb_handle* h, int level, int cap, int32_t* seeds, int* n)
{
    if (!h || !n) return CCTAGB_BAD_ARG;
    return guarded(h, [&] {
        cctagb::HostLevel hl;
        h->det->pipeline().download_level(level, hl);
        *n = int(hl.seeds.size());
        if (*n > cap) throw cctagb::Error{CCTAGB_BAD_ARG, "output capacity too small"};
        if (seeds) std::copy(hl.seeds.begin(), hl.seeds.end(), seeds);
    });
}

cctagb_status cctagb_level_loop_two(cctagb_handle* h, int level, int cap, int32_t* seed, int32_t* score,
                                    int32_t* keep, int32_t* n_filtered, int* n, int filtered_cap,
                                    int32_t* filtered, int* n_filtered_total)
{
    if (!h || !n || !n_filtered_total) return CCTAGB_BAD_ARG;
    if (refuse_if_streaming(h)) return CCTAGB_BAD_ARG;
    return guarded(h, [&] {
        const auto& all = h->det->last_loop_two();
        if (level < 0 || level >= int(all.size())) throw cctagb::Error{CCTAGB_BAD_ARG, "level out of range"};
        const cctagb::LoopTwoIn& g = all[size_t(level)];
        *n = int(g.seed.size());
        *n_filtered_total = int(g.flt.size());
        if (*n > cap || *n_filtered_total > filtered_cap)
            throw cctagb::Error{CCTAGB_BAD_ARG, "output capacity too small"};
        for (int i = 0; i < *n; ++i) {
            if (seed) seed[i] = g.seed[size_t(i)];
            if (score) score[i] = g.score[size_t(i)];
            if (keep) keep[i] = g.keep[size_t(i)];
            if (n_filtered) n_filtered[i] = g.foff[size_t(i) + 1] - g.foff[size_t(i)];
        }
        if (filtered) std::copy(g.flt.begin(), g.flt.end(), filtered);
    });
}

cctagb_status cctagb_get_stream(cctagb_handle* h, void** stream)
{
    if (!h || !stream) return CCTAGB_BAD_ARG;
    *stream = reinterpret_cast<void*>(h->det->pipeline().stream());
    return CCTAGB_OK;
}

cctagb_status cctagb_set_stage_timing(cctagb_handle* h, int enable)
{
    if (!h) return CCTAGB_BAD_ARG;
    if (refuse_if_streaming(h)) return CCTAGB_BAD_ARG;
    return guarded(h, [&] {
        h->det->pipeline().set_stage_timing(enable != 0);
        h->batch_timing = enable != 0;
        for (auto& b : h->batch) b->set_stage_timing(enable != 0);
        h->last_timed_batch = false;
    });
}

cctagb_status cctagb_stage_times(cctagb_handle* h, int cap, float* ms, int* n)
{
    if (!h || !n) return CCTAGB_BAD_ARG;
    *n = cctagb::kStageCount;
    if (cap < cctagb::kStageCount || !ms) return CCTAGB_BAD_ARG;
    const float* src = h->last_timed_batch && !h->batch.empty() ? h->batch[size_t(h->last_batch)]->stage_ms()
                                                                : h->det->pipeline().stage_ms();
    std::copy(src, src + cctagb::kStageCount, ms);
    return CCTAGB_OK;
}

const char* cctagb_stage_name(int stage) { return cctagb::stage_name(stage); }

cctagb_status cctagb_canny_from_derivatives(cctagb_handle* h, const int16_t* dx, const int16_t* dy, int w, int hgt,
                                            uint8_t* edges)
{
    if (!h) return CCTAGB_BAD_ARG;
    if (refuse_if_streaming(h)) return CCTAGB_BAD_ARG;
    return guarded(h, [&] { h->det->pipeline().canny_only(dx, dy, w, hgt, edges); });
}

cctagb_status cctagb_detect(cctagb_handle* h, const uint8_t* gray, int w, int hgt, size_t pitch, int frame_id,
                            cctagb_marker* out, int cap, int* n_out, cctagb_stats* stats)
{
    if (!h) return CCTAGB_BAD_ARG;
    if (refuse_if_streaming(h)) return CCTAGB_BAD_ARG;
    h->last_timed_batch = false;
    return guarded(h, [&] { h->det->detect(gray, w, hgt, pitch, false, frame_id, out, cap, n_out, stats); });
}

cctagb_status cctagb_detect_device(cctagb_handle* h, const uint8_t* d_gray, int w, int hgt, size_t pitch,
                                   int frame_id, cctagb_marker* out, int cap, int* n_out, cctagb_stats* stats)
{
    if (!h) return CCTAGB_BAD_ARG;
    if (refuse_if_streaming(h)) return CCTAGB_BAD_ARG;
    h->last_timed_batch = false;
    return guarded(h, [&] { h->det->detect(d_gray, w, hgt, pitch, true, frame_id, out, cap, n_out, stats); });
}

cctagb_status cctagb_host_frames(cctagb_handle* h, int n, uint8_t** out)
{
    if (!h || n < 0 || n > 64 || (n > 0 && !out)) return CCTAGB_BAD_ARG;
    return guarded(h, [&] {
        const size_t bytes = size_t(h->max_w) * size_t(h->max_h);
        while (int(h->host_frames.size()) < n) {
            uint8_t* p = nullptr;
            CCTAGB_CUDA(cudaMallocHost(&p, bytes));
            h->host_frames.push_back(p);
        }
        for (int i = 0; i < n; ++i) out[i] = h->host_frames[size_t(i)];
    });
}

cctagb_status cctagb_submit(cctagb_handle* h, const uint8_t* gray, int w, int hgt, size_t pitch, int is_device,
                            int frame_id, int* ticket)
{
    if (!h || !gray || !ticket || w <= 0 || hgt <= 0 || pitch < size_t(w)) return CCTAGB_BAD_ARG;
    return guarded(h, [&] {
        if (w > h->max_w || hgt > h->max_h) throw cctagb::Error{CCTAGB_TOO_LARGE, "frame larger than the handle"};
        h->start_stream();
        auto t = std::make_shared<Ticket>();
        t->gray = gray;
        t->w = w;
        t->h = hgt;
        t->pitch = pitch;
        t->is_device = is_device;
        t->frame_id = frame_id;
        {
            std::lock_guard<std::mutex> l(h->smu);
            *ticket = h->next_ticket++;
            h->tickets[*ticket] = t;
            h->queue.push_back(*ticket);
        }
        h->scv.notify_one();
    });
}

cctagb_status cctagb_wait(cctagb_handle* h, int ticket, cctagb_marker* out, int cap, int* n_out, cctagb_stats* stats)
{
    if (!h || !n_out || (cap > 0 && !out)) return CCTAGB_BAD_ARG;
    std::shared_ptr<Ticket> t;
    {
        std::unique_lock<std::mutex> l(h->smu);
        auto it = h->tickets.find(ticket);
        if (it == h->tickets.end()) {
            h->last_error = "unknown ticket";
            return CCTAGB_BAD_ARG;
        }
        t = it->second;
        h->sdone.wait(l, [&] { return t->done; });
        // a buffer too small for the markers keeps the ticket: the caller
        // can wait on it again with *n_out places
        if (t->status == CCTAGB_OK && t->n > cap) {
            *n_out = t->n;
            h->last_error = "marker output capacity too small";
            return CCTAGB_BAD_ARG;
        }
        h->tickets.erase(h->tickets.find(ticket));
    }
    *n_out = t->n;
    if (stats) *stats = t->stats;
    if (t->status != CCTAGB_OK) {
        h->last_error = "frame " + std::to_string(t->frame_id) + ": " + t->msg;
        return t->status;
    }
    std::copy(t->markers.begin(), t->markers.begin() + t->n, out);
    h->last_error.clear();
    return CCTAGB_OK;
}

cctagb_status cctagb_last_tasks(cctagb_handle* h, cctagb_cut_task* out, int cap, int* n)
{
    if (!h || !n || (cap > 0 && !out)) return CCTAGB_BAD_ARG;
    if (refuse_if_streaming(h)) return CCTAGB_BAD_ARG;
    return guarded(h, [&] {
        const auto& t = h->det->last_tasks();
        *n = int(t.size());
        if (*n > cap) throw cctagb::Error{CCTAGB_BAD_ARG, "output capacity too small"};
        std::copy(t.begin(), t.end(), out);
    });
}

cctagb_status cctagb_identify_tasks(cctagb_handle* h, const uint8_t* d_img, int w, int hgt, size_t pitch,
                                    const cctagb_cut_task* tasks, int n, int refine_mode, cctagb_ident_result* out)
{
    if (!h) return CCTAGB_BAD_ARG;
    if (refuse_if_streaming(h)) return CCTAGB_BAD_ARG;
    return guarded(h, [&] { h->det->identify_tasks(d_img, w, hgt, pitch, tasks, n, refine_mode, out); });
}

cctagb_status cctagb_cut_cost(cctagb_handle* h, const uint8_t* d_img, int w, int hgt, size_t pitch,
                              const cctagb_cut_task* tasks, int n, const float* centers, float* cost,
                              float* d_center, float* d_h)
{
    if (!h) return CCTAGB_BAD_ARG;
    if (refuse_if_streaming(h)) return CCTAGB_BAD_ARG;
    return guarded(h, [&] { h->det->cut_cost(d_img, w, hgt, pitch, tasks, n, centers, cost, d_center, d_h); });
}

cctagb_status cctagb_cut_cost_f64(cctagb_handle* h, const uint8_t* d_img, int w, int hgt, size_t pitch,
                                  const cctagb_cut_task* tasks, int n, const float* centers, float* cost,
                                  float* d_center, float* d_h)
{
    if (!h) return CCTAGB_BAD_ARG;
    if (refuse_if_streaming(h)) return CCTAGB_BAD_ARG;
    return guarded(h, [&] { h->det->cut_cost(d_img, w, hgt, pitch, tasks, n, centers, cost, d_center, d_h, true); });
}

cctagb_status cctagb_detect_batch(cctagb_handle* h, cctagb_frame* frames, int n)
{
    if (!h || n < 0 || (n > 0 && !frames)) return CCTAGB_BAD_ARG;
    if (refuse_if_streaming(h)) return CCTAGB_BAD_ARG;
    if (n == 0) return CCTAGB_OK;
    return guarded(h, [&] {
        // Waves of wf frames: the image stages of a wave's frames run as one
        // batched launch per kernel (on the lowest-priority batch stream, in
        // wave order), then frame j of the wave continues on its detection
        // slot.  The slots hold D = slots / wf waves in flight: wave k reuses
        // the slots (and batch-stage state) of wave k - D once that wave's
        // frames are done, so later waves' stages overlap earlier frames'
        // GPU and host stages.  A frame's result does not depend on the wave
        // or slot that ran it.
        const int S = h->slots();
        const int wf = std::max(1, std::min({h->params.batchWaveFrames, cctagb::kMaxBatchFrames, S, n}));
        const int D = std::max(1, std::min(S / wf, (n + wf - 1) / wf));
        h->ensure_slots(D * wf);
        h->ensure_batch(D);
        for (int i = 0; i < n; ++i) {
            frames[i].n_out = 0;
            frames[i].status = CCTAGB_INTERNAL;
        }
        std::vector<std::string> msg(static_cast<size_t>(n));
        std::mutex msg_mu;
        auto fail = [&](int i, cctagb_status st, std::string m) {
            std::lock_guard<std::mutex> l(msg_mu);
            frames[i].status = st;
            msg[size_t(i)] = std::move(m);
        };
        std::vector<std::vector<std::thread>> inflight(static_cast<size_t>(D));
        auto drain = [&](int d) {
            for (auto& t : inflight[size_t(d)]) t.join();
            inflight[size_t(d)].clear();
        };
        struct Joiner {  // every started frame is joined, also when a launch throws
            std::function<void()> f;
            ~Joiner() { f(); }
        } joiner{[&] {
            for (int d = 0; d < D; ++d) drain(d);
        }};
        for (int k = 0, w0 = 0; w0 < n; ++k, w0 += wf) {
            const int d = k % D, nw = std::min(wf, n - w0);
            drain(d);  // the wave that last used these slots is done
            const auto t0 = std::chrono::steady_clock::now();
            std::vector<cctagb::Pipeline*> pipes;
            std::vector<int> started;  // wave frame j -> its slot, -1 if it failed to start
            for (int j = 0; j < nw; ++j) {
                cctagb_frame& f = frames[w0 + j];
                const int s = d * wf + j;
                try {
                    h->slot(s).pipeline().prepare_batched(f.gray, f.w, f.h, f.pitch, f.is_device != 0, h->bstream);
                    pipes.push_back(&h->slot(s).pipeline());
                    started.push_back(s);
                } catch (const cctagb::Error& e) {
                    fail(w0 + j, e.status, e.msg);
                    started.push_back(-1);
                }
            }
            if (pipes.empty()) continue;
            cctagb::BatchStage& bs = *h->batch[size_t(d)];
            bs.run(pipes, h->bstream);
            CCTAGB_CUDA(cudaEventRecord(h->bdone[size_t(d)], h->bstream));
            h->last_timed_batch = h->batch_timing;
            h->last_batch = d;
            const cudaEvent_t done = h->bdone[size_t(d)];
            bool first = true;
            for (int j = 0; j < nw; ++j) {
                const int s = started[size_t(j)];
                if (s < 0) continue;
                const int launches = first ? bs.launches() : 0;
                first = false;
                inflight[size_t(d)].emplace_back([&, s, j, w0, t0, done, launches, d] {
                    cudaSetDevice(h->device);
                    cctagb_frame& f = frames[w0 + j];
                    try {
                        h->slot(s).detect_batched(done, -1.f, launches, t0, f.out, f.cap, &f.n_out, &f.stats);
                        f.stats.ms_image_stage = h->batch[size_t(d)]->elapsed_ms();
                        f.status = CCTAGB_OK;
                    } catch (const cctagb::Error& e) {
                        fail(w0 + j, e.status, e.msg);
                    } catch (const std::exception& e) {
                        fail(w0 + j, CCTAGB_INTERNAL, e.what());
                    } catch (...) {
                        fail(w0 + j, CCTAGB_INTERNAL, "unknown error");
                    }
                });
            }
        }
        joiner.f();
        joiner.f = [] {};
        for (int i = 0; i < n; ++i)
            if (frames[i].status != CCTAGB_OK)
                throw cctagb::Error{frames[i].status, "frame " + std::to_string(i) + ": " + msg[size_t(i)]};
    });
}

cctagb_status cctagb_tune_key(const char* gpu_name, int sm_count, int w, int hgt, int frames, int nCrowns, char* out,
                              int cap)
{
    if (!gpu_name || !out || cap < 1) return CCTAGB_BAD_ARG;
    const std::string k = cctagb::tune::key(gpu_name, sm_count, w, hgt, frames, nCrowns);
    if (k.size() + 1 > size_t(cap)) return CCTAGB_BAD_ARG;
    std::memcpy(out, k.c_str(), k.size() + 1);
    return CCTAGB_OK;
}

cctagb_status cctagb_tune_cache_get(const char* cache_path, const char* key, cctagb_tune_choice* out)
{
    if (!cache_path || !key || !out) return CCTAGB_BAD_ARG;
    try {
        cctagb_tune_choice c{};
        if (!cctagb::tune::cache_get(cache_path, key, c)) return CCTAGB_BAD_ARG;
        *out = c;
        return CCTAGB_OK;
    } catch (...) {
        return CCTAGB_INTERNAL;
    }
}

cctagb_status cctagb_tune_cache_put(const char* cache_path, const char* key, const cctagb_tune_choice* c)
{
    if (!cache_path || !key || !c) return CCTAGB_BAD_ARG;
    if (c->batchWaveFrames < 1 || c->batchWaveFrames > cctagb::kMaxBatchFrames) return CCTAGB_BAD_ARG;
    if (c->identLayout != CCTAGB_IDENT_AUTO && c->identLayout != CCTAGB_IDENT_BLOCK) return CCTAGB_BAD_ARG;
    if (c->hostThreads < 0 || c->hostThreads > 64) return CCTAGB_BAD_ARG;
    return guarded(nullptr, [&] { cctagb::tune::cache_put(cache_path, key, *c); });
}

cctagb_status cctagb_autotune(cctagb_handle* h, cctagb_frame* frames, int n, const char* cache_path, int reps,
                              cctagb_tune_choice* out)
{
    if (!h || !frames || n < 1 || !out || reps < 1 || reps > 100) return CCTAGB_BAD_ARG;
    if (refuse_if_streaming(h)) return CCTAGB_BAD_ARG;
    bool uniform = true;
    long long total_px = 0;
    for (int i = 0; i < n; ++i) {
        uniform = uniform && frames[i].w == frames[0].w && frames[i].h == frames[0].h;
        total_px += (long long)frames[i].w * frames[i].h;
    }
    std::string key;
    const cctagb_status ks = guarded(h, [&] {
        cudaDeviceProp prop{};
        CCTAGB_CUDA(cudaGetDeviceProperties(&prop, h->device));
        key = uniform ? cctagb::tune::key(prop.name, prop.multiProcessorCount, frames[0].w, frames[0].h, n,
                                          h->params.nCrowns)
                      : cctagb::tune::key_mixed(prop.name, prop.multiProcessorCount, total_px, n, h->params.nCrowns);
    });
    if (ks != CCTAGB_OK) return ks;
    cctagb_tune_choice best{};
    if (cache_path && cctagb::tune::cache_get(cache_path, key, best)) {
        const cctagb_status st = guarded(h, [&] { h->set_batch_config(best.batchWaveFrames, best.identLayout,
                                                                      best.hostThreads); });
        if (st != CCTAGB_OK) return st;
        *out = best;
        return CCTAGB_OK;
    }
    // Candidates: wave sizes 1, 2, 4, .. up to the frames (and slots) of a
    // call, each with both identification layouts, at the handle's pool
    // size; then, with the best of those, pools of 4, 8 and 16 threads.  The
    // least median wall time of a cctagb_detect_batch call wins.
    const int maxWave = std::max(1, std::min({n, h->slots(), cctagb::kMaxBatchFrames}));
    const int threads0 = h->params.hostThreads;
    std::vector<std::array<int, 3>> cand;
    for (int wf = 1; wf <= maxWave; wf *= 2)
        for (int layout : {CCTAGB_IDENT_AUTO, CCTAGB_IDENT_BLOCK}) cand.push_back({wf, layout, threads0});
    const cctagb_params saved = h->params;
    cctagb_tune_choice res{};
    float bestMs = 0.f;
    auto measure = [&](const std::array<int, 3>& c) -> cctagb_status {
        if (res.n_tried >= CCTAGB_TUNE_MAX_TRIED) return CCTAGB_OK;
        cctagb_status st = guarded(h, [&] { h->set_batch_config(c[0], c[1], c[2]); });
        if (st == CCTAGB_OK) st = cctagb_detect_batch(h, frames, n);  // untimed: graphs, slots, caches
        std::vector<float> ms;
        for (int r = 0; r < reps && st == CCTAGB_OK; ++r) {
            const auto t0 = std::chrono::steady_clock::now();
            st = cctagb_detect_batch(h, frames, n);
            ms.push_back(std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count());
        }
        if (st != CCTAGB_OK) return st;
        std::sort(ms.begin(), ms.end());
        const float perFrame = ms[ms.size() / 2] / float(n);
        const int k = res.n_tried++;
        res.tried_wave[k] = c[0];
        res.tried_layout[k] = c[1];
        res.tried_threads[k] = c[2];
        res.tried_ms_per_frame[k] = perFrame;
        if (k == 0 || perFrame < bestMs) {
            bestMs = perFrame;
            res.batchWaveFrames = c[0];
            res.identLayout = c[1];
            res.hostThreads = c[2];
        }
        return CCTAGB_OK;
    };
    cctagb_status st = CCTAGB_OK;
    for (const auto& c : cand)
        if (st == CCTAGB_OK) st = measure(c);
    const int base = h->default_pool_threads();
    for (int t : {4, 8, 16})
        if (st == CCTAGB_OK && t != (threads0 > 0 ? threads0 : base))
            st = measure({res.batchWaveFrames, res.identLayout, t});
    if (st != CCTAGB_OK) {
        guarded(h, [&] { h->set_batch_config(saved.batchWaveFrames, saved.identLayout, saved.hostThreads); });
        return st;
    }
    res.ms_per_frame = bestMs;
    res.from_cache = 0;
    {
        const cctagb_status s2 = guarded(h, [&] { h->set_batch_config(res.batchWaveFrames, res.identLayout,
                                                                       res.hostThreads); });
        if (s2 != CCTAGB_OK) return s2;
    }
    *out = res;
    if (cache_path) return guarded(h, [&] { cctagb::tune::cache_put(cache_path, key, res); });
    return CCTAGB_OK;
}

}  // extern "C"
