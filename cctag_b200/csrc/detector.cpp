// Detection driver (cctagDetection, Detection.cpp:773-999): image stage on
// the GPU, candidate stage on the host worker pool, level-0 re-fit, cut
// selection on the host, identification on the GPU, duplicate removal and
// sort.
#include "detector.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <future>
#include <list>

#include "bank_data.hpp"

namespace cctagb {

Detector::Detector(const cctagb_params& p, int max_w, int max_h, int max_batch, std::shared_ptr<ThreadPool> pool)
    : params_(p), pipe_(p, max_w, max_h, max_batch), pool_(std::move(pool))
{
    CCTAGB_CUDA(cudaMalloc(&d_bank_inv_, sizeof(float) * kMaxBankIds * kMaxBankRatios));
    if (p.nCrowns == 3) {
        for (const auto& row : kThreeCrownsBank) bank_.emplace_back(row, row + 5);
        upload_bank(bank_, d_bank_inv_);
    }
    int w = max_w, h = max_h;
    for (int l = 0; l < p.numberOfProcessedMultiresLayers; ++l) {
        idxmaps_.emplace_back(size_t(w) * h, -1);
        w /= 2;
        h /= 2;
    }
    CCTAGB_CUDA(cudaEventCreate(&ev_id0_));
    CCTAGB_CUDA(cudaEventCreate(&ev_id1_));
    ensure_ident_capacity(256);
    hl_.resize(idxmaps_.size());
    es_.resize(idxmaps_.size());
    if (!pool_) pool_ = make_host_pool(p.hostThreads);
}

Detector::~Detector()
{
    if (d_bank_inv_) cudaFree(d_bank_inv_);
    if (d_centers_) cudaFree(d_centers_);
    if (d_cost_) cudaFree(d_cost_);
    if (h_cost_) cudaFreeHost(h_cost_);
    if (d_tasks_) cudaFree(d_tasks_);
    if (d_res_) cudaFree(d_res_);
    if (h_tasks_) cudaFreeHost(h_tasks_);
    if (h_res_) cudaFreeHost(h_res_);
    if (frame_pinned_) cudaFreeHost(frame_pinned_);
    if (ev_id0_) cudaEventDestroy(ev_id0_);
    if (ev_id1_) cudaEventDestroy(ev_id1_);
}

void Detector::ensure_frame_pinned(size_t bytes)
{
    if (bytes <= frame_pinned_cap_) return;
    if (frame_pinned_) cudaFreeHost(frame_pinned_);
    frame_pinned_ = nullptr;
    frame_pinned_cap_ = 0;
    CCTAGB_CUDA(cudaMallocHost(&frame_pinned_, bytes));
    frame_pinned_cap_ = bytes;
}

void Detector::ensure_ident_capacity(int n)
{
    if (n <= ident_cap_) return;
    const int cap = std::max(n, 2 * ident_cap_);
    if (d_tasks_) cudaFree(d_tasks_);
    if (d_res_) cudaFree(d_res_);
    if (h_tasks_) cudaFreeHost(h_tasks_);
    if (h_res_) cudaFreeHost(h_res_);
    d_tasks_ = nullptr;
    d_res_ = nullptr;
    h_tasks_ = nullptr;
    h_res_ = nullptr;
    ident_cap_ = 0;
    CCTAGB_CUDA(cudaMalloc(&d_tasks_, sizeof(IdentTask) * cap));
    CCTAGB_CUDA(cudaMalloc(&d_res_, sizeof(IdentResult) * cap));
    CCTAGB_CUDA(cudaMallocHost(&h_tasks_, sizeof(IdentTask) * cap));
    CCTAGB_CUDA(cudaMallocHost(&h_res_, sizeof(IdentResult) * cap));
    ident_cap_ = cap;
}

void Detector::set_bank(const float* ratios, int n_ids, int n_ratios)
{
    if (!ratios || n_ids < 1 || n_ratios < 1) throw Error{CCTAGB_BANK_ERROR, "empty marker bank"};
    if (n_ratios != 2 * params_.nCrowns - 1)
        throw Error{CCTAGB_BANK_ERROR, "bank rows must hold 2*nCrowns-1 radius ratios"};
    if (n_ids > kMaxBankIds || n_ratios > kMaxBankRatios) throw Error{CCTAGB_BANK_ERROR, "bank too large"};
    std::vector<std::vector<float>> b(n_ids);
    for (int i = 0; i < n_ids; ++i) {
        b[i].assign(ratios + size_t(i) * n_ratios, ratios + size_t(i + 1) * n_ratios);
        for (float r : b[i])
            if (!(r > 1.f)) throw Error{CCTAGB_BANK_ERROR, "radius ratios must be > 1"};
    }
    upload_bank(b, d_bank_inv_);
    bank_ = std::move(b);
}

IdentParams Detector::ident_params(int refine_mode) const
{
    IdentParams ip{};
    ip.nSamples = std::min(params_.sampleCutLength, kMaxSamples);
    ip.beginSig = begin_signal(params_.nCrowns);
    ip.neighbourSize = params_.imagedCenterNeighbourSize;
    ip.gridN = params_.imagedCenterNGridSample;
    ip.minIdentProba = params_.minIdentProba;
    ip.nIds = bank_.empty() ? 0 : int(bank_.size());
    ip.nRatios = bank_.empty() ? 0 : int(bank_[0].size());
    ip.refineMode = refine_mode;
    ip.gnIterations = params_.gnIterations;
    ip.coarseRounds = params_.gnCoarseRounds;
    return ip;
}

void Detector::identify_on(const uint8_t* d_img, size_t pitch, const IdentTask* tasks, int n, const IdentParams& ip,
                           IdentResult* out)
{
    if (n <= 0) return;
    if (bank_.empty()) throw Error{CCTAGB_BANK_ERROR, "no marker bank for this number of crowns"};
    ensure_ident_capacity(n);
    std::memcpy(h_tasks_, tasks, sizeof(IdentTask) * n);
    cudaStream_t s = pipe_.stream();
    CCTAGB_CUDA(cudaMemcpyAsync(d_tasks_, h_tasks_, sizeof(IdentTask) * n, cudaMemcpyHostToDevice, s));
    CCTAGB_CUDA(cudaEventRecord(ev_id0_, s));
    launch_identify(d_img, pitch, d_tasks_, d_res_, n, d_bank_inv_, ip, s);
    CCTAGB_CUDA(cudaEventRecord(ev_id1_, s));
    CCTAGB_CUDA(cudaMemcpyAsync(h_res_, d_res_, sizeof(IdentResult) * n, cudaMemcpyDeviceToHost, s));
    CCTAGB_CUDA(cudaStreamSynchronize(s));
    std::memcpy(out, h_res_, sizeof(IdentResult) * n);
    pipe_.add_io((long long)sizeof(IdentTask) * n, (long long)sizeof(IdentResult) * n, 1);
}

void Detector::identify(const IdentTask* tasks, int n, IdentResult* out)
{
    int W, H;
    pipe_.level_size(0, &W, &H);
    identify_on(pipe_.level0_src(), size_t(W), tasks, n, ident_params(params_.refineMode), out);
}

namespace {

// Caller-given tasks must stay inside the image and within the kernel's limits.
void check_tasks(const IdentTask* tasks, int n, int w, int h, size_t pitch)
{
    if (n < 0 || (n > 0 && !tasks)) throw Error{CCTAGB_BAD_ARG, "bad task array"};
    if (w < 2 || h < 2 || pitch < size_t(w)) throw Error{CCTAGB_BAD_ARG, "bad image size or pitch"};
    for (int i = 0; i < n; ++i) {
        const IdentTask& t = tasks[i];
        const int* r = t.roi;
        if (r[0] < 0 || r[1] < 0 || r[2] < 2 || r[3] < 2 || r[0] + r[2] > w || r[1] + r[3] > h)
            throw Error{CCTAGB_BAD_ARG, "task " + std::to_string(i) + ": rectangle outside the image"};
        if (t.ncuts < 0 || t.ncuts > kMaxCuts)
            throw Error{CCTAGB_BAD_ARG, "task " + std::to_string(i) + ": ncuts out of range"};
        bool finite = std::isfinite(t.x0) && std::isfinite(t.y0) && std::isfinite(t.a) && std::isfinite(t.b);
        for (float q : t.Q) finite = finite && std::isfinite(q);
        for (int c = 0; c < t.ncuts; ++c) finite = finite && std::isfinite(t.stop[c][0]) && std::isfinite(t.stop[c][1]);
        if (!finite) throw Error{CCTAGB_BAD_ARG, "task " + std::to_string(i) + ": non-finite value"};
    }
}

}  // namespace

void Detector::identify_tasks(const uint8_t* d_img, int w, int h, size_t pitch, const IdentTask* tasks, int n,
                              int refine_mode, IdentResult* out)
{
    if (!d_img || (n > 0 && !out)) throw Error{CCTAGB_BAD_ARG, "bad image or output pointer"};
    check_tasks(tasks, n, w, h, pitch);
    identify_on(d_img, pitch, tasks, n, ident_params(refine_mode), out);
}

void Detector::cut_cost(const uint8_t* d_img, int w, int h, size_t pitch, const IdentTask* tasks, int n,
                        const float* centers, float* cost, float* d_center, float* d_h)
{
    if (!d_img || (n > 0 && !centers)) throw Error{CCTAGB_BAD_ARG, "bad image or center pointer"};
    check_tasks(tasks, n, w, h, pitch);
    if (n == 0) return;
    ensure_ident_capacity(n);
    if (n > cost_cap_) {
        if (d_centers_) cudaFree(d_centers_);
        if (d_cost_) cudaFree(d_cost_);
        if (h_cost_) cudaFreeHost(h_cost_);
        d_centers_ = nullptr;
        d_cost_ = nullptr;
        h_cost_ = nullptr;
        cost_cap_ = 0;
        CCTAGB_CUDA(cudaMalloc(&d_centers_, sizeof(float) * 2 * size_t(n)));
        CCTAGB_CUDA(cudaMalloc(&d_cost_, sizeof(float) * 12 * size_t(n)));
        CCTAGB_CUDA(cudaMallocHost(&h_cost_, sizeof(float) * 12 * size_t(n)));
        cost_cap_ = n;
    }
    std::memcpy(h_tasks_, tasks, sizeof(IdentTask) * n);
    std::memcpy(h_cost_, centers, sizeof(float) * 2 * size_t(n));
    cudaStream_t s = pipe_.stream();
    CCTAGB_CUDA(cudaMemcpyAsync(d_tasks_, h_tasks_, sizeof(IdentTask) * n, cudaMemcpyHostToDevice, s));
    CCTAGB_CUDA(cudaMemcpyAsync(d_centers_, h_cost_, sizeof(float) * 2 * size_t(n), cudaMemcpyHostToDevice, s));
    launch_cut_cost(d_img, pitch, d_tasks_, d_centers_, d_cost_, n, ident_params(params_.refineMode), s);
    CCTAGB_CUDA(cudaMemcpyAsync(h_cost_, d_cost_, sizeof(float) * 12 * size_t(n), cudaMemcpyDeviceToHost, s));
    CCTAGB_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < n; ++i) {
        const float* o = h_cost_ + 12 * size_t(i);
        if (cost) cost[i] = o[0];
        if (d_center) {
            d_center[2 * i] = o[1];
            d_center[2 * i + 1] = o[2];
        }
        if (d_h)
            for (int j = 0; j < 9; ++j) d_h[9 * size_t(i) + j] = o[3 + j];
    }
    pipe_.add_io((long long)(sizeof(IdentTask) + 8) * n, 48LL * n, 1);
}

namespace {

void fill_ellipse(const geo::Ellipse& e, cctagb_ellipse& o)
{
    o.cx = e.cx;
    o.cy = e.cy;
    o.a = e.a;
    o.b = e.b;
    o.angle = e.angle;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) o.m[r * 3 + c] = e.Q.m[r][c];
}

// CCTag::isEqual (CCTag.cpp:42-57): circles of radius b/2 around each
// center; equal when either contains the other's center.
bool markers_overlap(const MarkerCand& A, const MarkerCand& B)
{
    auto small = [](const geo::Ellipse& e) {
        return geo::Ellipse::from_params(e.cx, e.cy, e.b * 0.5f, e.b * 0.5f, e.angle);
    };
    const geo::Ellipse a = small(A.rescaled), b = small(B.rescaled);
    auto inside = [](const geo::Ellipse& e, float x, float y) {
        const geo::Mat3& Q = e.Q;
        const float s1 = geo::qform(Q, x, y);
        const float q0 = Q.m[0][0] * e.cx + Q.m[0][1] * e.cy + Q.m[0][2];
        const float q1 = Q.m[1][0] * e.cx + Q.m[1][1] * e.cy + Q.m[1][2];
        const float q2 = Q.m[2][0] * e.cx + Q.m[2][1] * e.cy + Q.m[2][2];
        return s1 * (x * q0 + y * q1 + q2) > 0;
    };
    return inside(a, b.cx, b.cy) || inside(b, a.cx, a.cy);
}

// Multiresolution.cpp:172-193 update(): keep the better of two overlapping
// identified markers.
void update(std::vector<MarkerCand>& list, const MarkerCand& m)
{
    bool flag = false;
    for (MarkerCand& cur : list) {
        if (cur.status > 0 && m.status > 0 && markers_overlap(cur, m)) {
            if (m.quality > cur.quality) cur = m;
            flag = true;
        }
    }
    if (!flag) list.push_back(m);
}

}  // namespace

void Detector::detect(const uint8_t* gray, int w, int h, size_t pitch, bool is_device, int frame_id,
                      cctagb_marker* out, int cap, int* n_out, cctagb_stats* stats)
{
    (void)frame_id;
    if (!n_out || (cap > 0 && !out)) throw Error{CCTAGB_BAD_ARG, "bad output arguments"};
    if (bank_.empty()) throw Error{CCTAGB_BANK_ERROR, "no marker bank for this number of crowns"};
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    last_tasks_.clear();
    pipe_.image_stage(gray, w, h, pitch, is_device);
    const int nl = pipe_.levels();

    // Candidate stage on the host worker pool: the per-level edge sets are
    // filled in parallel, then the phases of detect_from_edges spread their
    // seeds and candidates over the pool (deterministic for any pool size).
    const auto t1 = clk::now();
    std::vector<HostLevel>& hl = hl_;
    std::vector<EdgeSet>& es = es_;
    // A device frame is needed on the host for cut selection: its copy into
    // pinned memory rides with the edge-point downloads.
    const bool need_frame = params_.doIdentification && is_device;
    if (need_frame) {
        ensure_frame_pinned(size_t(w) * h);
        CCTAGB_CUDA(cudaMemcpyAsync(frame_pinned_, pipe_.level0_src(), size_t(w) * h, cudaMemcpyDeviceToHost,
                                    pipe_.stream()));
        pipe_.add_io(0, (long long)w * h, 0);
    }
    pipe_.download_levels(hl);
    const auto t1d = clk::now();
    auto fill_level = [&](int l) {
        EdgeSet& e = es[l];
        const HostLevel& L = hl[l];
        e.W = L.W;
        e.H = L.H;
        e.E = L.E;
        e.exy = L.exy;
        e.grad = L.grad;
        e.before = L.before;
        e.after = L.after;
        e.voff = L.voff;
        e.vlist = L.vlist;
        e.flow = L.flow;
        e.idxmap = idxmaps_[l].data();
        for (int i = 0; i < L.E; ++i) e.idxmap[size_t(L.exy[i] >> 16) * L.W + (L.exy[i] & 0xffff)] = i;
        e.reset_state();
    };
    pool_->parallel_for(nl, fill_level);
    std::vector<LevelJob> jobs(nl);
    for (int l = 0; l < nl; ++l) {
        jobs[l].es = &es[l];
        jobs[l].seeds = &hl[l].seeds;
        jobs[l].level = l;
        jobs[l].scale = float(1 << l);
    }
    detect_from_edges(jobs, params_,
                      [this](int n, const std::function<void(int)>& f) { pool_->parallel_for(n, f); });
    // Coarse levels first, as the reference's loop from the top level down.
    std::vector<MarkerCand> markers;
    for (int l = nl - 1; l >= 0; --l)
        for (auto& m : jobs[l].out) markers.push_back(std::move(m));
    geo::Pcg32 rng0(271828);
    refit_on_level0(es[0], markers, rng0);
    for (int l = 0; l < nl; ++l) {
        const HostLevel& L = hl[l];
        for (int i = 0; i < L.E; ++i) idxmaps_[l][size_t(L.exy[i] >> 16) * L.W + (L.exy[i] & 0xffff)] = -1;
    }
    const auto t2 = clk::now();

    // Identification.
    float ms_ident = 0.f, ms_cut = 0.f;
    if (params_.doIdentification && !markers.empty()) {
        const uint8_t* img = gray;
        size_t stride = pitch;
        if (is_device) {
            img = frame_pinned_;  // copied with the downloads
            stride = size_t(w);
        } else if (pitch != size_t(w)) {
            frame_host_.resize(size_t(w) * h);
            for (int y = 0; y < h; ++y) std::memcpy(&frame_host_[size_t(y) * w], gray + y * pitch, size_t(w));
            img = frame_host_.data();
            stride = size_t(w);
        }
        (void)stride;
        std::vector<IdentTask> all(markers.size());
        const auto tc0 = clk::now();
        pool_->parallel_for(int(markers.size()), [&](int i) {
            all[i] = IdentTask{};
            markers[i].status = identify_step1(markers[i], img, w, h, params_, all[i]);
        });
        ms_cut = std::chrono::duration<float, std::milli>(clk::now() - tc0).count();
        std::vector<IdentTask> tasks;
        std::vector<int> task_of(markers.size(), -1);
        for (size_t i = 0; i < markers.size(); ++i) {
            if (markers[i].status == CCTAGB_ID_RELIABLE) {
                task_of[i] = int(tasks.size());
                tasks.push_back(all[i]);
            }
        }
        last_tasks_ = tasks;
        std::vector<IdentResult> res(tasks.size());
        if (!tasks.empty()) {
            identify(tasks.data(), int(tasks.size()), res.data());
            CCTAGB_CUDA(cudaEventElapsedTime(&ms_ident, ev_id0_, ev_id1_));
        }
        for (size_t i = 0; i < markers.size(); ++i) {
            if (task_of[i] < 0) continue;
            const IdentResult& r = res[task_of[i]];
            MarkerCand& m = markers[i];
            m.status = r.status;
            m.cx_img = r.x;
            m.cy_img = r.y;
            m.quality = 1.f / r.residual;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) m.H.m[a][b] = r.H[a * 3 + b];
            if (r.status != CCTAGB_OPTI_HAS_DIVERGED) m.id = r.id;
            // Ring ellipses from the homography (Identification.cpp:1438-1459):
            // a singular H makes the marker degenerate.
            if (r.status != CCTAGB_OPTI_HAS_DIVERGED) {
                try {
                    (void)geo::inverse(m.H);
                } catch (...) {
                    m.status = CCTAGB_DEGENERATE;
                }
            }
        }
    }
    // Duplicate removal twice, then sort by id (Detection.cpp:975-989).
    std::vector<MarkerCand> prelim, fin;
    for (const auto& m : markers) update(prelim, m);
    for (const auto& m : prelim) update(fin, m);
    std::stable_sort(fin.begin(), fin.end(), [](const MarkerCand& a, const MarkerCand& b) { return a.id < b.id; });

    const int n = int(fin.size());
    *n_out = n;
    if (n > cap) throw Error{CCTAGB_BAD_ARG, "marker output capacity too small (" + std::to_string(n) + " markers)"};
    for (int i = 0; i < n; ++i) {
        const MarkerCand& m = fin[i];
        cctagb_marker& o = out[i];
        std::memset(&o, 0, sizeof(o));
        o.id = m.id;
        o.status = m.status;
        o.x = m.cx_img;
        o.y = m.cy_img;
        fill_ellipse(m.rescaled, o.outer);
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) o.homography[a * 3 + b] = m.H.m[a][b];
        o.quality = m.quality;
        o.pyramidLevel = m.level;
        o.scale = m.scale;
    }
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        for (int l = 0; l < nl; ++l) {
            stats->edge_points[l] = pipe_.counters(l).E;
            stats->seeds[l] = pipe_.counters(l).S;
        }
        stats->candidates = int(markers.size());
        stats->markers = n;
        stats->ms_image_stage = pipe_.last_image_stage_ms();
        stats->ms_host_candidates = std::chrono::duration<float, std::milli>(t2 - t1).count();
        stats->ms_identify = ms_ident;
        stats->ms_total = std::chrono::duration<float, std::milli>(clk::now() - t0).count();
        stats->h2d_bytes = pipe_.h2d_bytes();
        stats->d2h_bytes = pipe_.d2h_bytes();
        stats->kernel_launches = pipe_.kernel_launches();
        stats->ms_download = std::chrono::duration<float, std::milli>(t1d - t1).count();
        stats->ms_cut_selection = ms_cut;
    }
}

}  // namespace cctagb
