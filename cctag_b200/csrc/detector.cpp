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
    CCTAGB_CUDA(cudaEventCreate(&ev_id0_));
    CCTAGB_CUDA(cudaEventCreate(&ev_id1_));
    ensure_ident_capacity(256);
    hl_.resize(size_t(p.numberOfProcessedMultiresLayers));
    es_.resize(size_t(p.numberOfProcessedMultiresLayers));
    if (!pool_) pool_ = make_host_pool(p.hostThreads);
    std::vector<int> caps;
    for (int l = 0; l < p.numberOfProcessedMultiresLayers; ++l) caps.push_back(pipe_.level_capacity(l));
    loop1_ = std::make_unique<LoopOneGpu>(p, max_h, caps);
    if (p.gpuEllipseGrowing) grow_ = std::make_unique<GrowGpu>(p.hostSpinMicros, p.gpuGrowMaxPoints);
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
    if (d_cutin_) cudaFree(d_cutin_);
    if (h_cutin_) cudaFreeHost(h_cutin_);
    if (d_cutpts_) cudaFree(d_cutpts_);
    if (h_cutpts_) cudaFreeHost(h_cutpts_);
    if (d_st1_) cudaFree(d_st1_);
    if (h_st1_) cudaFreeHost(h_st1_);
    if (d_sel_) cudaFree(d_sel_);
    if (d_nsel_) cudaFree(d_nsel_);
    if (ev_id0_) cudaEventDestroy(ev_id0_);
    if (ev_id1_) cudaEventDestroy(ev_id1_);
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
    ip.layout = params_.identLayout;
    if (refine_mode == CCTAGB_REFINE_GAUSS_NEWTON) {
        // the coarse rounds only pick the basin Gauss-Newton then descends
        ip.gridN = params_.gnCoarseGrid;
        ip.neighbourSize = params_.gnCoarseNeighbourSize;
    }
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
    pipe_.host_wait(s);
    std::memcpy(out, h_res_, sizeof(IdentResult) * n);
    pipe_.add_io((long long)sizeof(IdentTask) * n, (long long)sizeof(IdentResult) * n, 1);
}

void Detector::ensure_cut_capacity(int nm, int npts)
{
    ensure_ident_capacity(nm);
    if (nm > cut_cap_) {
        if (d_cutin_) cudaFree(d_cutin_);
        if (h_cutin_) cudaFreeHost(h_cutin_);
        if (d_st1_) cudaFree(d_st1_);
        if (h_st1_) cudaFreeHost(h_st1_);
        if (d_sel_) cudaFree(d_sel_);
        if (d_nsel_) cudaFree(d_nsel_);
        d_cutin_ = nullptr;
        h_cutin_ = nullptr;
        d_st1_ = nullptr;
        h_st1_ = nullptr;
        d_sel_ = nullptr;
        d_nsel_ = nullptr;
        cut_cap_ = 0;
        const int cap = std::max(nm, 256);
        CCTAGB_CUDA(cudaMalloc(&d_cutin_, sizeof(CutSelectIn) * cap));
        CCTAGB_CUDA(cudaMallocHost(&h_cutin_, sizeof(CutSelectIn) * cap));
        CCTAGB_CUDA(cudaMalloc(&d_st1_, sizeof(int) * cap));
        CCTAGB_CUDA(cudaMallocHost(&h_st1_, sizeof(int) * cap));
        CCTAGB_CUDA(cudaMalloc(&d_sel_, sizeof(int16_t) * kMaxOuterPoints * size_t(cap)));
        CCTAGB_CUDA(cudaMalloc(&d_nsel_, sizeof(int) * cap));
        cut_cap_ = cap;
    }
    if (npts > pts_cap_) {
        if (d_cutpts_) cudaFree(d_cutpts_);
        if (h_cutpts_) cudaFreeHost(h_cutpts_);
        d_cutpts_ = nullptr;
        h_cutpts_ = nullptr;
        pts_cap_ = 0;
        const int cap = std::max(npts, 16384);
        CCTAGB_CUDA(cudaMalloc(&d_cutpts_, sizeof(DirPoint) * cap));
        CCTAGB_CUDA(cudaMallocHost(&h_cutpts_, sizeof(DirPoint) * cap));
        pts_cap_ = cap;
    }
}

void Detector::select_and_identify(int nm, int npts, int w, int h)
{
    if (bank_.empty()) throw Error{CCTAGB_BANK_ERROR, "no marker bank for this number of crowns"};
    cudaStream_t s = pipe_.stream();
    CCTAGB_CUDA(cudaMemcpyAsync(d_cutin_, h_cutin_, sizeof(CutSelectIn) * nm, cudaMemcpyHostToDevice, s));
    CCTAGB_CUDA(cudaMemcpyAsync(d_cutpts_, h_cutpts_, sizeof(DirPoint) * npts, cudaMemcpyHostToDevice, s));
    CCTAGB_CUDA(cudaMemcpyAsync(d_tasks_, h_tasks_, sizeof(IdentTask) * nm, cudaMemcpyHostToDevice, s));
    CutSelectParams cp{};
    cp.beginSig = begin_signal(params_.nCrowns);
    cp.nSamples = std::min(params_.sampleCutLength, kMaxSamples);
    cp.nRefine = params_.numSamplesOuterEdgePointsRefinement;
    cp.maxSelect = std::min(params_.numCutsInIdentStep, kMaxCuts);
    cp.nOuter = params_.nSamplesOuterEllipse;
    launch_outer_select(d_cutin_, d_cutpts_, cp.nOuter, d_sel_, d_nsel_, nm, s);
    launch_cut_select(pipe_.level0_src(), w, h, d_cutin_, d_cutpts_, d_sel_, d_nsel_, d_tasks_, d_st1_, nm, cp, s);
    CCTAGB_CUDA(cudaEventRecord(ev_id0_, s));
    launch_identify(pipe_.level0_src(), size_t(w), d_tasks_, d_res_, nm, d_bank_inv_,
                    ident_params(params_.refineMode), s);
    CCTAGB_CUDA(cudaEventRecord(ev_id1_, s));
    CCTAGB_CUDA(cudaMemcpyAsync(h_res_, d_res_, sizeof(IdentResult) * nm, cudaMemcpyDeviceToHost, s));
    CCTAGB_CUDA(cudaMemcpyAsync(h_st1_, d_st1_, sizeof(int) * nm, cudaMemcpyDeviceToHost, s));
    CCTAGB_CUDA(cudaMemcpyAsync(h_tasks_, d_tasks_, sizeof(IdentTask) * nm, cudaMemcpyDeviceToHost, s));
    pipe_.host_wait(s);
    pipe_.add_io((long long)(sizeof(CutSelectIn) + sizeof(IdentTask)) * nm + (long long)sizeof(DirPoint) * npts,
                 (long long)(sizeof(IdentResult) + sizeof(int) + sizeof(IdentTask)) * nm, 3);
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

void Detector::identify(const IdentTask* tasks, int n, IdentResult* out)
{
    int W, H;
    pipe_.level_size(0, &W, &H);
    check_tasks(tasks, n, W, H, size_t(W));
    identify_on(pipe_.level0_src(), size_t(W), tasks, n, ident_params(params_.refineMode), out);
}

void Detector::identify_tasks(const uint8_t* d_img, int w, int h, size_t pitch, const IdentTask* tasks, int n,
                              int refine_mode, IdentResult* out)
{
    if (!d_img || (n > 0 && !out)) throw Error{CCTAGB_BAD_ARG, "bad image or output pointer"};
    check_tasks(tasks, n, w, h, pitch);
    identify_on(d_img, pitch, tasks, n, ident_params(refine_mode), out);
}

void Detector::cut_cost(const uint8_t* d_img, int w, int h, size_t pitch, const IdentTask* tasks, int n,
                        const float* centers, float* cost, float* d_center, float* d_h, bool fp64)
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
    launch_cut_cost(d_img, pitch, d_tasks_, d_centers_, d_cost_, n, ident_params(params_.refineMode), s, fp64);
    CCTAGB_CUDA(cudaMemcpyAsync(h_cost_, d_cost_, sizeof(float) * 12 * size_t(n), cudaMemcpyDeviceToHost, s));
    pipe_.host_wait(s);
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
    const auto t0 = std::chrono::steady_clock::now();
    last_tasks_.clear();
    pipe_.image_stage(gray, w, h, pitch, is_device);
    after_image_stage(t0, w, h, out, cap, n_out, stats);
}

void Detector::detect_batched(cudaEvent_t stage_done, float stage_ms, int stage_launches,
                              std::chrono::steady_clock::time_point t0, cctagb_marker* out, int cap, int* n_out,
                              cctagb_stats* stats)
{
    if (!n_out || (cap > 0 && !out)) throw Error{CCTAGB_BAD_ARG, "bad output arguments"};
    if (bank_.empty()) throw Error{CCTAGB_BANK_ERROR, "no marker bank for this number of crowns"};
    last_tasks_.clear();
    pipe_.finish_batched(stage_done, stage_ms, stage_launches);
    int w = 0, h = 0;
    pipe_.level_size(0, &w, &h);
    after_image_stage(t0, w, h, out, cap, n_out, stats);
}

void Detector::after_image_stage(std::chrono::steady_clock::time_point t0, int w, int h, cctagb_marker* out, int cap,
                                 int* n_out, cctagb_stats* stats)
{
    using clk = std::chrono::steady_clock;
    const int nl = pipe_.levels();

    // Candidate stage on the host worker pool: the per-level edge sets are
    // filled in parallel, then the phases of detect_from_edges spread their
    // seeds and candidates over the pool (deterministic for any pool size).
    const auto t1 = clk::now();
    std::vector<HostLevel>& hl = hl_;
    std::vector<EdgeSet>& es = es_;
    pipe_.download_seeds_then_points(hl);
    // Loop 1 and the outlier removal run on the GPU while the host indexes the
    // edge points.
    {
        std::vector<const std::vector<int32_t>*> seeds(static_cast<size_t>(nl));
        int E[kMaxLevels] = {};
        for (int l = 0; l < nl; ++l) {
            seeds[size_t(l)] = &hl[l].seeds;
            E[l] = hl[l].E;
        }
        loop1_->launch(pipe_.level_views(), E, seeds, pipe_.stream());
    }
    pipe_.wait_points(hl);
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
        if (L.bidx) {  // the GPU's word + first-index plane, downloaded with the points
            e.bidx = reinterpret_cast<const EdgeSet::Word*>(L.bidx);
            e.WW = L.WW;
        } else {
            e.index_points();
        }
        e.reset_state();
    };
    // on this thread: with the GPU's index planes the levels only take
    // pointers (a pooled task could wait behind other frames' work)
    for (int l = 0; l < nl; ++l) fill_level(l);
    loop1_->collect(pipe_.stream(), loop2in_);
    pipe_.add_io(loop1_->h2d_bytes(), loop1_->d2h_bytes(), loop1_->launches());
    std::vector<LevelJob> jobs(nl);
    for (int l = 0; l < nl; ++l) {
        jobs[l].es = &es[l];
        jobs[l].seeds = &hl[l].seeds;
        jobs[l].level = l;
        jobs[l].scale = float(1 << l);
    }
    // Ellipse growing of the candidates on the GPU: their filtered points up,
    // outer points and ellipses down.
    GrowFn growFn = [&](std::vector<GrowJob>& gj) {
        std::vector<GrowTask> tasks(gj.size());
        std::vector<int32_t> pts;
        for (size_t k = 0; k < gj.size(); ++k) {
            tasks[k].level = gj[k].level;
            tasks[k].first = int(pts.size());
            tasks[k].count = int(gj[k].filtered->size());
            pts.insert(pts.end(), gj[k].filtered->begin(), gj[k].filtered->end());
        }
        int E[kMaxLevels] = {};
        for (int l = 0; l < nl; ++l) E[l] = hl[l].E;
        std::vector<GrowResult> res;
        std::vector<int32_t> outer;
        int stride = 0;
        grow_->run(pipe_.level_views(), E, tasks, pts, params_.ellipseGrowingEllipticHullWidth,
                   params_.thrMedianDistanceEllipse, pipe_.stream(), res, outer, stride);
        pipe_.add_io(grow_->h2d_bytes(), grow_->d2h_bytes(), grow_->launches());
        for (size_t k = 0; k < gj.size(); ++k) {
            const GrowResult& r = res[k];
            gj[k].status = r.status == kGrowKeep ? 1 : r.status == kGrowDrop ? 0 : 2;
            if (r.status != kGrowKeep) continue;
            const int32_t* o = outer.data() + k * size_t(stride);
            gj[k].outer->assign(o, o + r.nOuter);
            *gj[k].ellipse = geo::Ellipse::from_params(r.cx, r.cy, r.a, r.b, r.angle);
        }
    };
    int grown[2] = {};
    detect_from_edges(
        jobs, params_, [this](int n, const std::function<void(int)>& f) { pool_->parallel_for(n, f); }, &loop2in_,
        grow_ ? &growFn : nullptr, grown);
    // Coarse levels first, as the reference's loop from the top level down.
    std::vector<MarkerCand> markers;
    for (int l = nl - 1; l >= 0; --l)
        for (auto& m : jobs[l].out) markers.push_back(std::move(m));
    // Level-0 re-fit of coarse-level markers: hull and outlier removal on the
    // GPU, the ellipse fit on the host.
    {
        std::vector<RefitTask> rt;
        std::vector<int> rtIdx;
        for (size_t mi = 0; mi < markers.size(); ++mi) {
            MarkerCand& m = markers[mi];
            if (m.level > 0) {
                RefitHull h;
                refit_hull(m, h);
                RefitTask t;
                std::copy(h.qin, h.qin + 9, t.qin);
                std::copy(h.qout, h.qout + 9, t.qout);
                t.inCx = h.inCx;
                t.inCy = h.inCy;
                t.yc = h.yc;
                t.marker = int(mi);
                rt.push_back(t);
                rtIdx.push_back(int(mi));
            } else {
                m.rescaled_points = m.points.empty() ? std::vector<DirPoint>() : m.points.back();
            }
        }
        if (!rt.empty()) {
            std::vector<std::vector<int32_t>> flt;
            const long long h0 = loop1_->h2d_bytes(), d0 = loop1_->d2h_bytes();
            loop1_->refit(pipe_.level_views(), rt, pipe_.stream(), flt);
            pipe_.add_io(loop1_->h2d_bytes() - h0, loop1_->d2h_bytes() - d0, loop1_->refit_launches());
            pool_->parallel_for(int(rt.size()), [&](int k) {
                refit_apply(es[0], markers[size_t(rtIdx[size_t(k)])], flt[size_t(k)].data(), flt[size_t(k)].size());
            });
        }
    }
    const auto t2 = clk::now();

    // Identification: the outer points sorted by angle, subsampled, cut
    // selection and identification on the GPU, on the level-0 frame there (a
    // marker with more outer points than the sort kernel holds is sorted and
    // subsampled here).
    float ms_ident = 0.f, ms_cut = 0.f;
    if (params_.doIdentification && !markers.empty()) {
        const int nm = int(markers.size());
        const auto tc0 = clk::now();
        if (params_.nSamplesOuterEllipse < 0 || params_.nSamplesOuterEllipse > kMaxOuterPoints)
            throw Error{CCTAGB_BAD_ARG, "nSamplesOuterEllipse above " + std::to_string(kMaxOuterPoints)};
        std::vector<std::vector<DirPoint>> presorted(markers.size());
        std::vector<int> big;
        for (int i = 0; i < nm; ++i)
            if (markers[size_t(i)].rescaled_points.size() > size_t(kCutSortCap)) big.push_back(i);
        pool_->parallel_for(int(big.size()), [&](int k) {
            const MarkerCand& m = markers[size_t(big[size_t(k)])];
            presorted[size_t(big[size_t(k)])] =
                sorted_outer_points(m.rescaled, m.rescaled_points, size_t(params_.nSamplesOuterEllipse));
        });
        auto points_of = [&](int i) -> const std::vector<DirPoint>& {
            const MarkerCand& m = markers[size_t(i)];
            return m.rescaled_points.size() > size_t(kCutSortCap) ? presorted[size_t(i)] : m.rescaled_points;
        };
        int npts = 0;
        for (int i = 0; i < nm; ++i) npts += int(points_of(i).size());
        ensure_cut_capacity(nm, npts);
        int first = 0;
        for (int i = 0; i < nm; ++i) {
            const MarkerCand& m = markers[size_t(i)];
            const geo::Ellipse& e = m.rescaled;
            const auto& o = points_of(i);
            CutSelectIn& ci = h_cutin_[i];
            ci.cx = e.cx;
            ci.cy = e.cy;
            ci.a = e.a;
            ci.b = e.b;
            ci.cosA = std::cos(e.angle);
            ci.sinA = std::sin(e.angle);
            ci.scale = m.scale;
            ci.first = first;
            ci.count = int(o.size());
            ci.presorted = m.rescaled_points.size() > size_t(kCutSortCap) ? 1 : 0;
            std::copy(o.begin(), o.end(), h_cutpts_ + first);
            first += int(o.size());
            IdentTask& t = h_tasks_[i];
            t = IdentTask{};
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) t.Q[r * 3 + c] = e.Q.m[r][c];
            t.cx = e.cx;
            t.cy = e.cy;
            t.a = e.a;
            t.b = e.b;
            t.angle = e.angle;
            t.x0 = m.cx_img;
            t.y0 = m.cy_img;
            t.roi[0] = 0;
            t.roi[1] = 0;
            t.roi[2] = w;
            t.roi[3] = h;
        }
        ms_cut = std::chrono::duration<float, std::milli>(clk::now() - tc0).count();
        select_and_identify(nm, npts, w, h);
        CCTAGB_CUDA(cudaEventElapsedTime(&ms_ident, ev_id0_, ev_id1_));
        for (int i = 0; i < nm; ++i)
            if (h_st1_[i] == CCTAGB_ID_RELIABLE) last_tasks_.push_back(h_tasks_[i]);
        for (int i = 0; i < nm; ++i) {
            MarkerCand& m = markers[size_t(i)];
            if (h_st1_[i] != CCTAGB_ID_RELIABLE) {
                m.status = h_st1_[i];
                continue;
            }
            const IdentResult& r = h_res_[i];
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
        stats->grown_gpu = grown[0];
        stats->grown_host = grown[1];
    }
}

}  // namespace cctagb
