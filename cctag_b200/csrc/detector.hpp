// One detection handle: the device pipeline, the marker bank and the host
// stages that sit between the GPU kernels (the reference's cctagDetection,
// Detection.cpp:773-999).
#pragma once

#include <chrono>

#include <memory>
#include <vector>

#include "candidates.hpp"
#include "grow.hpp"
#include "thread_pool.hpp"
#include "ident_host.hpp"
#include "loop_one.hpp"
#include "pipeline.hpp"

namespace cctagb {

class Detector {
public:
    // pool: the host worker pool (shared by the detectors of a handle); null
    // makes one with a thread per core besides the caller.
    Detector(const cctagb_params& p, int max_w, int max_h, int max_batch,
             std::shared_ptr<ThreadPool> pool = nullptr);
    ~Detector();
    Detector(const Detector&) = delete;
    Detector& operator=(const Detector&) = delete;

    Pipeline& pipeline() { return pipe_; }
    void set_ident_layout(int layout) { params_.identLayout = layout; }
    void set_pool(std::shared_ptr<ThreadPool> pool) { pool_ = std::move(pool); }
    void set_bank(const float* ratios, int n_ids, int n_ratios);
    const std::vector<std::vector<float>>& bank() const { return bank_; }

    void detect(const uint8_t* gray, int w, int h, size_t pitch, bool is_device, int frame_id, cctagb_marker* out,
                int cap, int* n_out, cctagb_stats* stats);
    // The rest of a detection whose image stage ran in a batched launch
    // (Pipeline::prepare_batched, BatchStage::run, event stage_done); t0 is
    // the start of the frame's call, for the statistics.
    void detect_batched(cudaEvent_t stage_done, float stage_ms, int stage_launches,
                        std::chrono::steady_clock::time_point t0, cctagb_marker* out, int cap, int* n_out,
                        cctagb_stats* stats);

    // Identification of caller-given markers (ellipse + initial center + cuts)
    // on the frame last passed to the image stage.
    void identify(const IdentTask* tasks, int n, IdentResult* out);
    // Batched identification / cost and adjoints on a caller's device image
    // (cctagb_identify_tasks, cctagb_cut_cost).
    void identify_tasks(const uint8_t* d_img, int w, int h, size_t pitch, const IdentTask* tasks, int n,
                        int refine_mode, IdentResult* out);
    void cut_cost(const uint8_t* d_img, int w, int h, size_t pitch, const IdentTask* tasks, int n,
                  const float* centers, float* cost, float* d_center, float* d_h, bool fp64 = false);
    // Tasks handed to the identification kernel by the last detect().
    const std::vector<IdentTask>& last_tasks() const { return last_tasks_; }
    // Loop-two inputs (GPU loop 1 + outlier removal) of the last detect().
    const std::vector<LoopTwoIn>& last_loop_two() const { return loop2in_; }

private:
    void after_image_stage(std::chrono::steady_clock::time_point t0, int w, int h, cctagb_marker* out, int cap,
                           int* n_out, cctagb_stats* stats);
    void ensure_ident_capacity(int n);
    void ensure_cut_capacity(int nm, int npts);
    // Cut selection and identification of the h_cutin_ / h_cutpts_ /
    // h_tasks_ markers on the level-0 frame; results in h_res_, h_st1_.
    void select_and_identify(int nm, int npts, int w, int h);
    IdentParams ident_params(int refine_mode) const;
    void identify_on(const uint8_t* d_img, size_t pitch, const IdentTask* tasks, int n, const IdentParams& ip,
                     IdentResult* out);

    cctagb_params params_;
    Pipeline pipe_;
    std::vector<std::vector<float>> bank_;
    std::vector<HostLevel> hl_;                  // per level, pinned downloads
    std::vector<EdgeSet> es_;                    // per level, candidate-stage state
    std::unique_ptr<LoopOneGpu> loop1_;          // loop 1 + outlier removal on the GPU
    std::unique_ptr<GrowGpu> grow_;              // ellipse growing on the GPU (gpuEllipseGrowing)
    std::vector<LoopTwoIn> loop2in_;             // its results for the last frame
    std::shared_ptr<ThreadPool> pool_;
    CutSelectIn* d_cutin_ = nullptr;             // cut selection inputs (device / pinned)
    CutSelectIn* h_cutin_ = nullptr;
    DirPoint* d_cutpts_ = nullptr;               // sorted outer points of all markers
    DirPoint* h_cutpts_ = nullptr;
    int* d_st1_ = nullptr;                       // cut selection status per marker
    int16_t* d_sel_ = nullptr;                   // per marker: its selected outer points (k_outer_select)
    int* d_nsel_ = nullptr;
    int* h_st1_ = nullptr;
    int cut_cap_ = 0, pts_cap_ = 0;
    float* d_bank_inv_ = nullptr;                // kMaxBankIds x kMaxBankRatios
    IdentTask* d_tasks_ = nullptr;
    IdentResult* d_res_ = nullptr;
    IdentTask* h_tasks_ = nullptr;
    IdentResult* h_res_ = nullptr;
    int ident_cap_ = 0;
    float* d_centers_ = nullptr;
    float* d_cost_ = nullptr;
    float* h_cost_ = nullptr;
    int cost_cap_ = 0;
    std::vector<IdentTask> last_tasks_;
    cudaEvent_t ev_id0_ = nullptr, ev_id1_ = nullptr;
};

}  // namespace cctagb
