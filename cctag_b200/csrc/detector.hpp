// One detection handle: the device pipeline, the marker bank and the host
// stages that sit between the GPU kernels (the reference's cctagDetection,
// Detection.cpp:773-999).
#pragma once

#include <vector>

#include "pipeline.hpp"

namespace cctagb {

class Detector {
public:
    Detector(const cctagb_params& p, int max_w, int max_h, int max_batch);

    Pipeline& pipeline() { return pipe_; }
    void set_bank(const float* ratios, int n_ids, int n_ratios);
    const std::vector<std::vector<float>>& bank() const { return bank_; }

    void detect(const uint8_t* gray, int w, int h, size_t pitch, bool is_device, int frame_id, cctagb_marker* out,
                int cap, int* n_out, cctagb_stats* stats);

private:
    cctagb_params params_;
    Pipeline pipe_;
    std::vector<std::vector<float>> bank_;
};

}  // namespace cctagb
