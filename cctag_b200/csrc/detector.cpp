// Detection driver: image stage on the GPU, candidate stage on the host,
// identification on the GPU (Detection.cpp:773-999 of the reference).
#include "detector.hpp"

#include <chrono>
#include <cstring>

#include "bank_data.hpp"

namespace cctagb {

Detector::Detector(const cctagb_params& p, int max_w, int max_h, int max_batch)
    : params_(p), pipe_(p, max_w, max_h, max_batch)
{
    if (p.nCrowns == 3) {
        for (const auto& row : kThreeCrownsBank) bank_.emplace_back(row, row + 5);
    }
}

void Detector::set_bank(const float* ratios, int n_ids, int n_ratios)
{
    if (!ratios || n_ids < 1 || n_ratios < 1) throw Error{CCTAGB_BANK_ERROR, "empty marker bank"};
    if (n_ratios != 2 * params_.nCrowns - 1)
        throw Error{CCTAGB_BANK_ERROR, "bank rows must hold 2*nCrowns-1 radius ratios"};
    std::vector<std::vector<float>> b(n_ids);
    for (int i = 0; i < n_ids; ++i) {
        b[i].assign(ratios + size_t(i) * n_ratios, ratios + size_t(i + 1) * n_ratios);
        for (float r : b[i])
            if (!(r > 1.f)) throw Error{CCTAGB_BANK_ERROR, "radius ratios must be > 1"};
    }
    bank_ = std::move(b);
}

void Detector::detect(const uint8_t* gray, int w, int h, size_t pitch, bool is_device, int frame_id,
                      cctagb_marker* out, int cap, int* n_out, cctagb_stats* stats)
{
    (void)frame_id;
    if (!n_out || (cap > 0 && !out)) throw Error{CCTAGB_BAD_ARG, "bad output arguments"};
    if (bank_.empty()) throw Error{CCTAGB_BANK_ERROR, "no marker bank for this number of crowns"};
    const auto t0 = std::chrono::steady_clock::now();
    pipe_.image_stage(gray, w, h, pitch, is_device);
    *n_out = 0;
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        for (int l = 0; l < pipe_.levels(); ++l) {
            stats->edge_points[l] = pipe_.counters(l).E;
            stats->seeds[l] = pipe_.counters(l).S;
        }
        stats->ms_image_stage = pipe_.last_image_stage_ms();
        stats->ms_total = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
}

}  // namespace cctagb
