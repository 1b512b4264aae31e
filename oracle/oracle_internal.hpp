// TEST INFRASTRUCTURE ONLY -- C++ declarations shared by the oracle sources.
#pragma once
#include <cstdint>

namespace orc {

struct VoteParams {
    int distSearch;
    int thrGradientMagInVote;
    float angleVoting;
    float ratioVoting;
    int nCrowns;
    int minVotesToSelectCandidate;
};

void pyramid_down(const uint8_t* src, int sw, int sh, uint8_t* dst, int dw, int dh);
void derivatives(const uint8_t* src, int W, int H, int16_t* dx, int16_t* dy);
void canny(const int16_t* dx, const int16_t* dy, int W, int H, float thrLow, float thrHigh, uint8_t* edges,
           uint8_t* nms_out);
void thin_lut(int pass, uint8_t* lut);
void thin(uint8_t* edges, int W, int H);
int gradient_walk(const int32_t* idxmap, int W, int H, int px, int py, int gdx, int gdy, int dir, int nmax,
                  int thrGradient);
int vote(const uint8_t* edges, const int16_t* dxm, const int16_t* dym, int W, int H, const VoteParams& vp, int cap,
         int32_t* ex, int32_t* ey, int32_t* before, int32_t* after, int32_t* chosen_out, float* total_out,
         int32_t* nvotes, int32_t* is_max, float* flow_length, int32_t* voter_off, int32_t* voter_list,
         int32_t* seeds_push, int32_t* seeds_sorted, int32_t* n_seeds);

}  // namespace orc
