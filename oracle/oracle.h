// TEST INFRASTRUCTURE ONLY -- C entry points of the CPU oracle (see the
// headers of oracle_image.cpp and oracle_ident.cpp).  Only the test-suite,
// `__graft_entry__.smoke()` and the CPU-baseline leg of `bench.py` load it.
#pragma once
#include <stdint.h>

#include "cctag_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int distSearch;
    int thrGradientMagInVote;
    float angleVoting;
    float ratioVoting;
    int nCrowns;
    int minVotesToSelectCandidate;
} orc_vote_params;

void orc_pyramid_down(const uint8_t* src, int sw, int sh, uint8_t* dst, int dw, int dh);
void orc_derivatives(const uint8_t* src, int W, int H, int16_t* dx, int16_t* dy);
void orc_canny(const int16_t* dx, const int16_t* dy, int W, int H, float thrLow, float thrHigh, uint8_t* edges,
               uint8_t* nms_map);
void orc_thin_lut(int pass, uint8_t* lut);
void orc_thin(uint8_t* edges, int W, int H);
int orc_vote(const uint8_t* edges, const int16_t* dx, const int16_t* dy, int W, int H, const orc_vote_params* p,
             int cap, int32_t* ex, int32_t* ey, int32_t* before, int32_t* after, int32_t* chosen, float* total,
             int32_t* nvotes, int32_t* is_max, float* flow_length, int32_t* voter_off, int32_t* voter_list,
             int32_t* seeds_push, int32_t* seeds_sorted, int32_t* n_seeds);
void orc_level(const uint8_t* src, int W, int H, float thrLow, float thrHigh, int16_t* dx, int16_t* dy,
               uint8_t* edges);

typedef struct {
    int id, status;
    float x, y;                  /* imaged center */
    float cx, cy, a, b, angle;   /* outer ellipse, level-0 pixels */
    float quality;
    int level;
} orc_marker;

/* Whole detection on the CPU; fp64 != 0 runs the center refinement in FP64.
 * Returns the number of markers (all written when <= cap). */
int orc_detect(const uint8_t* gray, int W, int H, const cctagb_params* p, int fp64, orc_marker* out, int cap);

#ifdef __cplusplus
}
#endif
