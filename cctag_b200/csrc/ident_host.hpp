// Identification, host part: cut collection and selection (identify_step_1,
// Identification.cpp:1172-1301) and the record handed to the GPU kernel.
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "candidates.hpp"

namespace cctagb {

constexpr int kMaxCuts = 32;
constexpr int kMaxSamples = 128;
constexpr int kMaxBankIds = 128;
constexpr int kMaxBankRatios = 8;

// One marker to identify on the GPU.
struct IdentTask {
    float Q[9];                // outer ellipse conic, row-major (level-0 pixels)
    float cx, cy, a, b, angle; // its parameters
    float x0, y0;              // initial imaged center (centerImg)
    int ncuts;
    float stop[kMaxCuts][2];   // selected cut end points (refined outer edge)
};

struct IdentResult {
    int status;        // CCTAGB_ID_RELIABLE, CCTAGB_OPTI_HAS_DIVERGED, CCTAGB_ID_NOT_RELIABLE
    int id;
    float x, y;        // refined imaged center
    float H[9];        // marker plane -> image, row-major
    float residual;    // normalised residual (sqrt(cost) / barcode range)
    float score;       // mean identification probability of the winning id
    int nvalid;        // cuts inside the image at the end
    int pad;
};

struct IdentParams {
    int nSamples;           // sampleCutLength (<= kMaxSamples)
    float beginSig;         // 1 - (2 nCrowns - 1) * 0.15 for 3 crowns
    float neighbourSize;    // imagedCenterNeighbourSize
    int gridN;              // imagedCenterNGridSample (3 or 5)
    float minIdentProba;
    int nIds, nRatios;      // bank shape
    int refineMode;         // CCTAGB_REFINE_GRID / CCTAGB_REFINE_GAUSS_NEWTON
    int gnIterations;
};

// Cut selection of one marker (identify_step_1).  Returns the marker status
// (CCTAGB_ID_RELIABLE when cuts were selected) and fills `task`.
int identify_step1(const MarkerCand& m, const uint8_t* img, int W, int H, const cctagb_params& p, IdentTask& task);

// Signal start along the cut as a fraction of the unit radius.
float begin_signal(int nCrowns);

// Device side (identify.cu).  The bank lives in a device buffer of
// kMaxBankIds x kMaxBankRatios floats (1 / ratio) owned by the caller.
void upload_bank(const std::vector<std::vector<float>>& bank, float* d_bank_inv);
void launch_identify(const uint8_t* d_img, int W, int H, const IdentTask* d_tasks, IdentResult* d_res, int n,
                     const float* d_bank_inv, const IdentParams& ip, cudaStream_t s);

}  // namespace cctagb
