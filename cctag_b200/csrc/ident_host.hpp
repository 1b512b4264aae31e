// Identification, host part: cut collection and selection (identify_step_1,
// Identification.cpp:1172-1301) and the record handed to the GPU kernel.
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "candidates.hpp"

namespace cctagb {

constexpr int kMaxCuts = CCTAGB_MAX_CUTS;
constexpr int kMaxSamples = 128;
constexpr int kMaxBankIds = 128;
constexpr int kMaxBankRatios = 8;

// One marker to identify on the GPU (the ABI's cctagb_cut_task) and its
// result (cctagb_ident_result).
using IdentTask = cctagb_cut_task;
using IdentResult = cctagb_ident_result;

struct IdentParams {
    int nSamples;           // sampleCutLength (<= kMaxSamples)
    float beginSig;         // 1 - (2 nCrowns - 1) * 0.15 for 3 crowns
    float neighbourSize;    // imagedCenterNeighbourSize
    int gridN;              // imagedCenterNGridSample (3 or 5)
    float minIdentProba;
    int nIds, nRatios;      // bank shape
    int refineMode;         // CCTAGB_REFINE_GRID / CCTAGB_REFINE_GAUSS_NEWTON
    int gnIterations;       // Gauss-Newton cost evaluations at most
    int coarseRounds;       // grid rounds before Gauss-Newton
    int layout;             // CCTAGB_IDENT_AUTO / CCTAGB_IDENT_BLOCK
};

constexpr int kMaxOuterPoints = 256;    // outer points per marker (nSamplesOuterEllipse)
constexpr int kMaxRefineSamples = 64;   // numSamplesOuterEdgePointsRefinement

// Cut selection of one marker on the GPU (k_cut_select): its level-0 outer
// ellipse and its outer points, which the kernel sorts by angle and
// subsamples (getSortedOuterPoints) unless the host already did
// (`presorted`: more points than the kernel sorts in shared memory).
constexpr int kCutSortCap = 4096;
struct CutSelectIn {
    float cx, cy, a, b;     // the ellipse (cuts start at its center)
    float cosA, sinA;       // cos / sin of its angle, computed on the host
    float scale;            // the marker's pyramid scale (refinement length)
    int first, count;       // its outer points in the point array
    int presorted;          // 1: the points are the sorted selection
};

struct CutSelectParams {
    float beginSig;
    int nSamples;           // sampleCutLength
    int nRefine;            // numSamplesOuterEdgePointsRefinement
    int maxSelect;          // min(numCutsInIdentStep, kMaxCuts)
    int nOuter;             // nSamplesOuterEllipse (<= kMaxOuterPoints)
};

// geometry/Ellipse.cpp:259-300: up to `requested` outer points, sorted by the
// angle around the ellipse center, uniformly subsampled.
std::vector<DirPoint> sorted_outer_points(const geo::Ellipse& e, const std::vector<DirPoint>& pts, size_t requested);

// Writes stop[] and ncuts of tasks[i] (the rest filled by the host) and
// status[i] (CCTAGB_ID_RELIABLE, _TOO_FEW_OUTER_POINTS, _NO_COLLECTED_CUTS or
// _NO_SELECTED_CUTS).
void launch_cut_select(const uint8_t* d_img, int W, int H, const CutSelectIn* d_ins, const DirPoint* d_pts,
                       const int16_t* d_sel, const int* d_nsel, IdentTask* d_tasks, int* d_status, int n,
                       const CutSelectParams& cp, cudaStream_t s);
// The outer points of each marker sorted by angle and subsampled to at most
// nOuterReq (k_outer_select): sel[i * kMaxOuterPoints + k] is the k-th
// selected point of marker i (relative to its first), nsel[i] their number.
void launch_outer_select(const CutSelectIn* d_ins, const DirPoint* d_pts, int nOuterReq, int16_t* d_sel, int* d_nsel,
                         int n, cudaStream_t s);

// Signal start along the cut as a fraction of the unit radius.
float begin_signal(int nCrowns);

// Device side (identify.cu).  The bank lives in a device buffer of
// kMaxBankIds x kMaxBankRatios floats (1 / ratio) owned by the caller.
void upload_bank(const std::vector<std::vector<float>>& bank, float* d_bank_inv);
// Tasks carry their image rectangle; d_img rows are pitch bytes apart.
void launch_identify(const uint8_t* d_img, size_t pitch, const IdentTask* d_tasks, IdentResult* d_res, int n,
                     const float* d_bank_inv, const IdentParams& ip, cudaStream_t s);
// Cost and adjoints at given centers (cctagb_cut_cost): out is 12 floats per
// task (cost, d/dcenter x2, d/dH x9).
// fp64: every step in double precision (the check form of the adjoint).
void launch_cut_cost(const uint8_t* d_img, size_t pitch, const IdentTask* d_tasks, const float* d_centers,
                     float* d_out, int n, const IdentParams& ip, cudaStream_t s, bool fp64 = false);

}  // namespace cctagb
