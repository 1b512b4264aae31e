// TEST INFRASTRUCTURE ONLY -- declarations of the oracle's candidate stage
// (oracle_candidates.cpp) and of the marker record that identification reads.
#pragma once

#include <cstdint>
#include <vector>

#include "cctag_b200.h"
#include "oracle_geom.hpp"

namespace orc {

// EdgePointCollection (Types.hpp:19-158) of one pyramid level: the edge
// points, a dense W x H map from pixel to point, the links of the vote, the
// voter lists and the per-point flags the candidate stage sets.
struct EdgeCollection {
    int W = 0, H = 0;
    std::vector<int> map;  // point index of pixel (x, y) at y * W + x, -1 where there is none
    std::vector<int> x, y;
    std::vector<float> dx, dy, norm;  // EdgePoint::_grad, _normGrad
    std::vector<int> before, after;   // links of the vote, -1 where there is none
    std::vector<int> voff, vlist;     // voters of point i: vlist[voff[i], voff[i + 1])
    std::vector<float> flow;          // EdgePoint::_flowLength
    std::vector<uint8_t> processed_in, processed_aux;
    std::vector<uint64_t> processed;  // EdgePoint::_processed, one bit per ellipse-growing run
    std::vector<int> nSegmentOut;

    int at(int px, int py) const { return map[size_t(py) * size_t(W) + size_t(px)]; }
    int voters_size(int i) const { return voff[size_t(i) + 1] - voff[size_t(i)]; }
    // Fills the point arrays from raster-ordered edge points and resets the flags.
    void build(int w, int h, const int32_t* ex, const int32_t* ey, const int16_t* dxm, const int16_t* dym, int E,
               const int32_t* bef, const int32_t* aft, const int32_t* vo, const int32_t* vl, const float* fl);
};

// DirectedPoint2d
struct DPt {
    float x, y, dx, dy;
};

// The CCTag fields of a marker that the later stages read (CCTag.hpp).
struct Marker {
    float cx_img = 0, cy_img = 0;  // centerImg
    gm::Ellipse outer;             // _outerEllipse (center shifted by +0.5)
    gm::Ellipse rescaled;          // _rescaledOuterEllipse
    std::vector<std::vector<DPt>> points;
    std::vector<DPt> rescaled_points;
    int level = 0;
    float scale = 1.f;
    float quality = 0.f;
    int status = 0;
    int id = -1;
    float H[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
};

// The first maximumNbCandidatesLoopTwo loop-1 candidates of one level after
// the children collection and outlier removal of loop 2: seed, children count
// (0 when below minPointsSegmentCandidate), whether the candidate goes on to
// the ellipse growing, and its filtered children.
struct LoopTwoRecord {
    std::vector<int> seed, score, keep, foff{0}, flt;
};

// cctagDetectionFromEdges (Detection.cpp:568-693) on one level: markers are
// appended in candidate order.  With `rec`, the loop-two inputs are recorded
// and the stage stops there.
void candidates_from_edges(EdgeCollection& ec, const std::vector<int>& seeds, int level, float scale,
                           const cctagb_params& p, std::vector<Marker>& markers, LoopTwoRecord* rec);

// The level-0 re-fit of markers found on coarser levels (Multiresolution.cpp:
// 319-401); markers on level 0 take their outer points as they are.
void refit_on_level0(EdgeCollection& ec0, std::vector<Marker>& markers);

}  // namespace orc
