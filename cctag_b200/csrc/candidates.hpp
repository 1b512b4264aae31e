// Host candidate stage: seeds -> flow components -> outer ellipses -> marker
// candidates, and the level-0 re-fit of markers found on coarse levels
// (Detection.cpp:69-693, Vote.cpp:249-742, EllipseGrowing.cpp,
// Multiresolution.cpp:43-193,319-401 of the reference).
#pragma once

#include <cstdint>
#include <functional>
#include <vector>

#include "cctag_b200.h"
#include "geometry.hpp"

namespace cctagb {

// Host view of one level's edge-point collection (EdgePointCollection,
// Types.hpp:19-158) with the per-point state the candidate stage mutates.
struct EdgeSet {
    int W = 0, H = 0, E = 0;
    const int32_t* exy = nullptr;
    const int32_t* grad = nullptr;
    const int32_t* before = nullptr;
    const int32_t* after = nullptr;
    const int32_t* voff = nullptr;
    const int32_t* vlist = nullptr;
    const float* flow = nullptr;
    // Point index of a pixel: the points are in raster order, so a pixel's
    // index is its rank among the edge pixels.  bidx holds, per 32-pixel word
    // of each row (WW words per row), the word's edge pixels and the index of
    // its first one (the GPU's word + first-index plane, downloaded with the
    // points, or built by index_points): 1/16 of the bytes of a dense W x H
    // index map, so lookups stay in cache.
    struct Word {
        uint32_t bits;
        int32_t first;
    };
    const Word* bidx = nullptr;
    int WW = 0;
    std::vector<Word> own_bidx;  // index_points' copy

    std::vector<uint8_t> processed_in;  // loop 1 on the host
    std::vector<int32_t> n_segment_out;
    std::vector<uint32_t> link_stamp;  // edge linking: point visited in call `link_token`
    uint32_t link_token = 0;
    struct DfsFrame {  // one level of the ellipse-growing depth-first search
        int x, y, k;
    };

    int x(int i) const { return exy[i] & 0xffff; }
    int y(int i) const { return exy[i] >> 16; }
    float dx(int i) const { return float(int16_t(grad[i] & 0xffff)); }
    float dy(int i) const { return float(int16_t(grad[i] >> 16)); }
    float norm(int i) const { return std::sqrt(dx(i) * dx(i) + dy(i) * dy(i)); }
    int voters(int i) const { return voff[i + 1] - voff[i]; }
    int at(int px, int py) const
    {
        const Word w = bidx[size_t(py) * size_t(WW) + size_t(px >> 5)];
        const uint32_t bit = 1u << (px & 31);
        if (!(w.bits & bit)) return -1;
        const int i = w.first + __builtin_popcount(w.bits & (bit - 1u));
        return i < E ? i : -1;
    }
    // Builds bidx from exy[0, E) (own_bidx); throws unless the points are in
    // strict raster order.
    void index_points();
    void reset_state();
};

struct DirPoint {
    float x, y, dx, dy;
};

// A marker before identification (CCTag.hpp fields used downstream).
struct MarkerCand {
    float cx_img = 0, cy_img = 0;          // centerImg
    geo::Ellipse outer;                     // outer ellipse at its level (+0.5 shift)
    geo::Ellipse rescaled;                  // outer ellipse in level-0 pixels
    std::vector<std::vector<DirPoint>> points;
    std::vector<DirPoint> rescaled_points;  // outer points in level-0 pixels
    int level = 0;
    float scale = 1.f;
    float quality = 0.f;
    int status = 0;
    int id = -1;
    geo::Mat3 H = geo::Mat3::zero();
};

// One pyramid level's input to the candidate stage and its markers.
struct LevelJob {
    EdgeSet* es = nullptr;
    const std::vector<int32_t>* seeds = nullptr;  // processing order
    int level = 0;
    float scale = 1.f;
    std::vector<MarkerCand> out;
};

// Runs fn(i) for every i in [0, n), possibly concurrently; returns when all
// have finished.
using ParallelFor = std::function<void(int, const std::function<void(int)>&)>;

// One level's first maximumNbCandidatesLoopTwo loop-1 candidates (in loop-1
// order) after the children collection and LMedS outlier removal of loop 2
// (Detection.cpp:115-156): their seed, children count (score), whether they
// go on to the ellipse growing (keep), and their filtered children.
struct LoopTwoIn {
    std::vector<int32_t> seed, score;
    std::vector<float> flow;  // flow length of the seed (Vote.cpp:232)
    std::vector<uint8_t> keep;
    std::vector<int32_t> foff;  // candidate i: flt[foff[i], foff[i + 1]) (empty unless kept)
    std::vector<int32_t> flt;
    // flt[k]'s link chain: chain[k * chainLen + j], the point reached after
    // j + 1 alternating before / after links (before first), -1 past a
    // missing link; what addCandidateFlowtoCCTag walks (EllipseGrowing.cpp:63-178)
    std::vector<int32_t> chain;
    int chainLen = 0;
};

// Loop 1 and the outlier removal of loop 2 on the host, per level.
void link_and_filter(std::vector<LevelJob>& jobs, const cctagb_params& p, const ParallelFor& pf,
                     std::vector<LoopTwoIn>& out);

// Ellipse growing of one candidate done elsewhere (on the GPU): its level and
// filtered points in; its outer points, ellipse and status out (0 it leaves
// the list, 1 it stays, 2 not grown there: the host grows it).
struct GrowJob {
    int level = 0;
    const std::vector<int>* filtered = nullptr;
    std::vector<int>* outer = nullptr;
    geo::Ellipse* ellipse = nullptr;
    int status = 2;
};
using GrowFn = std::function<void(std::vector<GrowJob>&)>;

// Candidate markers of every level (cctagDetectionFromEdges, Detection.cpp:
// 568-693).  Loop 1 runs per level in seed order; loops 2 and 3 run per
// candidate (each with its own PCG32 stream, seed 271828), with the segment
// labels of loop 2 assigned in candidate order between them, so the result is
// the same for any ParallelFor.  With `given`, loop 1 and the outlier removal
// are taken from it (computed on the GPU) instead of being run here; with
// `grow`, the ellipse growing of the candidates goes to it.
// `grown` (optional) receives the candidates grown by `grow` and by the host.
void detect_from_edges(std::vector<LevelJob>& jobs, const cctagb_params& p, const ParallelFor& pf,
                       const std::vector<LoopTwoIn>* given = nullptr, const GrowFn* grow = nullptr,
                       int* grown = nullptr);

// Level-0 re-fit of markers detected on coarser levels (Multiresolution.cpp:
// 319-401), markers in parallel, each with its own PCG32 stream.
void refit_on_level0(EdgeSet& es0, std::vector<MarkerCand>& markers, const ParallelFor& pf);

// Pieces of the re-fit: the hull of a coarse-level marker (Multiresolution.cpp:
// 331-336: conics of its inner and outer ellipse, the inner center for the
// gradient test, the rescaled center row) ...
struct RefitHull {
    float qin[9], qout[9];
    float inCx, inCy, yc;
};
void refit_hull(const MarkerCand& m, RefitHull& h);
// ... the random stream of marker mi's outlier removal ...
inline geo::Pcg32 refit_rng(int mi) { return geo::Pcg32(271828, (uint64_t(1) << 62) | uint64_t(mi)); }
// ... and the ellipse fit to the filtered hull points (Multiresolution.cpp:
// 360-401), which updates the marker when n >= 5 and the fit succeeds.
void refit_apply(const EdgeSet& es0, MarkerCand& m, const int32_t* filtered, size_t n);

}  // namespace cctagb
