// Identification, host part: the outer points sorted by angle for the cut
// selection kernel (geometry/Ellipse.cpp:259-300), and the signal start.
#include "ident_host.hpp"

#include <algorithm>
#include <cmath>

namespace cctagb {

// geometry/Ellipse.cpp:259-300
std::vector<DirPoint> sorted_outer_points(const geo::Ellipse& e, const std::vector<DirPoint>& pts, size_t requested)
{
    std::vector<std::pair<float, size_t>> ang;
    ang.reserve(pts.size());
    // the correctly rounded float atan2 (pmath), as the GPU's sort
    for (size_t i = 0; i < pts.size(); ++i) ang.emplace_back(pm::atan2f_(pts[i].y - e.cy, pts[i].x - e.cx), i);
    std::sort(ang.begin(), ang.end());
    const size_t nOuter = std::min(requested, pts.size());
    // With one point the reference's step is a division by zero and the
    // index size_t(0 * inf) is undefined (on x86 it selects nothing); no cut
    // can come from fewer than two points, so nothing is selected.
    if (nOuter < 2) return {};
    const float step = std::max(1.f, float(pts.size()) / float(nOuter - 1));
    std::vector<DirPoint> res;
    res.reserve(nOuter);
    for (size_t k = 0;; ++k) {
        const size_t i = size_t(float(k) * step);
        if (i < ang.size()) res.push_back(pts[ang[i].second]);
        else break;
    }
    return res;
}

float begin_signal(int nCrowns)
{
    if (nCrowns == 3) return 1 - float(2 * nCrowns - 1) * 0.15f;
    if (nCrowns == 4) return 0.26f;
    return 0.f;
}

}  // namespace cctagb
