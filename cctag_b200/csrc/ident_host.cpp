// Identification, host part: outer-point subsampling, image cuts, cut
// selection with the sub-pixel outer edge refinement (Identification.cpp:
// 396-709, 1172-1301; geometry/Ellipse.cpp:259-300).  FP32 as the reference.
#include "ident_host.hpp"

#include <algorithm>
#include <cmath>
#include <map>

namespace cctagb {

namespace {

// Identification.hpp:197-219: bilinear sample, halved.
inline float bilinear(const uint8_t* img, int W, float x, float y)
{
    const int px = int(x), py = int(y);
    const uint8_t* p0 = img + px + size_t(py) * W;
    const float fx = x - float(px), fy = y - float(py);
    const float fx1 = 1.0f - fx, fy1 = 1.0f - fy;
    const float w1 = fx1 * fy1, w2 = fx * fy1, w3 = fx1 * fy, w4 = fx * fy;
    return (float(p0[0]) * w1 + float(p0[1]) * w2 + float(p0[W]) * w3 + float(p0[W + 1]) * w4) / 2;
}

// Identification.cpp:396-459 cutInterpolated: n samples from start+(stop-start)*begin
// to stop (end = 1); returns false (out of bounds) as soon as a sample leaves
// [1, W-1) x [1, H-1).
bool cut_interpolated(const uint8_t* img, int W, int H, float sx, float sy, float ex, float ey, float beginSig,
                      int n, float* sig)
{
    const float dX = ex - sx, dY = ey - sy;
    float xs = sx, ys = sy;
    if (beginSig != 0.f) {
        xs = sx + dX * beginSig;
        ys = sy + dY * beginSig;
    }
    const float stepX = (ex - xs) / (float(n) - 1.f);
    const float stepY = (ey - ys) / (float(n) - 1.f);
    float x = xs, y = ys;
    for (int i = 0; i < n; ++i) {
        if (x >= 1.f && x < float(W - 1) && y >= 1.f && y < float(H - 1)) {
            sig[i] = bilinear(img, W, x, y);
        } else {
            return false;
        }
        x += stepX;
        y += stepY;
    }
    return true;
}

// Boost.Accumulators immediate mean / variance (population), sample by
// sample: mean_n = (mean_{n-1} (n-1) + x) / n,
// var_n = var_{n-1} (n-1) / n + (x - mean_n)^2 / (n-1).
struct MeanVar {
    size_t n = 0;
    float mean = 0.f, var = 0.f;
    void add(float x)
    {
        ++n;
        mean = (mean * float(n - 1) + x) / float(n);
        if (n > 1) {
            const float t = x - mean;
            var = var * float(n - 1) / float(n) + t * t / float(n - 1);
        }
    }
};

// geometry/Ellipse.cpp:259-300
std::vector<DirPoint> sorted_outer_points(const geo::Ellipse& e, const std::vector<DirPoint>& pts, size_t requested)
{
    std::vector<std::pair<float, size_t>> ang;
    ang.reserve(pts.size());
    for (size_t i = 0; i < pts.size(); ++i) ang.emplace_back(std::atan2(pts[i].y - e.cy, pts[i].x - e.cx), i);
    std::sort(ang.begin(), ang.end());
    const size_t nOuter = std::min(requested, pts.size());
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

// Identification.cpp:659-709 convImageCut: 9-tap correlation with clamped
// borders, returns (max value, first location of the max).
std::pair<float, float> conv_cut(const float* k, const float* sig, int n)
{
    float best = 0.f;
    int loc = 0;
    for (int i = 0; i < n; ++i) {
        float t = 0;
        for (int j = 0; j < 9; ++j) {
            const int r = i - 4 + j;
            t += sig[r < 0 ? 0 : (r >= n ? n - 1 : r)] * k[j];
        }
        if (i == 0 || t > best) {
            best = t;
            loc = i;
        }
    }
    return {best, float(loc)};
}

// Identification.cpp:604-657 outerEdgeRefinement: moves the cut end to the
// strongest derivative response along the gradient, over 3*sqrt(2)*scale px.
bool outer_edge_refinement(DirPoint& stop, const uint8_t* img, int W, int H, float scale, int nRefine)
{
    const float len = 3.f * std::sqrt(2.f) * scale;
    const float hw = len / 2.f;
    const float gn = std::sqrt(stop.dx * stop.dx + stop.dy * stop.dy);
    const float gx = stop.dx / gn, gy = stop.dy / gn;
    const float ax = stop.x - hw * gx, ay = stop.y - hw * gy;
    const float bx = stop.x + hw * gx, by = stop.y + hw * gy;
    std::vector<float> sig(static_cast<size_t>(nRefine));
    if (!cut_interpolated(img, W, H, ax, ay, bx, by, 0.f, nRefine, sig.data())) return false;
    static const float kA[9] = {-0.0000f, -0.0003f, -0.1065f, -0.7863f, .0f, 0.7863f, 0.1065f, 0.0003f, 0.0000f};
    static const float kB[9] = {-0.0044f, -0.0540f, -0.2376f, -0.3450f, .0f, 0.3450f, 0.2376f, 0.0540f, 0.0044f};
    static const float kC[9] = {-0.0366f, -0.1113f, -0.1801f, -0.1594f, .0f, 0.1594f, 0.1801f, 0.1113f, 0.0366f};
    std::map<float, float> res;
    res.insert(conv_cut(kA, sig.data(), nRefine));
    res.insert(conv_cut(kB, sig.data(), nRefine));
    res.insert(conv_cut(kC, sig.data(), nRefine));
    const float maxLoc = res.rbegin()->second;
    const float step = len / (float(nRefine) - 1.f);
    stop.x = ax + step * maxLoc * gx;
    stop.y = ay + step * maxLoc * gy;
    return true;
}

}  // namespace

float begin_signal(int nCrowns)
{
    if (nCrowns == 3) return 1 - float(2 * nCrowns - 1) * 0.15f;
    if (nCrowns == 4) return 0.26f;
    return 0.f;
}

int identify_step1(const MarkerCand& m, const uint8_t* img, int W, int H, const cctagb_params& p, IdentTask& task)
{
    const geo::Ellipse& e = m.rescaled;
    const std::vector<DirPoint> outer = sorted_outer_points(e, m.rescaled_points, size_t(p.nSamplesOuterEllipse));
    if (outer.size() < 5) return CCTAGB_TOO_FEW_OUTER_POINTS;
    const float beginSig = begin_signal(p.nCrowns);
    const int n = std::min(p.sampleCutLength, kMaxSamples);
    // collectCuts (Identification.cpp:471-496)
    struct Cut {
        DirPoint stop;
        std::vector<float> sig;
    };
    std::vector<Cut> cuts;
    cuts.reserve(outer.size());
    std::vector<float> sig(static_cast<size_t>(n));
    for (const DirPoint& op : outer) {
        if (cut_interpolated(img, W, H, e.cx, e.cy, op.x, op.y, beginSig, n, sig.data())) cuts.push_back({op, sig});
    }
    if (cuts.empty()) return CCTAGB_NO_COLLECTED_CUTS;
    // selectCutCheapUniform (Identification.cpp:546-601)
    const size_t selectSize = std::min(size_t(std::min(p.numCutsInIdentStep, kMaxCuts)), cuts.size());
    std::vector<float> var;
    var.reserve(cuts.size());
    for (const Cut& c : cuts) {
        MeanVar mv;
        for (float v : c.sig) mv.add(v);
        var.push_back(mv.var);
    }
    const float varMax = *std::max_element(var.begin(), var.end());
    std::vector<size_t> keep;
    for (size_t i = 0; i < cuts.size(); ++i) {
        DirPoint& s = cuts[i].stop;
        float px, py;
        geo::point_on_ellipse(e, s.x, s.y, px, py);
        s.x = px;
        s.y = py;
        if (outer_edge_refinement(s, img, W, H, m.scale, p.numSamplesOuterEdgePointsRefinement))
            if (var[i] / varMax > 0.5f) keep.push_back(i);
    }
    const float step = std::max(1.f, float(keep.size()) / float(selectSize));
    int nsel = 0;
    for (size_t k = 0;; ++k) {
        const size_t i = size_t(float(k) * step);
        if (i < keep.size() && size_t(nsel) < selectSize) {
            task.stop[nsel][0] = cuts[keep[i]].stop.x;
            task.stop[nsel][1] = cuts[keep[i]].stop.y;
            ++nsel;
        } else {
            break;
        }
    }
    task.ncuts = nsel;
    if (nsel == 0) return CCTAGB_NO_SELECTED_CUTS;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) task.Q[r * 3 + c] = e.Q.m[r][c];
    task.cx = e.cx;
    task.cy = e.cy;
    task.a = e.a;
    task.b = e.b;
    task.angle = e.angle;
    task.x0 = m.cx_img;
    task.y0 = m.cy_img;
    task.roi[0] = 0;
    task.roi[1] = 0;
    task.roi[2] = W;
    task.roi[3] = H;
    return CCTAGB_ID_RELIABLE;
}

}  // namespace cctagb
