// TEST INFRASTRUCTURE ONLY -- CPU oracle of the candidate stage: seeds ->
// convex edge segments -> flow components -> outer ellipses -> markers, and
// the level-0 re-fit of markers found on coarse levels.
//
// Restated from the reference, in its own order of operations and with its
// own data structures (lists, a set of visited pixels, a recursive depth-first
// growth, full sorts for the medians), separately from the library's candidate
// stage:
//   Detection.cpp:69-113   constructFlowComponentFromSeed (loop 1)
//   Detection.cpp:115-267  completeFlowComponent (loop 2)
//   Detection.cpp:278-377  flowComponentAssembling
//   Detection.cpp:379-566  cctagDetectionFromEdgesLoopTwoIteration (loop 3)
//   Detection.cpp:568-693  cctagDetectionFromEdges
//   Vote.cpp:255-742       edgeLinking, edgeLinkingDir, childrenOf,
//                          outlierRemoval, isAnotherSegment
//   EllipseGrowing.cpp:63-551  addCandidateFlowtoCCTag, ellipseGrowingInit,
//                          connectedPoint, ellipseHull, ellipseGrowing2
//   Fitting.cpp:213-292    innerProdMin
//   Multiresolution.cpp:43-170, 319-401  intersectLineToTwoEllipses,
//                          selectEdgePointInEllipticHull, the re-fit.
//
// Determinism choices (the reference runs these loops with TBB over shared
// flags and one thread-local generator, so its output depends on the thread
// schedule): loop 1 runs in seed order (the reference's CCTAG_SERIALIZE
// order); loops 2 and 3 and the re-fit run candidate by candidate, each
// drawing from its own PCG32 stream (gm::candidate_stream / refit_stream);
// loop-two candidates keep their loop-one order.  Two guards where the
// reference cannot finish: the LMedS draws are capped at 7000, and
// isAnotherSegment needs 5 points on each side (rand_5_k would never return).
// A missing vote link in addCandidateFlowtoCCTag (the reference dereferences a
// null point) drops the candidate.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <deque>
#include <limits>
#include <list>
#include <set>
#include <stdexcept>
#include <vector>

#include "oracle_cand.hpp"

namespace orc {

using gm::Ellipse;
using gm::P2;

void EdgeCollection::build(int w, int h, const int32_t* ex, const int32_t* ey, const int16_t* dxm, const int16_t* dym,
                           int E, const int32_t* bef, const int32_t* aft, const int32_t* vo, const int32_t* vl,
                           const float* fl)
{
    W = w;
    H = h;
    map.assign(size_t(w) * size_t(h), -1);
    x.assign(ex, ex + E);
    y.assign(ey, ey + E);
    dx.resize(size_t(E));
    dy.resize(size_t(E));
    norm.resize(size_t(E));
    for (int i = 0; i < E; ++i) {
        const size_t q = size_t(ey[i]) * size_t(w) + size_t(ex[i]);
        map[q] = i;
        dx[size_t(i)] = float(dxm[q]);
        dy[size_t(i)] = float(dym[q]);
        norm[size_t(i)] = std::sqrt(dx[size_t(i)] * dx[size_t(i)] + dy[size_t(i)] * dy[size_t(i)]);
    }
    before.assign(bef, bef + E);
    after.assign(aft, aft + E);
    voff.assign(vo, vo + E + 1);
    vlist.assign(vl, vl + vo[E]);
    flow.assign(fl, fl + E);
    processed_in.assign(size_t(E), 0);
    processed_aux.assign(size_t(E), 0);
    processed.assign(size_t(E), 0);
    nSegmentOut.assign(size_t(E), -1);
}

namespace {

constexpr int kEdgeNotFound = -1;
constexpr int kConvexityLost = -2;

struct Candidate {
    int seed = -1;
    std::list<int> convexEdgeSegment;
    std::vector<int> outerEllipsePoints;
    Ellipse outerEllipse;
    std::vector<int> filteredChildren;
    int score = 0;
    size_t nLabel = 0;
    float averageReceivedVote = 0.f;
};

unsigned packxy(int x, int y) { return (unsigned(x) << 16) | (unsigned(y) & 0xFFFFu); }

P2 pt(const EdgeCollection& ec, int e) { return {float(ec.x[size_t(e)]), float(ec.y[size_t(e)])}; }

// Vote.cpp:272-394
void edge_linking_dir(EdgeCollection& ec, std::set<unsigned>& processed, int p, int dir, std::list<int>& seg,
                      size_t windowSize, float averageVoteMin)
{
    std::deque<float> phi;
    size_t i = 0;
    bool found = true;
    int stop = 0;
    const size_t maxLength = 100;
    float averageVote = float(ec.voters_size(p));
    while (i < maxLength && found && averageVote >= averageVoteMin) {
        const float angle =
            std::fmod(gm::atan2_cr(ec.dy[size_t(p)], ec.dx[size_t(p)]) + 2.0f * gm::kPi, 2.0f * gm::kPi);
        phi.push_back(angle);
        if (phi.size() > windowSize) phi.pop_front();
        const int shifting = int(std::round(((angle + gm::kPi / 4.0f) / (2.0f * gm::kPi)) * 8.0f)) - 1;
        static const int xoff[] = {1, 1, 0, -1, -1, -1, 0, 1};
        const int yoff[] = {0, dir * -1, dir * -1, dir * -1, 0, dir * 1, dir * 1, dir * 1};
        int j = 0;
        stop = 0;
        while (!stop) {
            if (j >= 8) {
                stop = kEdgeNotFound;
            } else {
                int sx, sy;
                if (dir == 1) {
                    sx = ec.x[size_t(p)] + xoff[(8 - shifting + j) % 8];
                    sy = ec.y[size_t(p)] + yoff[(8 - shifting + j) % 8];
                } else {
                    sx = ec.x[size_t(p)] + xoff[(shifting + j) % 8];
                    sy = ec.y[size_t(p)] + yoff[(shifting + j) % 8];
                }
                if (sx >= 0 && sx < ec.W && sy >= 0 && sy < ec.H && ec.at(sx, sy) >= 0 &&
                    processed.find(packxy(sx, sy)) == processed.end()) {
                    if (phi.size() == windowSize) {
                        if (float(dir) * gm::sin_cr(phi.back() - phi.front()) < 0.0f) stop = kConvexityLost;
                    } else {
                        const float s = float(dir) * gm::sin_cr(phi.back() - phi.front());
                        const float c = gm::cos_cr(phi.back() - phi.front());
                        if ((s < -0.707f && c > 0.f) || (s < 0.f && c < 0.f)) stop = kConvexityLost;
                    }
                    if (stop == 0) {
                        processed.insert(packxy(ec.x[size_t(p)], ec.y[size_t(p)]));
                        p = ec.at(sx, sy);
                        if (dir > 0) seg.push_back(p);
                        else seg.push_front(p);
                        averageVote = (averageVote * float(seg.size()) + float(ec.voters_size(p))) /
                                      (float(seg.size()) + 1.f);
                        stop = 1;
                    }
                    processed.insert(packxy(ec.x[size_t(p)], ec.y[size_t(p)]));
                }
            }
            ++j;
        }
        found = stop == 1;
        ++i;
    }
    if (i == maxLength || stop == kConvexityLost) {
        if (seg.size() > windowSize) {
            size_t n = 0;
            for (int q : seg) {
                if (n == seg.size() - windowSize) break;
                ec.processed_in[size_t(q)] = 1;
                ++n;
            }
        }
    } else if (stop == kEdgeNotFound) {
        for (int q : seg) ec.processed_in[size_t(q)] = 1;
    }
}

// Vote.cpp:255-270
void edge_linking(EdgeCollection& ec, std::list<int>& seg, int pmax, size_t windowSize, float averageVoteMin)
{
    std::set<unsigned> processed;
    seg.push_back(pmax);
    ec.processed_in[size_t(pmax)] = 1;
    processed.insert(packxy(ec.x[size_t(pmax)], ec.y[size_t(pmax)]));
    edge_linking_dir(ec, processed, pmax, 1, seg, windowSize, averageVoteMin);
    edge_linking_dir(ec, processed, pmax, -1, seg, windowSize, averageVoteMin);
}

// Vote.cpp:396-412
void children_of(const EdgeCollection& ec, const std::list<int>& edges, std::list<int>& children)
{
    size_t voteMax = 1;
    for (int e : edges) voteMax = size_t(std::max(int(voteMax), ec.voters_size(e)));
    for (int e : edges) {
        const int first = ec.voff[size_t(e)], last = ec.voff[size_t(e) + 1];
        if (last > first && size_t(last - first) >= voteMax / 14)
            for (int k = first; k < last; ++k) children.push_back(ec.vlist[size_t(k)]);
    }
}

std::vector<float> distances(const Ellipse& q, const std::vector<P2>& pts)
{
    std::vector<float> d;
    d.reserve(pts.size());
    for (const P2& p : pts) d.push_back(gm::distance_point_ellipse(q.Q, p.x, p.y));
    return d;
}

enum { NO_WEIGHT = 0, INV_GRAD_WEIGHT = 1 };

// Vote.cpp:414-576 outlierRemoval
void outlier_removal(const EdgeCollection& ec, const std::list<int>& children, std::vector<int>& filteredChildren,
                     float& SmFinal, float threshold, int weightedType, size_t maxSize, gm::Pcg& rng)
{
    filteredChildren.reserve(children.size());
    const size_t nSubsampleSize = std::min(children.size(), maxSize);
    const float step = float(children.size()) / float(nSubsampleSize);
    if (nSubsampleSize < 5) return;
    Ellipse qm;
    float Sm = 10000000.0f;
    std::vector<P2> pts;
    std::vector<float> weights;
    size_t k = 0, iEdgePoint = 0;
    for (int e : children) {
        if (iEdgePoint == size_t(float(k) * step)) {
            ++k;
            pts.push_back(pt(ec, e));
            if (weightedType == INV_GRAD_WEIGHT) weights.push_back(255 / ec.norm[size_t(e)]);
        }
        ++iEdgePoint;
    }
    size_t counter = 0, draws = 0;
    int perm[5];
    while (counter < 70 && draws < 7000) {
        ++draws;
        gm::rand_5_k(perm, pts.size(), rng);
        double A[5][5], b[5], temp[5];
        for (int i = 0; i < 5; ++i) {
            const double px = pts[size_t(perm[i])].x, py = pts[size_t(perm[i])].y;
            A[i][0] = px * px;
            A[i][1] = 2.0 * px * py;
            A[i][2] = py * py;
            A[i][3] = 2.0 * px;
            A[i][4] = 2.0 * py;
            b[i] = -1.0;
        }
        if (!gm::solve_5x5(A, b, temp)) {  // A.determinant() == 0
            ++counter;
            continue;
        }
        const float t0 = float(temp[0]), t1 = float(temp[1]), t2 = float(temp[2]), t3 = float(temp[3]),
                    t4 = float(temp[4]);
        if (!(t0 * t2 - t1 * t1 > 0)) {
            ++counter;
            continue;
        }
        gm::M3 Q = gm::m3_zero();
        Q.v[0][0] = t0;
        Q.v[0][1] = Q.v[1][0] = t1;
        Q.v[0][2] = Q.v[2][0] = t3;
        Q.v[1][1] = t2;
        Q.v[1][2] = Q.v[2][1] = t4;
        Q.v[2][2] = 1.f;
        try {
            const Ellipse q = gm::ellipse_from_matrix(Q);
            const float ratioSemiAxes = q.a / q.b;
            if (ratioSemiAxes < 0.04f || ratioSemiAxes > 25) {
                ++counter;
                continue;
            }
            std::vector<float> dist = distances(q, pts);
            if (weightedType != NO_WEIGHT)
                for (size_t i = 0; i < dist.size(); ++i) dist[i] = dist[i] * weights[i];
            const float S = gm::median_ref(dist);
            if (S < Sm) {
                counter = 0;
                qm = gm::ellipse_from_matrix(Q);
                Sm = S;
            } else {
                ++counter;
            }
        } catch (...) {
        }
    }
    std::vector<float> vDistFinal;
    for (int e : children) {
        float distFinal = std::numeric_limits<float>::max();
        const P2 q = pt(ec, e);
        if (weightedType == NO_WEIGHT) distFinal = gm::distance_point_ellipse(qm.Q, q.x, q.y);
        else distFinal = gm::distance_point_ellipse(qm.Q, q.x, q.y) * 255 / ec.norm[size_t(e)];
        if (distFinal < threshold * Sm) {
            filteredChildren.push_back(e);
            vDistFinal.push_back(distFinal);
        }
    }
    if (vDistFinal.empty()) return;
    SmFinal = gm::median_ref(vDistFinal);
}

std::vector<P2> points_of(const EdgeCollection& ec, const std::vector<int>& idx)
{
    std::vector<P2> v;
    v.reserve(idx.size());
    for (int e : idx) v.push_back(pt(ec, e));
    return v;
}

// numerical::ellipseFitting / circleFitting on edge points
Ellipse ellipse_fitting(const EdgeCollection& ec, const std::vector<int>& idx)
{
    return gm::fit_ellipse(points_of(ec, idx));
}
Ellipse circle_fitting(const EdgeCollection& ec, const std::vector<int>& idx)
{
    return gm::fit_circle(points_of(ec, idx));
}

// Fitting.cpp:213-292 innerProdMin (only its return value is used)
float inner_prod_min(const EdgeCollection& ec, const std::vector<int>& fc, float thrCosDiffMax)
{
    float mn = 1.1f;
    int pAngle1 = -1;
    const int p0 = fc.front();
    float normGrad = std::sqrt(ec.dx[size_t(p0)] * ec.dx[size_t(p0)] + ec.dy[size_t(p0)] * ec.dy[size_t(p0)]);
    const float gx0 = ec.dx[size_t(p0)] / normGrad;
    const float gy0 = ec.dy[size_t(p0)] / normGrad;
    for (size_t i = 1; i < fc.size(); ++i) {
        const int c = fc[i];
        normGrad = std::sqrt(ec.dx[size_t(c)] * ec.dx[size_t(c)] + ec.dy[size_t(c)] * ec.dy[size_t(c)]);
        const float gx = ec.dx[size_t(c)] / normGrad, gy = ec.dy[size_t(c)] / normGrad;
        const float innerProd = gx0 * gx + gy0 * gy;
        if (innerProd <= thrCosDiffMax) return innerProd;
        if (innerProd < mn) {
            mn = innerProd;
            pAngle1 = c;
        }
    }
    normGrad = std::sqrt(ec.dx[size_t(pAngle1)] * ec.dx[size_t(pAngle1)] +
                         ec.dy[size_t(pAngle1)] * ec.dy[size_t(pAngle1)]);
    const float gxmin = ec.dx[size_t(pAngle1)] / normGrad, gymin = ec.dy[size_t(pAngle1)] / normGrad;
    mn = 1.f;
    for (int c : fc) {
        normGrad = std::sqrt(ec.dx[size_t(c)] * ec.dx[size_t(c)] + ec.dy[size_t(c)] * ec.dy[size_t(c)]);
        const float chgx = ec.dx[size_t(c)] / normGrad, chgy = ec.dy[size_t(c)] / normGrad;
        const float innerProd = gxmin * chgx + gymin * chgy;
        if (innerProd <= thrCosDiffMax) return innerProd;
        if (innerProd < mn) mn = innerProd;
    }
    return mn;
}

// EllipseGrowing.cpp:345-376 isGoodEGPoints + ellipseGrowingInit
bool ellipse_growing_init(const EdgeCollection& ec, const std::vector<int>& fc, Ellipse& e)
{
    if (inner_prod_min(ec, fc, 0.25f) <= 0.25f) {
        e = ellipse_fitting(ec, fc);
        return true;
    }
    e = circle_fitting(ec, fc);
    return false;
}

// EllipseGrowing.cpp:378-422 connectedPoint (recursive, as the reference)
void connected_point(std::vector<int>& pts, int runId, EdgeCollection& ec, const Ellipse& qIn, const Ellipse& qOut,
                     int x, int y)
{
    const uint64_t threadMask = uint64_t(1) << runId;
    ec.processed[size_t(ec.at(x, y))] |= threadMask;
    static const int xoff[] = {1, 1, 0, -1, -1, -1, 0, 1};
    static const int yoff[] = {0, -1, -1, -1, 0, 1, 1, 1};
    for (int i = 0; i < 8; ++i) {
        const int sx = x + xoff[i], sy = y + yoff[i];
        if (sx >= 0 && sx < ec.W && sy >= 0 && sy < ec.H) {
            const int e = ec.at(sx, sy);
            if (e >= 0 && gm::is_in_hull(qIn, qOut, float(ec.x[size_t(e)]), float(ec.y[size_t(e)])) &&
                !(ec.processed[size_t(e)] & threadMask)) {
                const float gx = ec.dx[size_t(e)], gy = ec.dy[size_t(e)];
                const float ox = qIn.cx - float(ec.x[size_t(e)]), oy = qIn.cy - float(ec.y[size_t(e)]);
                if (gx * ox + gy * oy < 0) {
                    pts.push_back(e);
                    ec.processed[size_t(e)] |= threadMask;
                    connected_point(pts, runId, ec, qIn, qOut, sx, sy);
                }
            }
        }
    }
}

// EllipseGrowing.cpp:443-457
void ellipse_hull(EdgeCollection& ec, std::vector<int>& pts, const Ellipse& ellipse, float delta, int runId)
{
    Ellipse qIn, qOut;
    gm::compute_hull(ellipse, delta, qIn, qOut);
    const size_t initSize = pts.size();
    for (size_t i = 0; i < initSize; ++i) {
        const int e = pts[i];
        connected_point(pts, runId, ec, qIn, qOut, ec.x[size_t(e)], ec.y[size_t(e)]);
    }
}

int count_in_hull(const EdgeCollection& ec, const std::vector<int>& pts, const Ellipse& ellipse, float width)
{
    Ellipse qIn, qOut;
    gm::compute_hull(ellipse, width, qIn, qOut);
    int n = 0;
    for (int e : pts)
        if (gm::is_in_hull(qIn, qOut, float(ec.x[size_t(e)]), float(ec.y[size_t(e)]))) ++n;
    return n;
}

// EllipseGrowing.cpp:459-551 ellipseGrowing2
void ellipse_growing2(EdgeCollection& ec, const std::vector<int>& filteredChildren, std::vector<int>& outer,
                      Ellipse& ellipse, float width, int runId, bool goodInit)
{
    const uint64_t threadMask = uint64_t(1) << runId;
    for (int c : filteredChildren) {
        outer.push_back(c);
        ec.processed[size_t(c)] |= threadMask;
    }
    int lastSizePoints = 0;
    if (!goodInit) {
        int newSizePoints = int(outer.size());
        int maxNbPoints = newSizePoints;
        int nIterMax = 0, nIter = 0;
        std::vector<std::vector<int>> edgePointsSets{outer};
        std::vector<Ellipse> ellipsesSets{ellipse};
        ++nIter;
        while (newSizePoints - lastSizePoints > 0) {
            lastSizePoints = count_in_hull(ec, outer, ellipse, width);
            ellipse_hull(ec, outer, ellipse, width, runId);
            edgePointsSets.push_back(outer);
            ellipsesSets.push_back(ellipse);
            ellipse = circle_fitting(ec, outer);
            newSizePoints = count_in_hull(ec, outer, ellipse, width);
            if (newSizePoints > maxNbPoints) {
                maxNbPoints = newSizePoints;
                nIterMax = nIter;
            }
            ++nIter;
        }
        outer = edgePointsSets[size_t(nIterMax)];
        ellipse = ellipsesSets[size_t(nIterMax)];
        for (auto& v : edgePointsSets)
            for (int e : v) ec.processed[size_t(e)] &= ~threadMask;
        for (int e : outer) ec.processed[size_t(e)] |= threadMask;
    }
    ellipse = ellipse_fitting(ec, outer);
    size_t last = 0;
    while (outer.size() > last) {
        last = outer.size();
        ellipse_hull(ec, outer, ellipse, width, runId);
        ellipse = ellipse_fitting(ec, outer);
    }
}

float perimeter_quality(size_t n, const Ellipse& e) { return float(n) / float(gm::rasterize_perimeter(e)); }

// Detection.cpp:115-267 completeFlowComponent.  Returns whether the candidate
// enters the loop-two list; `filtered_ok` tells whether it reached the
// ellipse growing (>= 5 filtered children).
bool complete_flow_component(Candidate& c, EdgeCollection& ec, size_t& nSegmentOut, int runId,
                             const cctagb_params& p, gm::Pcg& rng, bool stop_after_filter, bool& filtered_ok)
{
    filtered_ok = false;
    try {
        std::list<int> children;
        children_of(ec, c.convexEdgeSegment, children);
        if (children.size() < size_t(p.minPointsSegmentCandidate)) return false;
        c.score = int(children.size());
        float SmFinal = 1e+10f;
        outlier_removal(ec, children, c.filteredChildren, SmFinal, p.threshRobustEstimationOfOuterEllipse,
                        INV_GRAD_WEIGHT, 60, rng);
        if (c.filteredChildren.size() < 5) return false;
        filtered_ok = true;
        if (stop_after_filter) return false;
        size_t nLabel;
        {
            long nSegmentCommon = -1;
            for (int e : c.filteredChildren)
                if (ec.nSegmentOut[size_t(e)] != -1) {
                    nSegmentCommon = ec.nSegmentOut[size_t(e)];
                    break;
                }
            if (nSegmentCommon == -1) nLabel = nSegmentOut++;
            else nLabel = size_t(nSegmentCommon);
            for (int e : c.filteredChildren) ec.nSegmentOut[size_t(e)] = int(nLabel);
        }
        const bool goodInit = ellipse_growing_init(ec, c.filteredChildren, c.outerEllipse);
        ellipse_growing2(ec, c.filteredChildren, c.outerEllipsePoints, c.outerEllipse,
                         p.ellipseGrowingEllipticHullWidth, runId, goodInit);
        c.nLabel = nLabel;
        std::vector<float> vDistFinal;
        for (int e : c.outerEllipsePoints) {
            const P2 q = pt(ec, e);
            vDistFinal.push_back(gm::distance_point_ellipse(c.outerEllipse.Q, q.x, q.y));
        }
        SmFinal = gm::median_ref(vDistFinal);
        if (SmFinal > p.thrMedianDistanceEllipse) return false;
        const float quality = perimeter_quality(c.outerEllipsePoints.size(), c.outerEllipse);
        if (quality > 1.1) return false;
        const float ratioSemiAxes = c.outerEllipse.a / c.outerEllipse.b;
        if (ratioSemiAxes < 0.05 || ratioSemiAxes > 20) return false;
        return true;
    } catch (...) {
        return false;
    }
}

bool is_on_the_same_side(float x1, float y1, float x2, float y2, const float line[3])
{
    const float s1 = x1 * line[0] + y1 * line[1] + line[2];
    const float s2 = x2 * line[0] + y2 * line[1] + line[2];
    return s1 * s2 > 0;
}

// EllipseGrowing.cpp:63-178 addCandidateFlowtoCCTag
bool add_candidate_flow(EdgeCollection& ec, const std::vector<int>& filteredChildren,
                        const std::vector<int>& outerEllipsePoints, const Ellipse& outerEllipse,
                        std::vector<std::vector<DPt>>& cctagPoints, size_t numCircles)
{
    cctagPoints.resize(numCircles);
    for (int e : outerEllipsePoints)
        cctagPoints.back().push_back(
            {float(ec.x[size_t(e)]), float(ec.y[size_t(e)]), ec.dx[size_t(e)], ec.dy[size_t(e)]});
    std::list<int> vProcessedEdgePoint;
    auto release = [&]() {
        for (int e : vProcessedEdgePoint) ec.processed_aux[size_t(e)] = 0;
    };
    size_t nGradientOut = 0, nAddedPoint = 0;
    for (int child : filteredChildren) {
        int dir = -1;
        int p = child;
        const float ox = float(ec.x[size_t(child)]), oy = float(ec.y[size_t(child)]);
        const float a = ox - outerEllipse.cx;
        const float b = oy - outerEllipse.cy;
        const float lineThroughCenter[3] = {a, b, -a * outerEllipse.cx - b * outerEllipse.cy};
        for (size_t j = 1; j < numCircles; ++j) {
            p = dir == -1 ? ec.before[size_t(p)] : ec.after[size_t(p)];
            if (p < 0) {
                release();
                throw std::out_of_range("addCandidateFlowtoCCTag: missing vote link");
            }
            if (!ec.processed_aux[size_t(p)]) {
                ec.processed_aux[size_t(p)] = 1;
                vProcessedEdgePoint.push_back(p);
                const float px = float(ec.x[size_t(p)]), py = float(ec.y[size_t(p)]);
                const float normGrad = std::sqrt(ec.dx[size_t(p)] * ec.dx[size_t(p)] + ec.dy[size_t(p)] * ec.dy[size_t(p)]);
                const float gx = ec.dx[size_t(p)] / normGrad, gy = ec.dy[size_t(p)] / normGrad;
                float tx = outerEllipse.cx - px, ty = outerEllipse.cy - py;
                const float distancePointToCenter = std::sqrt(tx * tx + ty * ty);
                tx /= distancePointToCenter;
                ty /= distancePointToCenter;
                if (gm::is_in_ellipse(outerEllipse, px, py) && is_on_the_same_side(ox, oy, px, py, lineThroughCenter)) {
                    if (float(-dir) * (gx * tx + gy * ty) < -0.5f && j >= numCircles - 2) ++nGradientOut;
                    cctagPoints[numCircles - j - 1].push_back({px, py, ec.dx[size_t(p)], ec.dy[size_t(p)]});
                    if (j >= numCircles - 2) ++nAddedPoint;
                } else {
                    cctagPoints.clear();
                    release();
                    return false;
                }
            }
            dir = -dir;
        }
    }
    release();
    if (float(nGradientOut) / float(nAddedPoint) > 0.5f) {
        cctagPoints.clear();
        return false;
    }
    return true;
}

// Vote.cpp:578-742 isAnotherSegment
bool is_another_segment(EdgeCollection& ec, Ellipse& outerEllipse, std::vector<int>& outerEllipsePoints,
                        const Candidate& another, std::vector<std::vector<DPt>>& cctagPoints, size_t numCircles,
                        float thrMedianDistanceEllipse, gm::Pcg& rng)
{
    const std::vector<int>& anotherOuter = another.outerEllipsePoints;
    if (outerEllipsePoints.size() < 5 || anotherOuter.size() < 5) return false;
    Ellipse qm;
    float Sm = std::numeric_limits<float>::max();
    const std::vector<P2> pts = points_of(ec, outerEllipsePoints);
    const std::vector<P2> anotherPts = points_of(ec, anotherOuter);
    const float SRef = gm::median_ref(distances(outerEllipse, pts));
    size_t cnt = 0;
    int perm[5];
    while (cnt < 100) {
        std::vector<P2> points;
        gm::rand_5_k(perm, outerEllipsePoints.size(), rng);
        for (int i = 0; i < 4; ++i) points.push_back(pts[size_t(perm[i])]);
        gm::rand_5_k(perm, anotherOuter.size(), rng);
        for (int i = 0; i < 4; ++i) points.push_back(anotherPts[size_t(perm[i])]);
        const Ellipse eToto = gm::fit_ellipse(points);  // outside the try, as in the reference
        try {
            const Ellipse q = gm::ellipse_from_matrix(eToto.Q);
            const float ratioSemiAxes = q.a / q.b;
            if (ratioSemiAxes < 0.12 || ratioSemiAxes > 8) {
                ++cnt;
                continue;
            }
            const float S1 = gm::median_ref(distances(q, pts));
            const float S2 = gm::median_ref(distances(q, anotherPts));
            const float S = S1 + S2;
            if (S < Sm) {
                cnt = 0;
                qm = q;
                Sm = S;
            } else {
                ++cnt;
            }
        } catch (...) {
            ++cnt;
        }
    }
    const float thr = 6;
    if (!(Sm < thr * SRef)) return false;
    std::vector<int> temp = outerEllipsePoints;
    temp.insert(temp.end(), anotherOuter.begin(), anotherOuter.end());
    const Ellipse outerEllipseTemp = ellipse_fitting(ec, temp);
    const float quality = perimeter_quality(temp.size(), outerEllipseTemp);
    if (!(quality < 1.1)) return false;
    std::vector<float> vDistFinal;
    for (int e : temp) {
        const P2 q = pt(ec, e);
        vDistFinal.push_back(gm::distance_point_ellipse(outerEllipseTemp.Q, q.x, q.y));
    }
    const float SmFinal = gm::median_ref(vDistFinal);
    if (!(SmFinal < thrMedianDistanceEllipse)) return false;
    if (!add_candidate_flow(ec, another.filteredChildren, anotherOuter, outerEllipseTemp, cctagPoints, numCircles))
        return false;
    outerEllipsePoints = temp;
    outerEllipse = outerEllipseTemp;
    return true;
}

// Detection.cpp:278-377 flowComponentAssembling
void flow_component_assembling(EdgeCollection& ec, float& quality, size_t iCandidate,
                               const std::vector<Candidate>& loopTwo, Ellipse& outerEllipse,
                               std::vector<int>& outerEllipsePoints, std::vector<std::vector<DPt>>& cctagPoints,
                               const cctagb_params& p, gm::Pcg& rng)
{
    const Candidate& candidate = loopTwo[iCandidate];
    int score = -1;
    size_t iMax = 0;
    const float ratioExpension = 2.5f;
    const Ellipse circularResearchArea =
        gm::ellipse_from_params(float(ec.x[size_t(candidate.seed)]), float(ec.y[size_t(candidate.seed)]),
                                ec.flow[size_t(candidate.seed)] * ratioExpension,
                                ec.flow[size_t(candidate.seed)] * ratioExpension, 0.f);
    for (size_t i = 0; i < loopTwo.size(); ++i) {
        if (i == iCandidate) continue;
        const Candidate& another = loopTwo[i];
        if (candidate.nLabel == another.nLabel) continue;
        const float r = ec.flow[size_t(another.seed)] / ec.flow[size_t(candidate.seed)];
        if (!(r > 0.666 && r < 1.5)) continue;
        if (gm::is_in_ellipse(circularResearchArea, float(ec.x[size_t(another.seed)]),
                              float(ec.y[size_t(another.seed)]))) {
            if (another.score > score) {
                score = another.score;
                iMax = i;
            }
        }
    }
    if (score > 0) {
        if (is_another_segment(ec, outerEllipse, outerEllipsePoints, loopTwo[iMax], cctagPoints,
                               size_t(p.nCrowns) * 2, p.thrMedianDistanceEllipse, rng))
            quality = perimeter_quality(outerEllipsePoints.size(), outerEllipse);
    }
}

// Detection.cpp:379-566 cctagDetectionFromEdgesLoopTwoIteration
void loop_two_iteration(std::vector<Marker>& markers, EdgeCollection& ec, const std::vector<Candidate>& loopTwo,
                        size_t iCandidate, int pyramidLevel, float scale, const cctagb_params& p, gm::Pcg& rng)
{
    const Candidate& candidate = loopTwo[iCandidate];
    std::vector<int> outerEllipsePoints = candidate.outerEllipsePoints;
    Ellipse outerEllipse = candidate.outerEllipse;
    std::vector<std::vector<DPt>> cctagPoints;
    try {
        float quality = perimeter_quality(outerEllipsePoints.size(), outerEllipse);
        if (p.searchForAnotherSegment && quality > 0.25 && quality < 0.7)
            flow_component_assembling(ec, quality, iCandidate, loopTwo, outerEllipse, outerEllipsePoints, cctagPoints,
                                      p, rng);
        if (!add_candidate_flow(ec, candidate.filteredChildren, candidate.outerEllipsePoints, outerEllipse,
                                cctagPoints, size_t(p.nCrowns) * 2))
            return;
        const Ellipse rescaleEllipse = gm::ellipse_from_params(outerEllipse.cx, outerEllipse.cy,
                                                               outerEllipse.a * scale, outerEllipse.b * scale,
                                                               outerEllipse.angle);
        const int realPixelPerimeter = gm::rasterize_perimeter(rescaleEllipse);
        const float realSizeOuterEllipsePoints = quality * float(realPixelPerimeter);
        if ((quality <= 0.35 && realSizeOuterEllipsePoints >= 300.0) ||
            (quality <= 0.45f && realSizeOuterEllipsePoints >= 200.0 && realSizeOuterEllipsePoints < 300.0) ||
            (quality <= 0.5f && realSizeOuterEllipsePoints >= 100.0 && realSizeOuterEllipsePoints < 200.0) ||
            (quality <= 0.5f && realSizeOuterEllipsePoints >= 70.0 && realSizeOuterEllipsePoints < 100.0) ||
            (quality <= 0.96f && realSizeOuterEllipsePoints >= 50.0 && realSizeOuterEllipsePoints < 70.0) ||
            (realSizeOuterEllipsePoints < 50.0))
            return;
        const float ratioSemiAxes = outerEllipse.a / outerEllipse.b;
        if (ratioSemiAxes > 8.0 || ratioSemiAxes < 0.125) return;
        Ellipse qIn, qOut;
        gm::compute_hull(outerEllipse, 3.6f, qIn, qOut);
        for (int e : outerEllipsePoints)
            if (!gm::is_in_hull(qIn, qOut, float(ec.x[size_t(e)]), float(ec.y[size_t(e)]))) return;
        float quality2 = 0;
        for (int e : outerEllipsePoints) quality2 += ec.norm[size_t(e)];
        quality2 *= scale;
        // CCTag(-1, center, points, outerEllipse, H, level, scale, quality2) (CCTag.hpp:67-92):
        // the stored ellipse is moved by +0.5 and scaled into level-0 pixels.
        Marker m;
        m.cx_img = outerEllipse.cx;
        m.cy_img = outerEllipse.cy;
        m.outer = gm::ellipse_from_params(outerEllipse.cx + 0.5f, outerEllipse.cy + 0.5f, outerEllipse.a,
                                          outerEllipse.b, outerEllipse.angle);
        m.rescaled = gm::ellipse_from_params(m.outer.cx * scale, m.outer.cy * scale, m.outer.a * scale,
                                             m.outer.b * scale, m.outer.angle);
        m.points = cctagPoints;
        m.level = pyramidLevel;
        m.scale = scale;
        m.quality = quality2;
        markers.push_back(m);
    } catch (...) {
    }
}

}  // namespace

void candidates_from_edges(EdgeCollection& ec, const std::vector<int>& seeds, int level, float scale,
                           const cctagb_params& p, std::vector<Marker>& markers, LoopTwoRecord* rec)
{
    if (seeds.empty()) return;
    const size_t nMaximumNbSeeds = size_t(std::max(ec.H / 2, p.maximumNbSeeds));
    const size_t nSeedsToProcess = std::min(seeds.size(), nMaximumNbSeeds);
    // loop 1, in seed order; candidates ranked by averageReceivedVote
    std::vector<Candidate> loopOne;
    for (size_t iSeed = 0; iSeed < nSeedsToProcess; ++iSeed) {
        const int seed = seeds[iSeed];
        if (ec.processed_in[size_t(seed)]) continue;
        Candidate c;
        c.seed = seed;
        edge_linking(ec, c.convexEdgeSegment, seed, size_t(p.windowSizeOnInnerEllipticSegment), p.averageVoteMin);
        int nReceivedVote = 0, nVotedPoints = 0;
        for (int e : c.convexEdgeSegment) {
            const int v = ec.voters_size(e);
            nReceivedVote += v;
            if (v > 0) ++nVotedPoints;
        }
        c.averageReceivedVote = float(nReceivedVote * nReceivedVote) / float(nVotedPoints);
        const auto it = std::lower_bound(loopOne.begin(), loopOne.end(), c, [](const Candidate& c1, const Candidate& c2) {
            return c1.averageReceivedVote > c2.averageReceivedVote;
        });
        loopOne.insert(it, c);
    }
    // loop 2
    const size_t nLoopTwo = std::min(loopOne.size(), size_t(p.maximumNbCandidatesLoopTwo));
    std::vector<Candidate> loopTwo;
    size_t nSegmentOut = 0;
    for (size_t i = 0; i < nLoopTwo; ++i) {
        gm::Pcg rng = gm::candidate_stream(level, i, 0);
        bool filtered_ok = false;
        if (complete_flow_component(loopOne[i], ec, nSegmentOut, int(i), p, rng, rec != nullptr, filtered_ok))
            loopTwo.push_back(loopOne[i]);
        if (rec) {
            const Candidate& c = loopOne[i];
            rec->seed.push_back(c.seed);
            rec->score.push_back(c.score);
            rec->keep.push_back(filtered_ok ? 1 : 0);
            if (filtered_ok) rec->flt.insert(rec->flt.end(), c.filteredChildren.begin(), c.filteredChildren.end());
            rec->foff.push_back(int(rec->flt.size()));
        }
    }
    if (rec) return;
    // loop 3
    for (size_t i = 0; i < loopTwo.size(); ++i) {
        gm::Pcg rng = gm::candidate_stream(level, i, 1);
        loop_two_iteration(markers, ec, loopTwo, i, level, scale, p, rng);
    }
}

namespace {

// Multiresolution.cpp:43-142 intersectLineToTwoEllipses
bool intersect_line_to_two_ellipses(int y, const Ellipse& qIn, const Ellipse& qOut, const EdgeCollection& ec,
                                    std::list<int>& pointsInHull)
{
    const std::vector<float> io = gm::intersect_with_line(qOut, float(y), true);
    const std::vector<float> ii = gm::intersect_with_line(qIn, float(y), true);
    auto take = [&](int x) {
        const int e = ec.at(x, y);
        if (e < 0) return;
        const float cx = qIn.cx - float(ec.x[size_t(e)]), cy = qIn.cy - float(ec.y[size_t(e)]);
        if (ec.dx[size_t(e)] * cx + ec.dy[size_t(e)] * cy < 0) pointsInHull.push_back(e);
    };
    if (io.size() == 2 && ii.size() == 2) {
        const int begin1 = std::max(0, int(io[0])), end1 = std::min(ec.W - 1, int(ii[0]));
        const int begin2 = std::max(0, int(ii[1])), end2 = std::min(ec.W - 1, int(io[1]));
        for (int x = begin1; x <= end1; ++x) take(x);
        for (int x = begin2; x <= end2; ++x) take(x);
    } else if (io.size() == 2 && ii.size() <= 1) {
        const int begin = std::max(0, int(io[0])), end = std::min(ec.W - 1, int(io[1]));
        for (int x = begin; x <= end; ++x) take(x);
    } else if (io.size() == 1 && ii.empty()) {
        if (io[0] >= 0 && io[0] < float(ec.W)) take(int(io[0]));
    } else {
        return false;
    }
    return true;
}

// Multiresolution.cpp:144-170 selectEdgePointInEllipticHull
void select_edge_points_in_elliptic_hull(const EdgeCollection& ec, const Ellipse& outerEllipse, float scale,
                                         std::list<int>& pointsInHull)
{
    Ellipse qIn, qOut;
    gm::compute_hull(outerEllipse, scale, qIn, qOut);
    const float yCenter = outerEllipse.cy;
    const int maxY = std::max(int(yCenter), 0);
    const int minY = std::min(int(yCenter), ec.H - 1);
    for (int y = maxY; y < ec.H; ++y)
        if (!intersect_line_to_two_ellipses(y, qIn, qOut, ec, pointsInHull)) break;
    for (int y = minY; y >= 0; --y)
        if (!intersect_line_to_two_ellipses(y, qIn, qOut, ec, pointsInHull)) break;
}

}  // namespace

void refit_on_level0(EdgeCollection& ec0, std::vector<Marker>& markers)
{
    for (size_t mi = 0; mi < markers.size(); ++mi) {
        Marker& marker = markers[mi];
        if (marker.level > 0) {
            const float scale = marker.scale;
            std::list<int> pointsInHull;
            select_edge_points_in_elliptic_hull(ec0, marker.rescaled, scale, pointsInHull);
            if (pointsInHull.size() < 5) continue;
            std::vector<int> rescaledOuterEllipsePoints;
            float SmFinal = 1e+10f;
            gm::Pcg rng = gm::refit_stream(mi);
            outlier_removal(ec0, pointsInHull, rescaledOuterEllipsePoints, SmFinal, 20.0f, NO_WEIGHT, 60, rng);
            if (rescaledOuterEllipsePoints.size() < 5) continue;
            try {
                const Ellipse fitted = ellipse_fitting(ec0, rescaledOuterEllipsePoints);
                std::vector<DPt> dp;
                for (int e : rescaledOuterEllipsePoints)
                    dp.push_back({float(ec0.x[size_t(e)]), float(ec0.y[size_t(e)]), ec0.dx[size_t(e)],
                                  ec0.dy[size_t(e)]});
                marker.cx_img = marker.cx_img * scale;
                marker.cy_img = marker.cy_img * scale;
                marker.rescaled = fitted;
                marker.rescaled_points = dp;
            } catch (...) {
            }
        } else {
            marker.rescaled_points = marker.points.empty() ? std::vector<DPt>() : marker.points.back();
        }
    }
}

}  // namespace orc

// ------------------------------------------------ geometry entry points --
// For the known-answer tests of the reference (test/fitEllipse.cpp,
// geometry/test/ellipse.cpp).  xy holds n (x, y) pairs; the fits return 0 and
// the ellipse (cx, cy, a, b, angle) / circle (cx, cy, r), or -1 where the
// reference throws.

extern "C" int orc_fit_ellipse(const float* xy, int n, float* out)
{
    std::vector<orc::gm::P2> p;
    for (int i = 0; i < n; ++i) p.push_back({xy[2 * i], xy[2 * i + 1]});
    try {
        const orc::gm::Ellipse e = orc::gm::fit_ellipse(p);
        out[0] = e.cx;
        out[1] = e.cy;
        out[2] = e.a;
        out[3] = e.b;
        out[4] = e.angle;
        return 0;
    } catch (const std::domain_error&) {
        return -1;
    }
}

extern "C" int orc_fit_circle(const float* xy, int n, float* out)
{
    std::vector<orc::gm::P2> p;
    for (int i = 0; i < n; ++i) p.push_back({xy[2 * i], xy[2 * i + 1]});
    try {
        const orc::gm::Ellipse e = orc::gm::fit_circle(p);
        out[0] = e.cx;
        out[1] = e.cy;
        out[2] = e.a;
        return 0;
    } catch (const std::domain_error&) {
        return -1;
    }
}

// Ellipse(center, a, b, angle).matrix(), row-major.
extern "C" int orc_ellipse_matrix(float cx, float cy, float a, float b, float angle, float* Q)
{
    try {
        const orc::gm::Ellipse e = orc::gm::ellipse_from_params(cx, cy, a, b, angle);
        for (int k = 0; k < 9; ++k) Q[k] = e.Q.v[k / 3][k % 3];
        return 0;
    } catch (const std::invalid_argument&) {
        return -1;
    }
}

// Ellipse(matrix): (cx, cy, a, b, angle), or -1 where the reference throws.
extern "C" int orc_ellipse_params(const float* Q, float* out)
{
    orc::gm::M3 m;
    for (int k = 0; k < 9; ++k) m.v[k / 3][k % 3] = Q[k];
    try {
        const orc::gm::Ellipse e = orc::gm::ellipse_from_matrix(m);
        out[0] = e.cx;
        out[1] = e.cy;
        out[2] = e.a;
        out[3] = e.b;
        out[4] = e.angle;
        return 0;
    } catch (const std::invalid_argument&) {
        return -1;
    }
}
