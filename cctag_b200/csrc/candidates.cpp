// Host candidate stage (see candidates.hpp).  The reference runs its three
// candidate loops with TBB and shared per-point flags, so its output depends
// on the thread schedule.  Here loop 1 runs per level in seed order (the order
// of the reference's single-threaded CCTAG_SERIALIZE build); loops 2 and 3 run
// per candidate on any number of threads, each candidate with its own PCG32
// stream (seed 271828, stream from level, candidate index and loop), and the
// only state they share (the segment labels of loop 2) is assigned in
// candidate order between the two loops.  The result is therefore the same
// for every thread count and schedule.
#include "candidates.hpp"
#include "cand_shared.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <deque>
#include <limits>
#include <stdexcept>

namespace cctagb {

using geo::Ellipse;
using geo::Pt;

void EdgeSet::index_points()
{
    WW = (W + 31) / 32;
    const size_t nw = size_t(WW) * size_t(H);
    own_bidx.assign(nw, Word{0u, 0});
    long long last = -1;
    for (int i = 0; i < E; ++i) {
        const int x = exy[i] & 0xffff, y = exy[i] >> 16;
        const long long pos = (long long)y * W + x;
        if (pos <= last || x >= W || y >= H) throw std::runtime_error("edge points not in raster order");
        last = pos;
        own_bidx[size_t(y) * WW + size_t(x >> 5)].bits |= 1u << (x & 31);
    }
    int32_t r = 0;
    for (size_t k = 0; k < nw; ++k) {
        own_bidx[k].first = r;
        r += int32_t(__builtin_popcount(own_bidx[k].bits));
    }
    bidx = own_bidx.data();
}

void EdgeSet::reset_state()
{
    // segment labels stay -1 between frames (phase C restores the ones it set)
    if (n_segment_out.size() < size_t(E)) n_segment_out.assign(size_t(E), -1);
    processed_in.clear();
    link_stamp.clear();
    link_token = 0;
}

namespace {

using cand::kConvexityLost;
using cand::kEdgeNotFound;

// The points one ellipse-growing run has marked (EdgePoint::_processed ==
// runId in the reference, a test private to the run): a per-thread stamp
// array, with a fresh token per run, so concurrent runs need no shared state.
struct RunMarks {
    std::vector<uint32_t> stamp;
    uint32_t token = 0;
    void begin(size_t E)
    {
        if (stamp.size() < E) stamp.assign(E, 0u);
        if (++token == 0) {  // wrapped: clear the stamps
            std::fill(stamp.begin(), stamp.end(), 0u);
            token = 1;
        }
    }
    void set(int i) { stamp[size_t(i)] = token; }
    void clear(int i) { stamp[size_t(i)] = 0u; }
    bool test(int i) const { return stamp[size_t(i)] == token; }
};

// Vote.cpp:272-394 edgeLinkingDir: follow the edge contour from p while the
// gradient direction keeps turning one way (convexity).
// The reference keeps the visited positions of one edgeLinking call in a set
// of packed (x, y); every such position is an edge point, so a per-point stamp
// equal to the call's token is the same set.
void edge_linking_dir(EdgeSet& es, int p, int dir, std::deque<int>& seg, size_t window, float averageVoteMin)
{
    // the last `window` gradient angles (the reference's deque), as a ring
    thread_local std::vector<float> ring;
    if (ring.size() < window + 1) ring.resize(window + 1);
    size_t head = 0, count = 0;  // oldest entry, entries held
    auto phi_front = [&]() { return ring[head]; };
    auto phi_back = [&]() { return ring[(head + count - 1) % (window + 1)]; };
    size_t i = 0;
    bool found = true;
    int stop = 0;
    const size_t maxLength = 100;
    float averageVote = float(es.voters(p));
    static const int xoff[8] = {1, 1, 0, -1, -1, -1, 0, 1};
    while (i < maxLength && found && averageVote >= averageVoteMin) {
        const float angle = cand::link_angle(es.dx(p), es.dy(p));
        ring[(head + count) % (window + 1)] = angle;
        if (++count > window) {
            head = (head + 1) % (window + 1);
            --count;
        }
        const int shifting = cand::link_shift(angle);
        const int yoff[8] = {0, -dir, -dir, -dir, 0, dir, dir, dir};
        int j = 0;
        stop = 0;
        while (!stop) {
            if (j >= 8) {
                stop = kEdgeNotFound;
            } else {
                const int k = dir == 1 ? (8 - shifting + j) % 8 : (shifting + j) % 8;
                const int sx = es.x(p) + xoff[k];
                const int sy = es.y(p) + yoff[k];
                if (sx >= 0 && sx < es.W && sy >= 0 && sy < es.H && es.at(sx, sy) >= 0 &&
                    es.link_stamp[es.at(sx, sy)] != es.link_token) {
                    if (cand::link_convexity_lost(phi_front(), phi_back(), count == window, dir))
                        stop = kConvexityLost;
                    if (stop == 0) {
                        es.link_stamp[p] = es.link_token;
                        p = es.at(sx, sy);
                        if (dir > 0) seg.push_back(p);
                        else seg.push_front(p);
                        averageVote = cand::link_average_vote(averageVote, int(seg.size()), es.voters(p));
                        stop = 1;
                    }
                    es.link_stamp[p] = es.link_token;
                }
            }
            ++j;
        }
        found = stop == 1;
        ++i;
    }
    if (i == maxLength || stop == kConvexityLost) {
        if (seg.size() > window) {
            size_t n = 0;
            for (int q : seg) {
                if (n == seg.size() - window) break;
                es.processed_in[q] = 1;
                ++n;
            }
        }
    } else if (stop == kEdgeNotFound) {
        for (int q : seg) es.processed_in[q] = 1;
    }
}

// Vote.cpp:255-270
void edge_linking(EdgeSet& es, std::deque<int>& seg, int pmax, size_t window, float averageVoteMin)
{
    if (++es.link_token == 0) {  // wrapped: clear the stamps
        std::fill(es.link_stamp.begin(), es.link_stamp.end(), 0u);
        es.link_token = 1;
    }
    seg.push_back(pmax);
    es.processed_in[pmax] = 1;
    es.link_stamp[pmax] = es.link_token;
    edge_linking_dir(es, pmax, 1, seg, window, averageVoteMin);
    edge_linking_dir(es, pmax, -1, seg, window, averageVoteMin);
}

// Vote.cpp:396-412: voters of the segment's points that received at least
// voteMax/14 votes.
void children_of(const EdgeSet& es, const std::deque<int>& seg, std::vector<int>& children)
{
    size_t voteMax = 1;
    for (int e : seg) voteMax = std::max(voteMax, size_t(es.voters(e)));
    for (int e : seg) {
        const int n = es.voters(e);
        if (n > 0 && size_t(n) >= voteMax / 14)
            for (int k = es.voff[e]; k < es.voff[e + 1]; ++k) children.push_back(es.vlist[k]);
    }
}

enum Weight { kNoWeight = 0, kInvGradWeight = 1 };

// geo::dist_point_ellipse over a point array, as a loop the compiler can
// vectorise (same operations per point, so the same values).
void dist_to_ellipse(const geo::Mat3& Q, const Pt* p, size_t n, float* out)
{
    const float q00 = Q.m[0][0], q01 = Q.m[0][1], q02 = Q.m[0][2], q11 = Q.m[1][1], q12 = Q.m[1][2], q22 = Q.m[2][2];
    for (size_t i = 0; i < n; ++i) {
        const float x = p[i].x, y = p[i].y;
        const float aux0 = x * x, aux1 = 2 * x * y, aux2 = 2 * x, aux3 = y * y, aux4 = 2 * y;
        const float t1 = x * q00 + y * q01 + q02;
        const float t2 = x * q01 + y * q11 + q12;
        const float denom = t1 * t1 + t2 * t2;
        const float dot = aux0 * q00 + aux1 * q01 + aux2 * q02 + aux3 * q11 + aux4 * q12 + q22;
        out[i] = dot * dot / denom;
    }
}

// Whether median_ref(v) (the element of rank n/2, NaN last) is below `bound`,
// without selecting it: that holds exactly when at least n/2 + 1 elements are.
bool median_below(const float* v, size_t n, float bound)
{
    size_t below = 0;
    for (size_t i = 0; i < n; ++i) below += v[i] < bound;
    return below >= n / 2 + 1;
}

// For 0 <= s1 < sm: the smallest float b >= 0 with s1 + b >= sm (float sum).
// The sum grows with b, so for any x >= 0, s1 + x < sm exactly when x < b.
// Binary search over the bit patterns of the non-negative floats, which are
// ordered as their values.
float sum_threshold(float s1, float sm)
{
    uint32_t lo = 0, hi = 0x7f800000u;  // +0 (s1 + 0 < sm) .. +inf (s1 + inf >= sm)
    while (hi - lo > 1) {
        const uint32_t mid = lo + (hi - lo) / 2;
        float x;
        std::memcpy(&x, &mid, 4);
        if (s1 + x >= sm) hi = mid; else lo = mid;
    }
    float b;
    std::memcpy(&b, &hi, 4);
    return b;
}

// Vote.cpp:414-576 outlierRemoval: LMedS ellipse from random 5-point subsets
// of (a regular subsample of) the points; keeps the points whose (weighted)
// distance is below threshold * median.  The reference retries forever when
// the conic of a draw is not a real ellipse; here the number of draws is
// capped (an outlier-free run needs < 100 draws, the cap is 100x that).
void outlier_removal(const EdgeSet& es, const std::vector<int>& children, std::vector<int>& filtered, float& SmFinal,
                     float threshold, int weightedType, size_t maxSize, geo::Pcg32& rng)
{
    filtered.reserve(children.size());
    const size_t nSub = std::min(children.size(), maxSize);
    if (nSub < 5) return;
    const float step = float(children.size()) / float(nSub);
    std::vector<Pt> pts;
    std::vector<float> weights;
    pts.reserve(children.size());
    size_t k = 0;
    for (size_t i = 0; i < children.size(); ++i) {
        if (i == size_t(float(k) * step)) {
            ++k;
            const int e = children[i];
            pts.push_back({float(es.x(e)), float(es.y(e))});
            if (weightedType == kInvGradWeight) weights.push_back(255.f / es.norm(e));
        }
    }
    Ellipse qm;
    float Sm = 10000000.0f;
    size_t counter = 0, draws = 0;
    int perm[5];
    std::vector<float> dist(pts.size());
    while (counter < 70 && draws < 7000) {
        ++draws;
        rng.rand5(perm, pts.size());
        geo::Mat3 Q;
        const int kind = cand::lmeds_conic(pts.data(), perm, Q);
        if (kind == 0) {
            ++counter;
            continue;
        }
        if (kind == 2) continue;  // the reference's exception: not counted
        {
            dist_to_ellipse(Q, pts.data(), pts.size(), dist.data());
            if (weightedType != kNoWeight)
                for (size_t i = 0; i < dist.size(); ++i) dist[i] *= weights[i];
            // most draws do not improve on Sm: decide that by counting
            if (!median_below(dist.data(), dist.size(), Sm)) {
                ++counter;
                continue;
            }
            const float S = geo::median_ref(dist);
            if (S < Sm) {
                counter = 0;
                qm.Q = Q;
                Sm = S;
            } else {
                ++counter;
            }
        }
    }
    std::vector<float> vd;
    vd.reserve(children.size());
    for (int e : children) {
        float d = geo::dist_point_ellipse(qm.Q, float(es.x(e)), float(es.y(e)));
        if (weightedType == kInvGradWeight) d = d * 255 / es.norm(e);
        if (d < threshold * Sm) {
            filtered.push_back(e);
            vd.push_back(d);
        }
    }
    if (vd.empty()) return;
    SmFinal = geo::median_ref(vd);
}

// Fitting.cpp:213-292 innerProdMin (only its return value is used).
float inner_prod_min(const EdgeSet& es, const std::vector<int>& fc, float thr)
{
    if (fc.empty()) return 1.1f;
    const int p0 = fc.front();
    float ng = std::sqrt(es.dx(p0) * es.dx(p0) + es.dy(p0) * es.dy(p0));
    const float gx0 = es.dx(p0) / ng, gy0 = es.dy(p0) / ng;
    float mn = 1.1f;
    int pA = -1;
    for (size_t i = 1; i < fc.size(); ++i) {
        const int q = fc[i];
        ng = std::sqrt(es.dx(q) * es.dx(q) + es.dy(q) * es.dy(q));
        const float ip = gx0 * (es.dx(q) / ng) + gy0 * (es.dy(q) / ng);
        if (ip <= thr) return ip;
        if (ip < mn) {
            mn = ip;
            pA = q;
        }
    }
    if (pA < 0) return mn;
    ng = std::sqrt(es.dx(pA) * es.dx(pA) + es.dy(pA) * es.dy(pA));
    const float gxm = es.dx(pA) / ng, gym = es.dy(pA) / ng;
    mn = 1.f;
    for (int q : fc) {
        ng = std::sqrt(es.dx(q) * es.dx(q) + es.dy(q) * es.dy(q));
        const float ip = gxm * (es.dx(q) / ng) + gym * (es.dy(q) / ng);
        if (ip <= thr) return ip;
        if (ip < mn) mn = ip;
    }
    return mn;
}

Ellipse fit_points(const EdgeSet& es, const std::vector<int>& idx)
{
    std::vector<Pt> p(idx.size());
    for (size_t i = 0; i < idx.size(); ++i) p[i] = {float(es.x(idx[i])), float(es.y(idx[i]))};
    return geo::fit_ellipse(p.data(), p.size());
}

Ellipse fit_circle_points(const EdgeSet& es, const std::vector<int>& idx)
{
    std::vector<Pt> p(idx.size());
    for (size_t i = 0; i < idx.size(); ++i) p[i] = {float(es.x(idx[i])), float(es.y(idx[i]))};
    return geo::fit_circle(p.data(), p.size());
}

// EllipseGrowing.cpp:345-357 (isGoodEGPoints) + :359-376 (ellipseGrowingInit)
bool ellipse_growing_init(const EdgeSet& es, const std::vector<int>& fc, Ellipse& e)
{
    if (inner_prod_min(es, fc, 0.25f) <= 0.25f) {
        e = fit_points(es, fc);
        return true;
    }
    e = fit_circle_points(es, fc);
    return false;
}

// EllipseGrowing.cpp:378-422 connectedPoint: depth-first growth through
// 8-neighbours inside the hull whose gradient points away from the center,
// from listed point p.  Iterative form of the reference's recursion (same
// visiting order).  Returns whether p is saturated: every edge pixel around
// it is marked, so no later pass can grow anything from it (marks only grow
// until the growing loop resets them).
bool connected_point(std::vector<int>& pts, RunMarks& mk, EdgeSet& es, const Ellipse& qIn, const Ellipse& qOut,
                     int p, std::vector<EdgeSet::DfsFrame>& st)
{
    static const int xoff[8] = {1, 1, 0, -1, -1, -1, 0, 1};
    static const int yoff[8] = {0, -1, -1, -1, 0, 1, 1, 1};
    using Frame = EdgeSet::DfsFrame;
    st.clear();
    mk.set(p);  // the reference marks the start point; a listed point already is
    st.push_back({es.x(p), es.y(p), 0});
    bool saturated = true;
    while (!st.empty()) {
        Frame& f = st.back();
        if (f.k >= 8) {
            st.pop_back();
            continue;
        }
        const int k = f.k++;
        const bool start = st.size() == 1;
        const int sx = f.x + xoff[k], sy = f.y + yoff[k];
        if (sx < 0 || sx >= es.W || sy < 0 || sy >= es.H) continue;
        const int e = es.at(sx, sy);
        if (e < 0) continue;
        if (mk.test(e)) continue;
        bool grow = geo::is_in_hull(qIn, qOut, float(es.x(e)), float(es.y(e)));
        if (grow) {
            const float ox = qIn.cx - float(es.x(e)), oy = qIn.cy - float(es.y(e));
            grow = es.dx(e) * ox + es.dy(e) * oy < 0;
        }
        if (grow) {
            pts.push_back(e);
            mk.set(e);
            st.push_back({sx, sy, 0});
        } else if (start) {
            saturated = false;  // an unmarked edge pixel another hull may take
        }
    }
    return saturated;
}

// EllipseGrowing.cpp:443-457.  sat[i]: list point i is saturated (skipped:
// it would add nothing and mark nothing).
void ellipse_hull(EdgeSet& es, std::vector<int>& pts, const Ellipse& e, float delta, RunMarks& mk,
                  std::vector<uint8_t>& sat, std::vector<EdgeSet::DfsFrame>& st)
{
    Ellipse qIn, qOut;
    geo::compute_hull(e, delta, qIn, qOut);
    const size_t init = pts.size();
    sat.resize(init, 0);
    for (size_t i = 0; i < init; ++i)
        if (!sat[i] && connected_point(pts, mk, es, qIn, qOut, pts[i], st)) sat[i] = 1;
}

size_t count_in_hull(const EdgeSet& es, const std::vector<int>& pts, const Ellipse& e, float width)
{
    Ellipse qIn, qOut;
    geo::compute_hull(e, width, qIn, qOut);
    size_t n = 0;
    for (int p : pts)
        if (geo::is_in_hull(qIn, qOut, float(es.x(p)), float(es.y(p)))) ++n;
    return n;
}

// EllipseGrowing.cpp:459-551 ellipseGrowing2
void ellipse_growing2(EdgeSet& es, const std::vector<int>& fc, std::vector<int>& outer, Ellipse& ellipse, float width,
                      bool goodInit)
{
    thread_local RunMarks mk;
    thread_local std::vector<uint8_t> sat;  // saturated list points (connected_point)
    thread_local std::vector<EdgeSet::DfsFrame> st;  // connected_point's depth-first stack
    mk.begin(size_t(es.E));
    sat.clear();
    outer = fc;
    for (int c : fc) mk.set(c);
    if (!goodInit) {
        int newSize = int(outer.size());
        int maxNb = newSize, nIterMax = 0, lastSize = 0, nIter = 0;
        std::vector<std::vector<int>> sets{outer};
        std::vector<Ellipse> ells{ellipse};
        ++nIter;
        while (newSize - lastSize > 0) {
            lastSize = int(count_in_hull(es, outer, ellipse, width));
            ellipse_hull(es, outer, ellipse, width, mk, sat, st);
            sets.push_back(outer);
            ells.push_back(ellipse);
            ellipse = fit_circle_points(es, outer);
            newSize = int(count_in_hull(es, outer, ellipse, width));
            if (newSize > maxNb) {
                maxNb = newSize;
                nIterMax = nIter;
            }
            ++nIter;
        }
        outer = sets[nIterMax];
        ellipse = ells[nIterMax];
        for (auto& s : sets)
            for (int p : s) mk.clear(p);
        for (int p : outer) mk.set(p);
        sat.clear();  // marks were taken back
    }
    ellipse = fit_points(es, outer);
    size_t lastSize = 0;
    while (outer.size() > lastSize) {
        lastSize = outer.size();
        ellipse_hull(es, outer, ellipse, width, mk, sat, st);
        ellipse = fit_points(es, outer);
    }
}

struct Candidate {
    int seed = -1;
    std::deque<int> segment;
    std::vector<int> outer;
    Ellipse outerEllipse;
    std::vector<int> filtered;
    std::vector<int> chains;  // per filtered point, its numCircles - 1 link hops (LoopTwoIn::chain)
    int score = 0;
    size_t nLabel = 0;
    float averageReceivedVote = 0.f;
    float flow = 0.f;  // flow length of the seed
};

float quality_of(size_t npts, const Ellipse& e) { return float(npts) / float(geo::rasterize_perimeter(e)); }

// Detection.cpp:115-267 completeFlowComponent, in three phases so that the
// per-candidate work can run in parallel: (B) children and LMedS outlier
// removal, (C) segment labels -- sequential, in candidate order, as the
// reference assigns them -- and (D) ellipse growing and the final checks.
// Phase B: returns whether the candidate continues (>= 5 filtered children).
bool flow_component_filter(Candidate& c, EdgeSet& es, const cctagb_params& p, geo::Pcg32& rng)
{
    try {
        std::vector<int> children;
        children_of(es, c.segment, children);
        if (children.size() < size_t(p.minPointsSegmentCandidate)) return false;
        c.score = int(children.size());
        float SmFinal = 1e+10f;
        outlier_removal(es, children, c.filtered, SmFinal, p.threshRobustEstimationOfOuterEllipse, kInvGradWeight, 60,
                        rng);
        return c.filtered.size() >= 5;
    } catch (...) {
        return false;
    }
}

// Phase C (Detection.cpp:157-189)
void flow_component_label(Candidate& c, EdgeSet& es, size_t& nSegmentOut)
{
    long common = -1;
    for (int q : c.filtered)
        if (es.n_segment_out[q] != -1) {
            common = es.n_segment_out[q];
            break;
        }
    const size_t nLabel = common == -1 ? nSegmentOut++ : size_t(common);
    for (int q : c.filtered) es.n_segment_out[q] = int32_t(nLabel);
    c.nLabel = nLabel;
}

// Phase D: returns whether the candidate enters the second list.
bool flow_component_grow(Candidate& c, EdgeSet& es, const cctagb_params& p)
{
    try {
        const bool goodInit = ellipse_growing_init(es, c.filtered, c.outerEllipse);
        ellipse_growing2(es, c.filtered, c.outer, c.outerEllipse, p.ellipseGrowingEllipticHullWidth, goodInit);
        std::vector<float> vd;
        vd.reserve(c.outer.size());
        for (int q : c.outer) vd.push_back(geo::dist_point_ellipse(c.outerEllipse.Q, float(es.x(q)), float(es.y(q))));
        if (vd.empty()) return false;
        const float SmFinal = geo::median_ref(vd);
        if (SmFinal > p.thrMedianDistanceEllipse) return false;
        // the reference's literals are doubles: a float compares with 1.1, 0.05 as a double
        if (quality_of(c.outer.size(), c.outerEllipse) > 1.1) return false;
        const float ratio = c.outerEllipse.a / c.outerEllipse.b;
        if (ratio < 0.05 || ratio > 20) return false;
        return true;
    } catch (...) {
        return false;
    }
}

bool same_side(float x1, float y1, float x2, float y2, const float line[3])
{
    const float s1 = x1 * line[0] + y1 * line[1] + line[2];
    const float s2 = x2 * line[0] + y2 * line[1] + line[2];
    return s1 * s2 > 0;
}

// EllipseGrowing.hpp:24-33 isInEllipse: p^T Q p and p^T Q c have the same sign.
bool in_ellipse(const Ellipse& e, float x, float y)
{
    const geo::Mat3& Q = e.Q;
    const float s1 = geo::qform(Q, x, y);
    const float qc0 = Q.m[0][0] * e.cx + Q.m[0][1] * e.cy + Q.m[0][2];
    const float qc1 = Q.m[1][0] * e.cx + Q.m[1][1] * e.cy + Q.m[1][2];
    const float qc2 = Q.m[2][0] * e.cx + Q.m[2][1] * e.cy + Q.m[2][2];
    const float s2 = x * qc0 + y * qc1 + qc2;
    return s1 * s2 > 0;
}

// EllipseGrowing.cpp:63-178 addCandidateFlowtoCCTag.  The links walked from
// fc[k] are chains[k * (numCircles - 1) + j - 1].
bool add_candidate_flow(EdgeSet& es, const std::vector<int>& fc, const std::vector<int>& chains,
                        const std::vector<int>& outer, const Ellipse& oe, std::vector<std::vector<DirPoint>>& pts,
                        size_t numCircles)
{
    if (chains.size() != fc.size() * (numCircles - 1)) throw std::logic_error("link chains do not match the points");
    pts.resize(numCircles);
    for (int e : outer) pts.back().push_back({float(es.x(e)), float(es.y(e)), es.dx(e), es.dy(e)});
    // The reference marks visited points in a shared per-point flag and clears
    // it on return; a per-thread stamp (this call's token) gives the same
    // visits and lets candidates run concurrently.
    thread_local std::vector<uint32_t> stamp;
    thread_local uint32_t token = 0;
    if (stamp.size() < size_t(es.E)) stamp.assign(size_t(es.E), 0u);
    if (++token == 0) {  // wrapped: clear the stamps
        std::fill(stamp.begin(), stamp.end(), 0u);
        token = 1;
    }
    auto first_visit = [&](int q) {
        if (stamp[size_t(q)] == token) return false;
        stamp[size_t(q)] = token;
        return true;
    };
    for (auto& v : pts) v.reserve(v.size() + fc.size());
    // in_ellipse's transformed center, the same for every point
    const geo::Mat3& Q = oe.Q;
    const float qc0 = Q.m[0][0] * oe.cx + Q.m[0][1] * oe.cy + Q.m[0][2];
    const float qc1 = Q.m[1][0] * oe.cx + Q.m[1][1] * oe.cy + Q.m[1][2];
    const float qc2 = Q.m[2][0] * oe.cx + Q.m[2][1] * oe.cy + Q.m[2][2];
    size_t nGradientOut = 0, nAdded = 0;
    for (size_t k = 0; k < fc.size(); ++k) {
        const int p0 = fc[k];
        const int* chain = chains.data() + k * (numCircles - 1);
        int dir = -1;
        int p = p0;
        const float ox = float(es.x(p0)), oy = float(es.y(p0));
        const float a = ox - oe.cx, b = oy - oe.cy;
        const float line[3] = {a, b, -a * oe.cx - b * oe.cy};
        for (size_t j = 1; j < numCircles; ++j) {
            p = chain[j - 1];  // dir == -1 ? before[p] : after[p]
            if (p < 0) {
                throw std::out_of_range("EdgePointCollection: missing link");
            }
            if (first_visit(p)) {
                const DirPoint q{float(es.x(p)), float(es.y(p)), es.dx(p), es.dy(p)};
                const bool inside = geo::qform(Q, q.x, q.y) * (q.x * qc0 + q.y * qc1 + qc2) > 0;
                if (inside && same_side(ox, oy, q.x, q.y, line)) {
                    if (j >= numCircles - 2) {
                        // gradient against the direction to the center (the last two circles only)
                        const float ng = std::sqrt(q.dx * q.dx + q.dy * q.dy);
                        const float gx = q.dx / ng, gy = q.dy / ng;
                        float tx = oe.cx - q.x, ty = oe.cy - q.y;
                        const float dc = std::sqrt(tx * tx + ty * ty);
                        tx /= dc;
                        ty /= dc;
                        if (float(-dir) * (gx * tx + gy * ty) < -0.5f) ++nGradientOut;
                    }
                    pts[numCircles - j - 1].push_back(q);
                    if (j >= numCircles - 2) ++nAdded;
                } else {
                    pts.clear();
                    return false;
                }
            }
            dir = -dir;
        }
    }
    if (float(nGradientOut) / float(nAdded) > 0.5f) {
        pts.clear();
        return false;
    }
    return true;
}

// Vote.cpp:578-742 isAnotherSegment
bool is_another_segment(EdgeSet& es, Ellipse& outerEllipse, std::vector<int>& outer, const Candidate& another,
                        std::vector<std::vector<DirPoint>>& pts, size_t numCircles, float thrMedian, geo::Pcg32& rng)
{
    const std::vector<int>& aout = another.outer;
    if (outer.size() < 5 || aout.size() < 5) return false;
    std::vector<Pt> P(outer.size()), AP(aout.size());
    for (size_t i = 0; i < outer.size(); ++i) P[i] = {float(es.x(outer[i])), float(es.y(outer[i]))};
    for (size_t i = 0; i < aout.size(); ++i) AP[i] = {float(es.x(aout[i])), float(es.y(aout[i]))};
    std::vector<float> d, d2(AP.size());
    d.reserve(std::max(P.size(), AP.size()));
    for (const Pt& q : P) d.push_back(geo::dist_point_ellipse(outerEllipse.Q, q.x, q.y));
    const float SRef = geo::median_ref(d);
    Ellipse qm;
    float Sm = std::numeric_limits<float>::max();
    size_t cnt = 0;
    int perm[5];
    while (cnt < 100) {
        Pt pp[8];
        rng.rand5(perm, outer.size());
        for (int i = 0; i < 4; ++i) pp[i] = P[perm[i]];
        rng.rand5(perm, aout.size());
        for (int i = 0; i < 4; ++i) pp[4 + i] = AP[perm[i]];
        // The fit of the eight points sits outside the reference's try block
        // (Vote.cpp:640-645): a fit that throws ends the whole loop-3
        // iteration of this candidate, not just the draw.
        const Ellipse fit8 = geo::fit_ellipse(pp, 8);
        try {
            const Ellipse q = Ellipse::from_matrix(fit8.Q);
            const float ratio = q.a / q.b;
            if (ratio < 0.12 || ratio > 8) {
                ++cnt;
                continue;
            }
            d.resize(P.size());
            dist_to_ellipse(q.Q, P.data(), P.size(), d.data());
            // S = S1 + S2 >= S1 (S2 >= 0): no improvement unless S1 < Sm
            if (!median_below(d.data(), d.size(), Sm)) {
                ++cnt;
                continue;
            }
            // distances are >= 0 or NaN, so S < Sm needs S2 < Sm, and holds
            // exactly when S2 is below sum_threshold(S1, Sm): most draws are
            // decided by counting
            dist_to_ellipse(q.Q, AP.data(), AP.size(), d2.data());
            if (!median_below(d2.data(), d2.size(), Sm)) {
                ++cnt;
                continue;
            }
            const float S1 = geo::median_ref(d);
            if (!median_below(d2.data(), d2.size(), sum_threshold(S1, Sm))) {
                ++cnt;
                continue;
            }
            const float S2 = geo::median_ref(d2);
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
    if (!(Sm < 6.f * SRef)) return false;
    std::vector<int> merged = outer;
    merged.insert(merged.end(), aout.begin(), aout.end());
    const Ellipse fitted = fit_points(es, merged);
    if (!(quality_of(merged.size(), fitted) < 1.1)) return false;
    d.clear();
    for (int q : merged) d.push_back(geo::dist_point_ellipse(fitted.Q, float(es.x(q)), float(es.y(q))));
    const float SmFinal = geo::median_ref(d);
    if (!(SmFinal < thrMedian)) return false;
    if (!add_candidate_flow(es, another.filtered, another.chains, aout, fitted, pts, numCircles)) return false;
    outer = merged;
    outerEllipse = fitted;
    return true;
}

// Detection.cpp:278-377 flowComponentAssembling
void flow_component_assembling(EdgeSet& es, float& quality, size_t ci, const std::vector<Candidate>& loop2,
                               Ellipse& outerEllipse, std::vector<int>& outer,
                               std::vector<std::vector<DirPoint>>& pts, const cctagb_params& p, geo::Pcg32& rng)
{
    const Candidate& c = loop2[ci];
    int score = -1;
    size_t iMax = 0;
    const float r = c.flow * 2.5f;
    const Ellipse area = Ellipse::from_params(float(es.x(c.seed)), float(es.y(c.seed)), r, r, 0.f);
    for (size_t i = 0; i < loop2.size(); ++i) {
        if (i == ci) continue;
        const Candidate& o = loop2[i];
        if (c.nLabel == o.nLabel) continue;
        const float ratio = o.flow / c.flow;
        if (!(ratio > 0.666 && ratio < 1.5)) continue;
        if (in_ellipse(area, float(es.x(o.seed)), float(es.y(o.seed)))) {
            if (o.score > score) {
                score = o.score;
                iMax = i;
            }
        }
    }
    if (score > 0) {
        if (is_another_segment(es, outerEllipse, outer, loop2[iMax], pts, size_t(p.nCrowns) * 2,
                               p.thrMedianDistanceEllipse, rng))
            quality = quality_of(outer.size(), outerEllipse);
    }
}

// Detection.cpp:379-566 cctagDetectionFromEdgesLoopTwoIteration
void loop_two_iteration(EdgeSet& es, const std::vector<Candidate>& loop2, size_t ci, int level, float scale,
                        const cctagb_params& p, geo::Pcg32& rng, std::vector<MarkerCand>& markers)
{
    const Candidate& c = loop2[ci];
    std::vector<int> outer = c.outer;
    Ellipse oe = c.outerEllipse;
    std::vector<std::vector<DirPoint>> pts;
    try {
        float quality = quality_of(outer.size(), oe);
        if (p.searchForAnotherSegment && quality > 0.25 && quality < 0.7)
            flow_component_assembling(es, quality, ci, loop2, oe, outer, pts, p, rng);
        if (!add_candidate_flow(es, c.filtered, c.chains, c.outer, oe, pts, size_t(p.nCrowns) * 2)) return;
        const Ellipse rescale = Ellipse::from_params(oe.cx, oe.cy, oe.a * scale, oe.b * scale, oe.angle);
        const float realSize = quality * float(geo::rasterize_perimeter(rescale));
        if ((quality <= 0.35 && realSize >= 300.0f) ||
            (quality <= 0.45f && realSize >= 200.0f && realSize < 300.0f) ||
            (quality <= 0.5f && realSize >= 100.0f && realSize < 200.0f) ||
            (quality <= 0.5f && realSize >= 70.0f && realSize < 100.0f) ||
            (quality <= 0.96f && realSize >= 50.0f && realSize < 70.0f) || (realSize < 50.0f))
            return;
        const float ratio = oe.a / oe.b;
        if (ratio > 8.0f || ratio < 0.125f) return;
        Ellipse qIn, qOut;
        geo::compute_hull(oe, 3.6f, qIn, qOut);
        for (int q : outer)
            if (!geo::is_in_hull(qIn, qOut, float(es.x(q)), float(es.y(q)))) return;
        float quality2 = 0;
        for (int q : outer) quality2 += es.norm(q);
        quality2 *= scale;
        // CCTag constructor (CCTag.hpp:67-92): centerImg = ellipse center,
        // stored ellipse shifted by +0.5, rescaled copy in level-0 pixels.
        MarkerCand m;
        m.cx_img = oe.cx;
        m.cy_img = oe.cy;
        m.outer = Ellipse::from_params(oe.cx + 0.5f, oe.cy + 0.5f, oe.a, oe.b, oe.angle);
        m.rescaled = Ellipse::from_params(m.outer.cx * scale, m.outer.cy * scale, m.outer.a * scale,
                                          m.outer.b * scale, m.outer.angle);
        m.points = std::move(pts);
        m.level = level;
        m.scale = scale;
        m.quality = quality2;
        markers.push_back(std::move(m));
    } catch (...) {
    }
}

}  // namespace

namespace {

// Loop 1 (Detection.cpp:69-113, 609-627) of one level: convex segments from
// the seeds in order, ranked by averageReceivedVote.  The reference inserts
// each candidate before the first one with a key <= its own (std::lower_bound
// with '>'), i.e. key descending and, for equal keys, newest first.
void link_level(EdgeSet& es, const std::vector<int32_t>& seeds, const cctagb_params& p, std::vector<Candidate>& loop1)
{
    loop1.clear();
    es.processed_in.assign(size_t(es.E), 0);
    es.link_stamp.assign(size_t(es.E), 0u);
    es.link_token = 0;
    if (seeds.empty()) return;
    const size_t nMax = size_t(std::max(es.H / 2, p.maximumNbSeeds));
    const size_t nProc = std::min(seeds.size(), nMax);
    std::vector<Candidate> made;
    made.reserve(nProc);
    for (size_t s = 0; s < nProc; ++s) {
        const int seed = seeds[s];
        if (es.processed_in[seed]) continue;
        Candidate c;
        c.seed = seed;
        c.flow = es.flow[seed];
        edge_linking(es, c.segment, seed, size_t(p.windowSizeOnInnerEllipticSegment), p.averageVoteMin);
        int nReceived = 0, nVoted = 0;
        for (int q : c.segment) {
            const int v = es.voters(q);
            nReceived += v;
            if (v > 0) ++nVoted;
        }
        c.averageReceivedVote = float(nReceived * nReceived) / float(nVoted);
        made.push_back(std::move(c));
    }
    std::vector<int> order(made.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = int(i);
    std::sort(order.begin(), order.end(), [&](int x, int y) {
        const float kx = made[x].averageReceivedVote, ky = made[y].averageReceivedVote;
        if (kx > ky) return true;
        if (ky > kx) return false;
        return x > y;
    });
    loop1.reserve(made.size());
    for (int i : order) loop1.push_back(std::move(made[i]));
}

// PCG32 stream of one candidate in one phase: results do not depend on how
// candidates are spread over threads.
geo::Pcg32 candidate_rng(int level, size_t index, int phase)
{
    return cand::candidate_rng(level, uint64_t(index), phase);
}

}  // namespace

namespace {

struct LevelState {
    std::vector<Candidate> loop1, loop2;
    std::vector<uint8_t> keep;
    std::vector<std::vector<MarkerCand>> out3;
};

// Phases A (loop 1, one task per level) and B (children and outlier removal,
// one task per candidate).
void phases_a_b(std::vector<LevelJob>& jobs, const cctagb_params& p, const ParallelFor& pf,
                std::vector<LevelState>& st)
{
    const int nl = int(jobs.size());
    pf(nl, [&](int l) { link_level(*jobs[l].es, *jobs[l].seeds, p, st[l].loop1); });
    std::vector<std::pair<int, int>> tasks;
    for (int l = 0; l < nl; ++l) {
        const size_t n2 = std::min(st[l].loop1.size(), size_t(p.maximumNbCandidatesLoopTwo));
        st[l].keep.assign(n2, 0);
        for (size_t i = 0; i < n2; ++i) tasks.emplace_back(l, int(i));
    }
    pf(int(tasks.size()), [&](int t) {
        const int l = tasks[t].first, i = tasks[t].second;
        geo::Pcg32 rng = candidate_rng(jobs[l].level, size_t(i), 0);
        Candidate& c = st[l].loop1[i];
        st[l].keep[i] = flow_component_filter(c, *jobs[l].es, p, rng) ? 1 : 0;
        // the link chains of the filtered points, from the host's links
        const int len = 2 * p.nCrowns - 1;
        const EdgeSet& es = *jobs[l].es;
        c.chains.clear();
        if (st[l].keep[i])
            for (int p0 : c.filtered) {
                int q = p0;
                for (int j = 0; j < len; ++j) {
                    q = q < 0 ? -1 : (j & 1) ? es.after[q] : es.before[q];
                    c.chains.push_back(q);
                }
            }
    });
}

}  // namespace

void link_and_filter(std::vector<LevelJob>& jobs, const cctagb_params& p, const ParallelFor& pf,
                     std::vector<LoopTwoIn>& out)
{
    std::vector<LevelState> st(jobs.size());
    phases_a_b(jobs, p, pf, st);
    out.assign(jobs.size(), {});
    for (size_t l = 0; l < jobs.size(); ++l) {
        LoopTwoIn& o = out[l];
        o.foff.push_back(0);
        for (size_t i = 0; i < st[l].keep.size(); ++i) {
            const Candidate& c = st[l].loop1[i];
            o.seed.push_back(c.seed);
            o.flow.push_back(c.flow);
            o.score.push_back(c.score);
            o.keep.push_back(st[l].keep[i]);
            if (st[l].keep[i]) {
                o.flt.insert(o.flt.end(), c.filtered.begin(), c.filtered.end());
                o.chain.insert(o.chain.end(), c.chains.begin(), c.chains.end());
            }
            o.foff.push_back(int32_t(o.flt.size()));
        }
        o.chainLen = 2 * p.nCrowns - 1;
    }
}

void detect_from_edges(std::vector<LevelJob>& jobs, const cctagb_params& p, const ParallelFor& pf,
                       const std::vector<LoopTwoIn>* given, const GrowFn* grow, int* grown)
{
    if (grown) grown[0] = grown[1] = 0;
    const int nl = int(jobs.size());
    std::vector<LevelState> st(static_cast<size_t>(nl));
    if (!given) {
        phases_a_b(jobs, p, pf, st);
    } else {
        if (given->size() != jobs.size()) throw std::runtime_error("loop-two inputs do not match the levels");
        for (int l = 0; l < nl; ++l) {
            const LoopTwoIn& g = (*given)[size_t(l)];
            const size_t n2 = g.seed.size();
            st[l].loop1.resize(n2);
            st[l].keep.assign(g.keep.begin(), g.keep.end());
            for (size_t i = 0; i < n2; ++i) {
                Candidate& c = st[l].loop1[i];
                c.seed = g.seed[i];
                c.flow = g.flow[i];
                c.score = g.score[i];
                c.filtered.assign(g.flt.begin() + g.foff[i], g.flt.begin() + g.foff[i + 1]);
                if (g.chainLen != 2 * p.nCrowns - 1 || g.chain.size() != g.flt.size() * size_t(g.chainLen))
                    throw std::runtime_error("loop-two inputs without their link chains");
                c.chains.assign(g.chain.begin() + size_t(g.foff[i]) * g.chainLen,
                                g.chain.begin() + size_t(g.foff[i + 1]) * g.chainLen);
            }
        }
    }
    std::vector<std::pair<int, int>> tasks;
    for (int l = 0; l < nl; ++l)
        for (size_t i = 0; i < st[l].keep.size(); ++i) tasks.emplace_back(l, int(i));
    // Phase C: segment labels in candidate order.
    for (int l = 0; l < nl; ++l) {
        size_t nSegmentOut = 0;
        for (size_t i = 0; i < st[l].keep.size(); ++i)
            if (st[l].keep[i]) flow_component_label(st[l].loop1[i], *jobs[l].es, nSegmentOut);
    }
    // The labels are kept in the candidates (nLabel): put the per-point ones
    // back to -1 for the next frame.
    for (int l = 0; l < nl; ++l)
        for (size_t i = 0; i < st[l].keep.size(); ++i)
            if (st[l].keep[i])
                for (int q : st[l].loop1[i].filtered) jobs[l].es->n_segment_out[q] = -1;
    // Phase D: ellipse growing, each run with its own point marks.
    if (grow) {
        std::vector<GrowJob> gj;
        std::vector<std::pair<int, int>> idx;
        for (const auto& t : tasks) {
            Candidate& c = st[t.first].loop1[size_t(t.second)];
            if (!st[t.first].keep[size_t(t.second)]) continue;
            GrowJob g;
            g.level = t.first;
            g.filtered = &c.filtered;
            g.outer = &c.outer;
            g.ellipse = &c.outerEllipse;
            gj.push_back(g);
            idx.push_back(t);
        }
        (*grow)(gj);
        std::vector<int> rest;  // not grown there
        for (size_t k = 0; k < gj.size(); ++k) {
            if (gj[k].status == 2) rest.push_back(int(k));
            else if (gj[k].status == 0) st[idx[k].first].keep[size_t(idx[k].second)] = 0;
        }
        pf(int(rest.size()), [&](int r) {
            const auto& t = idx[size_t(rest[size_t(r)])];
            if (!flow_component_grow(st[t.first].loop1[size_t(t.second)], *jobs[t.first].es, p))
                st[t.first].keep[size_t(t.second)] = 0;
        });
        if (grown) {
            grown[0] = int(gj.size() - rest.size());
            grown[1] = int(rest.size());
        }
    } else {
        if (grown)
            for (const auto& t : tasks) grown[1] += st[t.first].keep[size_t(t.second)] ? 1 : 0;
        pf(int(tasks.size()), [&](int t) {
            const int l = tasks[t].first, i = tasks[t].second;
            if (st[l].keep[i] && !flow_component_grow(st[l].loop1[i], *jobs[l].es, p)) st[l].keep[i] = 0;
        });
    }
    tasks.clear();
    for (int l = 0; l < nl; ++l) {
        for (size_t i = 0; i < st[l].keep.size(); ++i)
            if (st[l].keep[i]) st[l].loop2.push_back(std::move(st[l].loop1[i]));
        st[l].out3.assign(st[l].loop2.size(), {});
        for (size_t i = 0; i < st[l].loop2.size(); ++i) tasks.emplace_back(l, int(i));
    }
    // Phase E: loop 3 (Detection.cpp:677-688), markers kept in candidate order.
    pf(int(tasks.size()), [&](int t) {
        const int l = tasks[t].first, i = tasks[t].second;
        geo::Pcg32 rng = candidate_rng(jobs[l].level, size_t(i), 1);
        loop_two_iteration(*jobs[l].es, st[l].loop2, size_t(i), jobs[l].level, jobs[l].scale, p, rng, st[l].out3[i]);
    });
    for (int l = 0; l < nl; ++l) {
        jobs[l].out.clear();
        for (auto& v : st[l].out3)
            for (auto& m : v) jobs[l].out.push_back(std::move(m));
    }
}

namespace {

// Multiresolution.cpp:43-142 intersectLineToTwoEllipses
bool intersect_line_two(int y, const Ellipse& qIn, const Ellipse& qOut, const EdgeSet& es, std::vector<int>& hull)
{
    float io[2], ii[2];
    const int no = geo::intersect_line(qOut, float(y), true, io);
    const int ni = geo::intersect_line(qIn, float(y), true, ii);
    auto take = [&](int x) {
        const int e = es.at(x, y);
        if (e < 0) return;
        const float cx = qIn.cx - float(es.x(e)), cy = qIn.cy - float(es.y(e));
        if (es.dx(e) * cx + es.dy(e) * cy < 0) hull.push_back(e);
    };
    if (no == 2 && ni == 2) {
        const int b1 = std::max(0, int(io[0])), e1 = std::min(es.W - 1, int(ii[0]));
        const int b2 = std::max(0, int(ii[1])), e2 = std::min(es.W - 1, int(io[1]));
        for (int x = b1; x <= e1; ++x) take(x);
        for (int x = b2; x <= e2; ++x) take(x);
    } else if (no == 2 && ni <= 1) {
        const int b = std::max(0, int(io[0])), e = std::min(es.W - 1, int(io[1]));
        for (int x = b; x <= e; ++x) take(x);
    } else if (no == 1 && ni == 0) {
        if (io[0] >= 0 && io[0] < float(es.W)) take(int(io[0]));
    } else {
        return false;
    }
    return true;
}

}  // namespace

void refit_hull(const MarkerCand& m, RefitHull& h)
{
    Ellipse qIn, qOut;
    geo::compute_hull(m.rescaled, m.scale, qIn, qOut);
    for (int k = 0; k < 9; ++k) {
        h.qin[k] = qIn.Q.m[k / 3][k % 3];
        h.qout[k] = qOut.Q.m[k / 3][k % 3];
    }
    h.inCx = qIn.cx;
    h.inCy = qIn.cy;
    h.yc = m.rescaled.cy;
}

void refit_apply(const EdgeSet& es0, MarkerCand& m, const int32_t* filtered, size_t n)
{
    if (n < 5) return;
    try {
        std::vector<int> f(filtered, filtered + n);
        const Ellipse fitted = fit_points(es0, f);
        std::vector<DirPoint> dp;
        dp.reserve(n);
        for (int e : f) dp.push_back({float(es0.x(e)), float(es0.y(e)), es0.dx(e), es0.dy(e)});
        m.cx_img *= m.scale;
        m.cy_img *= m.scale;
        m.rescaled = fitted;
        m.rescaled_points = std::move(dp);
    } catch (...) {
    }
}

void refit_on_level0(EdgeSet& es0, std::vector<MarkerCand>& markers, const ParallelFor& pf)
{
    pf(int(markers.size()), [&](int mi) {
        MarkerCand& m = markers[size_t(mi)];
        if (m.level > 0) {
            // each marker its own PCG32 stream, apart from the candidate loops'
            geo::Pcg32 rng = refit_rng(mi);
            RefitHull h;
            refit_hull(m, h);
            Ellipse qIn, qOut;
            qIn.cx = h.inCx;
            qIn.cy = h.inCy;
            for (int k = 0; k < 9; ++k) {
                qIn.Q.m[k / 3][k % 3] = h.qin[k];
                qOut.Q.m[k / 3][k % 3] = h.qout[k];
            }
            std::vector<int> hull;
            const int maxY = std::max(int(h.yc), 0);
            const int minY = std::min(int(h.yc), es0.H - 1);
            for (int y = maxY; y < es0.H; ++y)
                if (!intersect_line_two(y, qIn, qOut, es0, hull)) break;
            for (int y = minY; y >= 0; --y)
                if (!intersect_line_two(y, qIn, qOut, es0, hull)) break;
            if (hull.size() < 5) return;
            std::vector<int> filtered;
            float SmFinal = 1e+10f;
            outlier_removal(es0, hull, filtered, SmFinal, 20.0f, kNoWeight, 60, rng);
            refit_apply(es0, m, filtered.data(), filtered.size());
        } else {
            m.rescaled_points = m.points.empty() ? std::vector<DirPoint>() : m.points.back();
        }
    });
}

}  // namespace cctagb
