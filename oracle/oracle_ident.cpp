// TEST INFRASTRUCTURE ONLY -- CPU oracle for identification and end-to-end
// detection.
//
// Restates, on the CPU, the reference's identification path
// (Identification.cpp:50-1480, Identification.hpp:102-384, ImageCut.hpp,
// geometry/Ellipse.cpp:161-214,259-300, EllipseFromPoints.cpp:29-48,
// optimization/conditioner.hpp:22-44) and drives a whole detection:
// oracle image stage and vote (oracle_image.cpp), the candidate stage, this
// identification, duplicate removal and sort (Detection.cpp:773-999).
//
// The candidate stage (flow components, ellipse growing and fitting) is the
// oracle's own restatement (oracle_candidates.cpp).
//
// Identification is a template on the scalar type: with float it follows the
// reference's FP32 arithmetic and evaluation order (pairwise cut differences
// accumulated as the reference does, sample positions by repeated addition,
// sticky out-of-bounds flags); with double it is the FP64 localisation oracle.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <vector>

#include "oracle.h"
#include "oracle_internal.hpp"
#include "oracle_bank.hpp"
#include "oracle_cand.hpp"

namespace orc {

using DirPoint = DPt;
using MarkerCand = Marker;

template <class T>
struct M3T {
    T m[9];
};

template <class T>
M3T<T> mul3(const M3T<T>& a, const M3T<T>& b)
{
    M3T<T> r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i * 3 + j] = a.m[i * 3] * b.m[j] + a.m[i * 3 + 1] * b.m[3 + j] + a.m[i * 3 + 2] * b.m[6 + j];
    return r;
}

template <class T>
bool inv3(const M3T<T>& a, M3T<T>& r)
{
    const T* m = a.m;
    const T c00 = m[4] * m[8] - m[5] * m[7];
    const T c01 = m[5] * m[6] - m[3] * m[8];
    const T c02 = m[3] * m[7] - m[4] * m[6];
    const T det = m[0] * c00 + m[1] * c01 + m[2] * c02;
    if (det == T(0) || !std::isfinite(det)) return false;
    const T id = T(1) / det;
    r.m[0] = c00 * id;
    r.m[1] = (m[2] * m[7] - m[1] * m[8]) * id;
    r.m[2] = (m[1] * m[5] - m[2] * m[4]) * id;
    r.m[3] = c01 * id;
    r.m[4] = (m[0] * m[8] - m[2] * m[6]) * id;
    r.m[5] = (m[2] * m[3] - m[0] * m[5]) * id;
    r.m[6] = c02 * id;
    r.m[7] = (m[1] * m[6] - m[0] * m[7]) * id;
    r.m[8] = (m[0] * m[4] - m[1] * m[3]) * id;
    return true;
}

// Identification.hpp:102-113
template <class T>
void apply_h(const M3T<T>& H, T x, T y, T& ox, T& oy)
{
    const T u = H.m[0] * x + H.m[1] * y + H.m[2];
    const T v = H.m[3] * x + H.m[4] * y + H.m[5];
    const T w = H.m[6] * x + H.m[7] * y + H.m[8];
    ox = u / w;
    oy = v / w;
}

// Identification.hpp:197-219
template <class T>
T bilinear(const uint8_t* img, int W, T x, T y)
{
    const int px = int(x), py = int(y);
    const uint8_t* p0 = img + px + size_t(py) * W;
    const T fx = x - T(px), fy = y - T(py);
    const T fx1 = T(1) - fx, fy1 = T(1) - fy;
    const T w1 = fx1 * fy1, w2 = fx * fy1, w3 = fx1 * fy, w4 = fx * fy;
    return (T(p0[0]) * w1 + T(p0[1]) * w2 + T(p0[W]) * w3 + T(p0[W + 1]) * w4) / 2;
}

template <class T>
struct Ell {
    T cx, cy, a, b, angle;
    M3T<T> Q;
};

// Ellipse.cpp:161-214
template <class T>
void canonic(const Ell<T>& e, M3T<T>& C, M3T<T>& Tp, M3T<T>& Td)
{
    const T* Q = e.Q.m;
    const T q1 = Q[0], q2 = Q[1], q3 = Q[2], q4 = Q[4], q5 = Q[5], q6 = Q[8];
    const T par1 = q1, par2 = 2 * q2, par3 = q4, par4 = 2 * q3, par5 = 2 * q5;
    const T th = T(0.5) * std::atan2(par2, par1 - par3);
    const T ct = std::cos(th), st = std::sin(th);
    const T s2 = st * st, c2 = ct * ct, cs = st * ct;
    const T Au = par4 * ct + par5 * st, Av = -par4 * st + par5 * ct;
    const T Auu = par1 * c2 + par3 * s2 + par2 * cs, Avv = par1 * s2 + par3 * c2 - par2 * cs;
    const T tu = -Au / (2 * Auu), tv = -Av / (2 * Avv);
    const T uc = tu * ct - tv * st, vc = tu * st + tv * ct;
    const T t1 = ct * (ct * q1 + q2 * st) + st * (ct * q2 + q4 * st);
    const T t2 = ct * (ct * q2 + q4 * st) - st * (ct * q1 + q2 * st);
    const T t3 = ct * q3 + q5 * st + uc * (ct * q1 + q2 * st) + vc * (ct * q2 + q4 * st);
    const T t4 = ct * (ct * q4 - q2 * st) - st * (ct * q2 - q1 * st);
    const T t5 = ct * q5 - q3 * st + uc * (ct * q2 - q1 * st) + vc * (ct * q4 - q2 * st);
    const T t6 = q6 + uc * (q3 + q1 * uc + q2 * vc) + vc * (q5 + q2 * uc + q4 * vc) + q3 * uc + q5 * vc;
    const T c[9] = {t1, t2, t3, t2, t4, t5, t3, t5, t6};
    const T tp[9] = {ct, st, -ct * uc - st * vc, -st, ct, st * uc - ct * vc, 0, 0, ct * ct + st * st};
    const T td[9] = {ct, -st, uc, st, ct, vc, 0, 0, T(1)};
    for (int k = 0; k < 9; ++k) {
        C.m[k] = c[k];
        Tp.m[k] = tp[k];
        Td.m[k] = td[k];
    }
}

// Identification.cpp:739-798
template <class T>
M3T<T> homography(const M3T<T>& C, const M3T<T>& Tp, const M3T<T>& Td, T x, T y)
{
    T xc, yc;
    apply_h(Tp, x, y, xc, yc);
    const T Q11 = C.m[0], Q22 = C.m[4], Q33 = C.m[8];
    M3T<T> h;
    h.m[0] = Q33;       h.m[1] = Q22 * xc * yc;        h.m[2] = -Q33 * xc;
    h.m[3] = 0;         h.m[4] = -Q11 * xc * xc - Q33; h.m[5] = -Q33 * yc;
    h.m[6] = -Q11 * xc; h.m[7] = Q22 * yc;             h.m[8] = -Q33;
    const T d[3] = {std::sqrt((Q22 * Q33 / Q11 * (Q11 * xc * xc + Q22 * yc * yc + Q33))), Q33,
                    std::sqrt(-Q22 * (Q11 * xc * xc + Q33))};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) h.m[i * 3 + j] *= d[j];
    return mul3(Td, h);
}

// Ellipse.cpp:103-159, semi axes only
template <class T>
void axes_of(const M3T<T>& Qm, T& a, T& b)
{
    const T* Q = Qm.m;
    const T p0 = Q[0], p1 = 2 * Q[1], p2 = Q[4], p3 = 2 * Q[2], p4 = 2 * Q[5], p5 = Q[8];
    const T th = T(0.5) * std::atan2(p1, p0 - p2);
    const T ct = std::cos(th), st = std::sin(th);
    const T s2 = st * st, c2 = ct * ct, cs = st * ct;
    const T Au = p3 * ct + p4 * st, Av = -p3 * st + p4 * ct;
    const T Auu = p0 * c2 + p2 * s2 + p1 * cs, Avv = p0 * s2 + p2 * c2 - p1 * cs;
    if (Auu == T(0) || Avv == T(0)) {
        a = b = 0;
        return;
    }
    const T tu = -Au / (2 * Auu), tv = -Av / (2 * Avv);
    const T wc = p5 - Auu * tu * tu - Avv * tv * tv;
    a = std::sqrt(std::fabs(-wc / Auu));
    b = std::sqrt(std::fabs(-wc / Avv));
}

template <class T>
struct Cut {
    T sx, sy;  // stop
    std::vector<T> sig;
    bool oob = false;
};

// Identification.cpp:216-280 extractSignalUsingHomography (begin != 0, end == 1)
template <class T>
void extract(Cut<T>& c, const uint8_t* img, int W, int H, const M3T<T>& Hm, const M3T<T>& Hi, T beginSig, int n)
{
    T bx, by;
    apply_h(Hi, c.sx, c.sy, bx, by);
    const T xs = bx * beginSig, ys = by * beginSig;
    const T stepX = (bx - xs) / (T(n) - T(1)), stepY = (by - ys) / (T(n) - T(1));
    T x = xs, y = ys;
    for (int i = 0; i < n; ++i) {
        T xr, yr;
        apply_h(Hm, x, y, xr, yr);
        if (xr >= T(0) && xr < T(W - 1) && yr >= T(0) && yr < T(H - 1)) c.sig[i] = bilinear(img, W, xr, yr);
        else c.oob = true;
        x += stepX;
        y += stepY;
    }
}

// Identification.cpp:1122-1158 costFunctionGlob.  The FP32 form accumulates
// std::pow(float, int) (a double) into a float, as the reference.
template <class T>
T cost(std::vector<Cut<T>>& cuts, const uint8_t* img, int W, int H, const M3T<T>& Hm, T beginSig, int n, bool& flag)
{
    flag = true;
    M3T<T> Hi;
    if (!inv3(Hm, Hi)) {
        flag = false;
        return std::numeric_limits<T>::max();
    }
    for (auto& c : cuts) extract(c, img, W, H, Hm, Hi, beginSig, n);
    T res = 0;
    size_t resSize = 0;
    for (size_t i = 0; i + 1 < cuts.size(); ++i)
        for (size_t j = i + 1; j < cuts.size(); ++j)
            if (!cuts[i].oob && !cuts[j].oob) {
                for (int k = 0; k < n; ++k) {
                    const T d = cuts[i].sig[k] - cuts[j].sig[k];
                    res = T(double(res) + double(d) * double(d));
                }
                ++resSize;
            }
    if (resSize == 0) {
        flag = false;
        return std::numeric_limits<T>::max();
    }
    return res / T(resSize);
}

// Identification.hpp:351-371 computeMedian
template <class T>
T median_of(std::vector<T> v)
{
    const size_t s = v.size() / 2 + 1;
    std::vector<T> out(s);
    std::partial_sort_copy(v.begin(), v.end(), out.begin(), out.end());
    if (v.size() % 2) return out.back();
    return T((double(out[s - 1]) + double(out[s - 2])) / 2.0);
}

struct IdentOut {
    int status = 0, id = -1;
    double x = 0, y = 0, residual = 0, score = 0;
    double H[9] = {};
};

// Identification.cpp:813-965 refineConicFamilyGlob (+ :980-1109) then
// :50-193 orazioDistanceRobust and :1408-1436 ID vote.
template <class T>
IdentOut identify_step2(const uint8_t* img, int W, int H, const Ell<T>& e, T x0, T y0,
                        const std::vector<std::pair<float, float>>& stops, const cctagb_params& p,
                        const std::vector<std::vector<float>>& bank)
{
    IdentOut out;
    const int n = p.sampleCutLength;
    const T beginSig = T(1 - float(2 * p.nCrowns - 1) * 0.15f);
    std::vector<Cut<T>> cuts(stops.size());
    for (size_t i = 0; i < stops.size(); ++i) {
        cuts[i].sx = stops[i].first;
        cuts[i].sy = stops[i].second;
        cuts[i].sig.assign(size_t(n), T(0));
    }
    M3T<T> C, Tp, Td;
    canonic(e, C, Tp, Td);
    // conditioner (meanAB of this ellipse; the reference keeps the first
    // ellipse's value in a function-local static, which cancels up to rounding)
    const T sqrt2 = std::sqrt(T(2));
    const T meanAB = (e.a + e.b) / T(2);
    M3T<T> mT{{sqrt2 / meanAB, 0, -sqrt2 * e.cx / meanAB, 0, sqrt2 / meanAB, -sqrt2 * e.cy / meanAB, 0, 0, T(1)}};
    M3T<T> mTi;
    inv3(mT, mTi);
    M3T<T> mTiT;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) mTiT.m[i * 3 + j] = mTi.m[j * 3 + i];
    const M3T<T> Qc = mul3(mTiT, mul3(e.Q, mTi));
    T ca, cb;
    axes_of(Qc, ca, cb);
    const int gridN = p.imagedCenterNGridSample;
    T ns = T(p.imagedCenterNeighbourSize);
    const T maxSemi = std::max(e.a, e.b);
    T cx = x0, cy = y0;
    M3T<T> Hopt{};
    T minRes = std::numeric_limits<T>::max();
    while (ns * maxSemi > T(0.02)) {
        const T size = ns * std::max(ca, cb);
        const T half = size / T(2), step = size / T(gridN - 1);
        const T ccx = mT.m[0] * cx + mT.m[1] * cy + mT.m[2];
        const T ccy = mT.m[3] * cx + mT.m[4] * cy + mT.m[5];
        bool has = false;
        T best = std::numeric_limits<T>::max();
        T bx = cx, by = cy;
        M3T<T> bH{};
        for (int i = 0; i < gridN; ++i)
            for (int j = 0; j < gridN; ++j) {
                T px, py;
                apply_h(mTi, ccx - half + T(i) * step, ccy - half + T(j) * step, px, py);
                const M3T<T> Hm = homography(C, Tp, Td, px, py);
                bool readable;
                const T r = cost(cuts, img, W, H, Hm, beginSig, n, readable);
                if (readable) {
                    has = true;
                    if (r < best) {
                        best = r;
                        bx = px;
                        by = py;
                        bH = Hm;
                    }
                }
            }
        if (!has) {
            out.status = CCTAGB_OPTI_HAS_DIVERGED;
            out.x = double(cx);
            out.y = double(cy);
            return out;
        }
        cx = bx;
        cy = by;
        Hopt = bH;
        minRes = best;
        ns /= T((gridN - 1) / 2);
    }
    out.x = double(cx);
    out.y = double(cy);
    for (int k = 0; k < 9; ++k) out.H[k] = double(Hopt.m[k]);
    M3T<T> Hi;
    inv3(Hopt, Hi);
    for (auto& c : cuts) extract(c, img, W, H, Hopt, Hi, beginSig, n);
    std::vector<size_t> ok;
    for (size_t i = 0; i < cuts.size(); ++i)
        if (!cuts[i].oob) ok.push_back(i);
    std::vector<T> bar(static_cast<size_t>(n));
    std::vector<T> col(ok.size());
    for (int k = 0; k < n; ++k) {
        for (size_t q = 0; q < ok.size(); ++q) col[q] = cuts[ok[q]].sig[k];
        bar[k] = ok.empty() ? T(0) : median_of(col);
    }
    const T mag = *std::max_element(bar.begin(), bar.end()) - *std::min_element(bar.begin(), bar.end());
    const T residual = std::sqrt(minRes) / mag;
    out.residual = double(residual);
    if (residual > T(2.7f) || !(residual == residual)) {
        out.status = CCTAGB_OPTI_HAS_DIVERGED;
        return out;
    }
    // Orazio distance per cut (FP32 statistics as the reference in both variants)
    std::vector<std::vector<float>> votes(bank.size());
    const float stepX = (1.f - float(beginSig)) / (float(n) - 1.f);
    for (size_t q = 0; q < ok.size(); ++q) {
        const Cut<T>& c = cuts[ok[q]];
        std::vector<float> sg(c.sig.begin(), c.sig.end());
        float mean = 0.f, var = 0.f;
        int cnt = 0;
        for (int k = 30; k < n; ++k) {
            ++cnt;
            mean = (mean * float(cnt - 1) + sg[k]) / float(cnt);
            if (cnt > 1) {
                const float t = sg[k] - mean;
                var = var * float(cnt - 1) / float(cnt) + t * t / float(cnt - 1);
            }
        }
        float mub = 0.f, muw = 0.f;
        int ni = 0, nsup = 0;
        bool acc = false;
        for (int k = 0; k < n; ++k) {
            if (!acc && sg[k] < mean) acc = true;
            if (acc) {
                if (sg[k] < mean) {
                    ++ni;
                    mub = (mub * float(ni - 1) + sg[k]) / float(ni);
                } else {
                    ++nsup;
                    muw = (muw * float(nsup - 1) + sg[k]) / float(nsup);
                }
            }
        }
        std::map<float, int> sorted;
        for (size_t idc = 0; idc < bank.size(); ++idc) {
            float x = float(beginSig), dist = 0.f;
            for (int k = 0; k < n; ++k) {
                int ldum = 0;
                for (float r : bank[idc])
                    if (1.f / r <= x) ++ldum;
                const float digit = float(-(ldum % 2) * 2 + 1);
                float d;
                if (digit == -1.f) {
                    const float t = std::max(sg[k] - mub, 0.f);
                    d = t * t / (2.0f * var);
                } else {
                    const float t = std::min(sg[k] - muw, 0.f);
                    d = t * t / (2.0f * var);
                }
                dist += d;
                x += stepX;
            }
            sorted[std::exp(-dist)] = int(idc);
        }
        votes[sorted.rbegin()->second].push_back(sorted.rbegin()->first);
    }
    int iMax = 0;
    size_t maxSize = 0;
    for (size_t i = 0; i < votes.size(); ++i)
        if (votes[i].size() > maxSize) {
            iMax = int(i);
            maxSize = votes[i].size();
        }
    float score = 0;
    for (float v : votes[iMax]) score += v;
    score /= float(votes[iMax].size());
    out.id = iMax;
    out.score = score;
    out.status = score > p.minIdentProba ? CCTAGB_ID_RELIABLE : CCTAGB_ID_NOT_RELIABLE;
    return out;
}

// ------------------------------------------- identify_step_1 (restated) --
float bil_f(const uint8_t* img, int W, float x, float y) { return bilinear<float>(img, W, x, y); }

bool cut_interp(const uint8_t* img, int W, int H, float sx, float sy, float ex, float ey, float beginSig, int n,
                float* sig)
{
    float xs = sx, ys = sy;
    if (beginSig != 0.f) {
        xs = sx + (ex - sx) * beginSig;
        ys = sy + (ey - sy) * beginSig;
    }
    const float stepX = (ex - xs) / (float(n) - 1.f), stepY = (ey - ys) / (float(n) - 1.f);
    float x = xs, y = ys;
    for (int i = 0; i < n; ++i) {
        if (!(x >= 1.f && x < float(W - 1) && y >= 1.f && y < float(H - 1))) return false;
        sig[i] = bil_f(img, W, x, y);
        x += stepX;
        y += stepY;
    }
    return true;
}

int identify_step1(const MarkerCand& m, const uint8_t* img, int W, int H, const cctagb_params& p,
                   std::vector<std::pair<float, float>>& stops)
{
    const gm::Ellipse& e = m.rescaled;
    const auto& pts = m.rescaled_points;
    // Ellipse.cpp:259-300
    std::vector<std::pair<float, size_t>> ang;
    for (size_t i = 0; i < pts.size(); ++i) ang.emplace_back(std::atan2(pts[i].y - e.cy, pts[i].x - e.cx), i);
    std::sort(ang.begin(), ang.end());
    const size_t nOuter = std::min(size_t(p.nSamplesOuterEllipse), pts.size());
    if (nOuter < 2) return CCTAGB_TOO_FEW_OUTER_POINTS;  // the step would divide by zero
    const float stepO = std::max(1.f, float(pts.size()) / float(nOuter - 1));
    std::vector<DirPoint> outer;
    for (size_t k = 0;; ++k) {
        const size_t i = size_t(float(k) * stepO);
        if (i >= ang.size()) break;
        outer.push_back(pts[ang[i].second]);
    }
    if (outer.size() < 5) return CCTAGB_TOO_FEW_OUTER_POINTS;
    // Identification.cpp:1221-1235: the signal starts at startSig of the radius
    const float beginSig = p.nCrowns == 3 ? 1 - float(2 * p.nCrowns - 1) * 0.15f : (p.nCrowns == 4 ? 0.26f : 0.f);
    const int n = p.sampleCutLength;
    std::vector<DirPoint> cstop;
    std::vector<float> cvar;
    std::vector<float> sig(static_cast<size_t>(n));
    for (const DirPoint& op : outer) {
        if (!cut_interp(img, W, H, e.cx, e.cy, op.x, op.y, beginSig, n, sig.data())) continue;
        float mean = 0.f, var = 0.f;
        for (int k = 0; k < n; ++k) {
            mean = (mean * float(k) + sig[k]) / float(k + 1);
            if (k > 0) {
                const float t = sig[k] - mean;
                var = var * float(k) / float(k + 1) + t * t / float(k);
            }
        }
        cstop.push_back(op);
        cvar.push_back(var);
    }
    if (cstop.empty()) return CCTAGB_NO_COLLECTED_CUTS;
    const size_t selectSize = std::min(size_t(p.numCutsInIdentStep), cstop.size());
    const float varMax = *std::max_element(cvar.begin(), cvar.end());
    std::vector<size_t> keep;
    const int nr = p.numSamplesOuterEdgePointsRefinement;
    std::vector<float> rs(static_cast<size_t>(nr));
    for (size_t i = 0; i < cstop.size(); ++i) {
        DirPoint& s = cstop[i];
        // EllipseFromPoints.cpp:29-48 pointOnEllipse
        {
            const float x = s.x - e.cx, y = s.y - e.cy;
            float tx = x * std::cos(e.angle) + y * std::sin(e.angle);
            float ty = -x * std::sin(e.angle) + y * std::cos(e.angle);
            const float cs = std::sqrt(tx * tx / (e.a * e.a) + ty * ty / (e.b * e.b));
            tx /= cs;
            ty /= cs;
            s.x = tx * std::cos(e.angle) - ty * std::sin(e.angle) + e.cx;
            s.y = tx * std::sin(e.angle) + ty * std::cos(e.angle) + e.cy;
        }
        // Identification.cpp:604-657 outerEdgeRefinement
        const float len = 3.f * std::sqrt(2.f) * m.scale, hw = len / 2.f;
        const float gn = std::sqrt(s.dx * s.dx + s.dy * s.dy);
        const float gx = s.dx / gn, gy = s.dy / gn;
        const float ax = s.x - hw * gx, ay = s.y - hw * gy;
        if (!cut_interp(img, W, H, ax, ay, s.x + hw * gx, s.y + hw * gy, 0.f, nr, rs.data())) continue;
        static const float kk[3][9] = {
            {-0.0000f, -0.0003f, -0.1065f, -0.7863f, .0f, 0.7863f, 0.1065f, 0.0003f, 0.0000f},
            {-0.0044f, -0.0540f, -0.2376f, -0.3450f, .0f, 0.3450f, 0.2376f, 0.0540f, 0.0044f},
            {-0.0366f, -0.1113f, -0.1801f, -0.1594f, .0f, 0.1594f, 0.1801f, 0.1113f, 0.0366f}};
        std::map<float, float> res;
        for (int q = 0; q < 3; ++q) {
            std::vector<float> o(static_cast<size_t>(nr));
            for (int a = 0; a < nr; ++a) {
                float t = 0;
                for (int j = 0; j < 9; ++j) {
                    const int r = a - 4 + j;
                    t += rs[r < 0 ? 0 : (r >= nr ? nr - 1 : r)] * kk[q][j];
                }
                o[a] = t;
            }
            const auto it = std::max_element(o.begin(), o.end());
            res.insert({*it, float(it - o.begin())});
        }
        const float stp = len / (float(nr) - 1.f);
        s.x = ax + stp * res.rbegin()->second * gx;
        s.y = ay + stp * res.rbegin()->second * gy;
        if (cvar[i] / varMax > 0.5f) keep.push_back(i);
    }
    const float step = std::max(1.f, float(keep.size()) / float(selectSize));
    stops.clear();
    for (size_t k = 0;; ++k) {
        const size_t i = size_t(float(k) * step);
        if (i < keep.size() && stops.size() < selectSize) stops.push_back({cstop[keep[i]].x, cstop[keep[i]].y});
        else break;
    }
    if (stops.empty()) return CCTAGB_NO_SELECTED_CUTS;
    return CCTAGB_ID_RELIABLE;
}

// CCTag::isEqual (CCTag.cpp:42-57) and update (Multiresolution.cpp:172-193)
bool overlap(const MarkerCand& A, const MarkerCand& B)
{
    auto inside = [](const gm::Ellipse& big, float x, float y) {
        const gm::Ellipse e = gm::ellipse_from_params(big.cx, big.cy, big.b * 0.5f, big.b * 0.5f, big.angle);
        const float s1 = gm::quad(e.Q, x, y);
        const float q0 = e.Q.v[0][0] * e.cx + e.Q.v[0][1] * e.cy + e.Q.v[0][2];
        const float q1 = e.Q.v[1][0] * e.cx + e.Q.v[1][1] * e.cy + e.Q.v[1][2];
        const float q2 = e.Q.v[2][0] * e.cx + e.Q.v[2][1] * e.cy + e.Q.v[2][2];
        return s1 * (x * q0 + y * q1 + q2) > 0;
    };
    return inside(A.rescaled, B.rescaled.cx, B.rescaled.cy) || inside(B.rescaled, A.rescaled.cx, A.rescaled.cy);
}

void update(std::vector<MarkerCand>& list, const MarkerCand& m)
{
    bool flag = false;
    for (auto& c : list)
        if (c.status > 0 && m.status > 0 && overlap(c, m)) {
            if (m.quality > c.quality) c = m;
            flag = true;
        }
    if (!flag) list.push_back(m);
}

}  // namespace orc

namespace orc {
struct StepOneRec {
    int status;
    std::vector<std::pair<float, float>> stops;
};
}  // namespace orc

static int detect_impl(const uint8_t* gray, int W, int H, const cctagb_params* pp, int fp64, orc_marker* out, int cap,
                       std::vector<orc::StepOneRec>* rec, std::vector<orc::LoopTwoRecord>* l2 = nullptr)
{
    using namespace orc;
    const cctagb_params& p = *pp;
    std::vector<std::vector<float>> bank;
    for (const auto& row : kBankThreeCrowns) bank.emplace_back(row, row + 5);
    const int nl = p.numberOfProcessedMultiresLayers;
    std::vector<std::vector<uint8_t>> lvl(nl);
    std::vector<int> lw(nl), lh(nl);
    lvl[0].assign(gray, gray + size_t(W) * H);
    lw[0] = W;
    lh[0] = H;
    for (int l = 1; l < nl; ++l) {
        lw[l] = lw[l - 1] / 2;
        lh[l] = lh[l - 1] / 2;
        lvl[l].resize(size_t(lw[l]) * lh[l]);
        pyramid_down(lvl[l - 1].data(), lw[l - 1], lh[l - 1], lvl[l].data(), lw[l], lh[l]);
    }
    std::vector<EdgeCollection> ec(static_cast<size_t>(nl));
    std::vector<std::vector<int>> seeds(static_cast<size_t>(nl));
    std::vector<MarkerCand> markers;
    const float lo = p.cannyThrLow * 256.f, hi = p.cannyThrHigh * 256.f;
    for (int l = 0; l < nl; ++l) {
        const int w = lw[l], h = lh[l];
        std::vector<int16_t> dx(size_t(w) * h), dy(size_t(w) * h);
        std::vector<uint8_t> e(size_t(w) * h);
        derivatives(lvl[l].data(), w, h, dx.data(), dy.data());
        canny(dx.data(), dy.data(), w, h, lo, hi, e.data(), nullptr);
        thin(e.data(), w, h);
        const int cap_e = w * h;
        std::vector<int32_t> x(cap_e), y(cap_e), b(cap_e), a(cap_e), ch(cap_e), nv(cap_e), im(cap_e), vo(cap_e + 1),
            vl(cap_e), sp(cap_e), ss(cap_e);
        std::vector<float> tot(cap_e), fl(cap_e);
        int32_t ns = 0;
        VoteParams vp{p.distSearch, p.thrGradientMagInVote, p.angleVoting, p.ratioVoting, p.nCrowns,
                      p.minVotesToSelectCandidate};
        const int E = vote(e.data(), dx.data(), dy.data(), w, h, vp, cap_e, x.data(), y.data(), b.data(), a.data(),
                           ch.data(), tot.data(), nv.data(), im.data(), fl.data(), vo.data(), vl.data(), sp.data(),
                           ss.data(), &ns);
        ec[size_t(l)].build(w, h, x.data(), y.data(), dx.data(), dy.data(), E, b.data(), a.data(), vo.data(), vl.data(),
                            fl.data());
        seeds[size_t(l)].assign(ss.begin(), ss.begin() + ns);
    }
    if (l2) {  // loop 1 and the outlier removal only
        l2->assign(size_t(nl), {});
        std::vector<MarkerCand> none;
        for (int l = 0; l < nl; ++l)
            candidates_from_edges(ec[size_t(l)], seeds[size_t(l)], l, float(1 << l), p, none, &(*l2)[size_t(l)]);
        return 0;
    }
    // Multiresolution.cpp:272-300: levels from the coarsest down
    for (int l = nl - 1; l >= 0; --l)
        candidates_from_edges(ec[size_t(l)], seeds[size_t(l)], l, float(1 << l), p, markers, nullptr);
    refit_on_level0(ec[0], markers);
    if (p.doIdentification) {
        for (auto& m : markers) {
            std::vector<std::pair<float, float>> stops;
            const int st = identify_step1(m, gray, W, H, p, stops);
            m.status = st;
            if (rec) rec->push_back({st, stops});
            if (st != CCTAGB_ID_RELIABLE) continue;
            IdentOut r;
            if (fp64) {
                Ell<double> e{m.rescaled.cx, m.rescaled.cy, m.rescaled.a, m.rescaled.b, m.rescaled.angle, {}};
                for (int k = 0; k < 9; ++k) e.Q.m[k] = m.rescaled.Q.v[k / 3][k % 3];
                // recompute the conic in FP64 from the parameters
                {
                    const double c = std::cos(e.angle), s = std::sin(e.angle);
                    const double Ri[9] = {c, s, -(c * e.cx + s * e.cy), -s, c, s * e.cx - c * e.cy, 0, 0, 1};
                    const double D[3] = {1.0 / (e.a * e.a), 1.0 / (e.b * e.b), -1.0};
                    for (int i = 0; i < 3; ++i)
                        for (int j = 0; j < 3; ++j) {
                            double v = 0;
                            for (int k = 0; k < 3; ++k) v += Ri[k * 3 + i] * D[k] * Ri[k * 3 + j];
                            e.Q.m[i * 3 + j] = v;
                        }
                }
                r = identify_step2<double>(gray, W, H, e, m.cx_img, m.cy_img, stops, p, bank);
            } else {
                Ell<float> e{m.rescaled.cx, m.rescaled.cy, m.rescaled.a, m.rescaled.b, m.rescaled.angle, {}};
                for (int k = 0; k < 9; ++k) e.Q.m[k] = m.rescaled.Q.v[k / 3][k % 3];
                r = identify_step2<float>(gray, W, H, e, m.cx_img, m.cy_img, stops, p, bank);
            }
            m.status = r.status;
            m.cx_img = float(r.x);
            m.cy_img = float(r.y);
            m.quality = float(1.0 / r.residual);
            if (r.status != CCTAGB_OPTI_HAS_DIVERGED) m.id = r.id;
            for (int k = 0; k < 9; ++k) m.H[k] = float(r.H[k]);
        }
    }
    std::vector<MarkerCand> pre, fin;
    for (const auto& m : markers) update(pre, m);
    for (const auto& m : pre) update(fin, m);
    std::stable_sort(fin.begin(), fin.end(), [](const MarkerCand& a, const MarkerCand& b) { return a.id < b.id; });
    const int n = std::min(cap, int(fin.size()));
    for (int i = 0; i < n; ++i) {
        out[i].id = fin[i].id;
        out[i].status = fin[i].status;
        out[i].x = fin[i].cx_img;
        out[i].y = fin[i].cy_img;
        out[i].cx = fin[i].rescaled.cx;
        out[i].cy = fin[i].rescaled.cy;
        out[i].a = fin[i].rescaled.a;
        out[i].b = fin[i].rescaled.b;
        out[i].angle = fin[i].rescaled.angle;
        out[i].quality = fin[i].quality;
        out[i].level = fin[i].level;
    }
    return int(fin.size());
}

// Parameters::Parameters(nCrowns) defaults (Params.hpp:27-66, Params.cpp:38-75).
extern "C" int orc_detect(const uint8_t* gray, int W, int H, const cctagb_params* pp, int fp64, orc_marker* out,
                          int cap)
{
    return detect_impl(gray, W, H, pp, fp64, out, cap, nullptr);
}

// The identify_step_1 outcome of every candidate, in candidate order: its
// status and the selected cut ends (cap_cuts pairs per candidate).
extern "C" int orc_cut_selection(const uint8_t* gray, int W, int H, const cctagb_params* pp, int* status, int* ncuts,
                                 float* stops, int cap_cuts, int cap)
{
    std::vector<orc::StepOneRec> rec;
    detect_impl(gray, W, H, pp, 0, nullptr, 0, &rec);
    const int n = std::min(cap, int(rec.size()));
    for (int i = 0; i < n; ++i) {
        status[i] = rec[size_t(i)].status;
        const int k = std::min(cap_cuts, int(rec[size_t(i)].stops.size()));
        ncuts[i] = rec[size_t(i)].status == CCTAGB_ID_RELIABLE ? k : 0;
        for (int j = 0; j < k; ++j) {
            stops[(size_t(i) * cap_cuts + j) * 2] = rec[size_t(i)].stops[size_t(j)].first;
            stops[(size_t(i) * cap_cuts + j) * 2 + 1] = rec[size_t(i)].stops[size_t(j)].second;
        }
    }
    return int(rec.size());
}

// Loop 1 and the outlier removal of loop 2 (host restatement) for one level:
// the layout of cctagb_level_loop_two.
extern "C" int orc_loop_two(const uint8_t* gray, int W, int H, const cctagb_params* pp, int level, int cap,
                            int32_t* seed, int32_t* score, int32_t* keep, int32_t* n_filtered, int filtered_cap,
                            int32_t* filtered, int* n_filtered_total)
{
    std::vector<orc::LoopTwoRecord> l2;
    detect_impl(gray, W, H, pp, 0, nullptr, 0, nullptr, &l2);
    if (level < 0 || level >= int(l2.size())) return -1;
    const orc::LoopTwoRecord& g = l2[size_t(level)];
    const int n = int(g.seed.size());
    if (n > cap || int(g.flt.size()) > filtered_cap) return -1;
    for (int i = 0; i < n; ++i) {
        seed[i] = g.seed[size_t(i)];
        score[i] = g.score[size_t(i)];
        keep[i] = g.keep[size_t(i)];
        n_filtered[i] = g.foff[size_t(i) + 1] - g.foff[size_t(i)];
    }
    std::copy(g.flt.begin(), g.flt.end(), filtered);
    *n_filtered_total = int(g.flt.size());
    return n;
}

extern "C" void orc_params_default(cctagb_params* p, int nCrowns)
{
    std::memset(p, 0, sizeof(*p));
    p->cannyThrLow = 0.01f;
    p->cannyThrHigh = 0.04f;
    p->distSearch = 30;
    p->thrGradientMagInVote = 2500;
    p->angleVoting = 0.f;
    p->ratioVoting = 4.f;
    p->averageVoteMin = 0.f;
    p->thrMedianDistanceEllipse = 3.f;
    p->maximumNbSeeds = 500;
    p->maximumNbCandidatesLoopTwo = 40;
    p->nCrowns = nCrowns;
    p->nCircles = 2 * nCrowns;
    p->minPointsSegmentCandidate = 10;
    p->minVotesToSelectCandidate = 3;
    p->threshRobustEstimationOfOuterEllipse = 30.f;
    p->ellipseGrowingEllipticHullWidth = 2.3f;
    p->windowSizeOnInnerEllipticSegment = 20;
    p->numberOfMultiresLayers = 4;
    p->numberOfProcessedMultiresLayers = 4;
    p->nSamplesOuterEllipse = 150;
    p->numCutsInIdentStep = 22;
    p->numSamplesOuterEdgePointsRefinement = 20;
    p->cutsSelectionTrials = 500;
    p->sampleCutLength = 100;
    p->imagedCenterNGridSample = 5;
    p->imagedCenterNeighbourSize = 0.20f;
    p->minIdentProba = 1e-6f;
    p->useLMDif = 1;
    p->searchForAnotherSegment = 1;
    p->doIdentification = 1;
    p->maxEdges = 20000;
}
