// TEST INFRASTRUCTURE ONLY -- the oracle's geometry for the candidate stage:
// ellipses as parameters and conic matrix, point-conic distance, hulls,
// rasterised perimeters, line intersections, medians, the PCG32 generator
// and the two point fits.  Restated from the reference's geometry sources
// (geometry/Ellipse.cpp, geometry/Distance.cpp, geometry/EllipseFromPoints.cpp,
// EllipseGrowing.hpp, Statistic.cpp/.hpp, Fitting.cpp) in the reference's FP32
// arithmetic, independently of the library's own geometry code.
//
// Where the reference's arithmetic lives in a third-party library whose last
// bits depend on the platform, the oracle pins it the way the library does:
//  * libm's float sin / cos / atan2 -> the correctly rounded float (the double
//    function of the C library, rounded once);
//  * Eigen's float 5x5 LU solve of the LMedS conic -> an FP64 Gaussian
//    elimination with partial pivoting (first largest pivot, row operations
//    in column order, back substitution from the last row);
//  * Eigen's EigenSolver / JacobiSVD inside the two fits -> the FP64 cores of
//    include/cctag_b200/portable/fit_core.hpp (whose eigen recipe is checked
//    against an independent float64 solver in the tests);
//  * medianRef's std::sort on values that may hold NaN -> NaN ordered last.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "cctag_b200/portable/fit_core.hpp"

namespace orc {
namespace gm {

inline float sin_cr(float x) { return float(std::sin(double(x))); }
inline float cos_cr(float x) { return float(std::cos(double(x))); }
inline float atan2_cr(float y, float x) { return float(std::atan2(double(y), double(x))); }

constexpr float kPi = 3.14159265358979323846f;  // boost::math::constants::pi<float>()

struct M3 {
    float v[3][3];
};

inline M3 m3_zero()
{
    M3 z;
    std::memset(&z, 0, sizeof z);
    return z;
}

// Eigen's lazy 3x3 product: r(i, j) = (a(i,0) b(0,j) + a(i,1) b(1,j)) + a(i,2) b(2,j).
inline M3 m3_mul(const M3& a, const M3& b)
{
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.v[i][j] = a.v[i][0] * b.v[0][j] + a.v[i][1] * b.v[1][j] + a.v[i][2] * b.v[2][j];
    return r;
}

inline M3 m3_t(const M3& a)
{
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.v[i][j] = a.v[j][i];
    return r;
}

// numerical::geometry::Ellipse (geometry/Ellipse.hpp): parameters and matrix.
struct Ellipse {
    float cx = 0.f, cy = 0.f, a = 0.f, b = 0.f, angle = 0.f;
    M3 Q = m3_zero();
};

// Ellipse::computeMatrix (Ellipse.cpp:229-251): Q = R^-T diag(1/a^2, 1/b^2, -1)
// R^-1 with R = [cos -sin cx; sin cos cy; 0 0 1].  R^-1 is taken in closed form
// (the library's choice too; Eigen would divide its cofactors by a determinant
// that rounds near 1).
inline void compute_matrix(Ellipse& e)
{
    const float c = cos_cr(e.angle), s = sin_cr(e.angle);
    M3 ri;
    ri.v[0][0] = c;
    ri.v[0][1] = s;
    ri.v[0][2] = -(c * e.cx + s * e.cy);
    ri.v[1][0] = -s;
    ri.v[1][1] = c;
    ri.v[1][2] = s * e.cx - c * e.cy;
    ri.v[2][0] = 0.f;
    ri.v[2][1] = 0.f;
    ri.v[2][2] = 1.f;
    M3 d = m3_zero();
    d.v[0][0] = 1.f / (e.a * e.a);
    d.v[1][1] = 1.f / (e.b * e.b);
    d.v[2][2] = -1.f;
    e.Q = m3_mul(m3_t(ri), m3_mul(d, ri));  // _matrix = diag * tmpInv; _matrix = tmpInv^T * _matrix
}

// Ellipse(center, a, b, angle) / init (Ellipse.cpp:32-50).
inline Ellipse ellipse_from_params(float cx, float cy, float a, float b, float angle)
{
    if (a < 0.f || b < 0.f) throw std::invalid_argument("Semi axes must be real positive!");
    Ellipse e;
    e.cx = cx;
    e.cy = cy;
    e.a = a;
    e.b = b;
    e.angle = angle;
    compute_matrix(e);
    return e;
}

// boost::math::sign
inline int sign_of(float v) { return v > 0.f ? 1 : (v < 0.f ? -1 : 0); }

// Ellipse::computeParameters (Ellipse.cpp:103-159).
inline void compute_parameters(Ellipse& e)
{
    const M3& m = e.Q;
    const float par0 = m.v[0][0], par1 = 2.f * m.v[0][1], par2 = m.v[1][1], par3 = 2.f * m.v[0][2],
                par4 = 2.f * m.v[1][2], par5 = m.v[2][2];
    const float thetarad = 0.5f * atan2_cr(par1, par0 - par2);
    const float cost = cos_cr(thetarad), sint = sin_cr(thetarad);
    const float sin_squared = sint * sint, cos_squared = cost * cost, cos_sin = sint * cost;
    const float Ao = par5;
    const float Au = par3 * cost + par4 * sint;
    const float Av = -par3 * sint + par4 * cost;
    const float Auu = par0 * cos_squared + par2 * sin_squared + par1 * cos_sin;
    const float Avv = par0 * sin_squared + par2 * cos_squared - par1 * cos_sin;
    if (Auu == 0 || Avv == 0) {
        e.cx = e.cy = e.a = e.b = e.angle = 0.f;
        return;
    }
    const float tuCentre = -Au / (2.0f * Auu);
    const float tvCentre = -Av / (2.0f * Avv);
    const float wCentre = Ao - Auu * tuCentre * tuCentre - Avv * tvCentre * tvCentre;
    const float ucx = tuCentre * cost - tvCentre * sint;
    const float ucy = tuCentre * sint + tvCentre * cost;
    const float Ru = -wCentre / Auu;
    const float Rv = -wCentre / Avv;
    const float aAux = std::sqrt(std::fabs(Ru)) * float(sign_of(Ru));
    const float bAux = std::sqrt(std::fabs(Rv)) * float(sign_of(Rv));
    if (aAux < 0.f || bAux < 0.f) throw std::invalid_argument("Semi axes must be real positive!");
    e.cx = ucx;
    e.cy = ucy;
    e.a = aAux;
    e.b = bAux;
    e.angle = thetarad;
}

// Ellipse(const Matrix3f&) (Ellipse.cpp:26-30).
inline Ellipse ellipse_from_matrix(const M3& Q)
{
    Ellipse e;
    e.Q = Q;
    compute_parameters(e);
    return e;
}

// p^T (Q p) for p = (x, y, 1), the Eigen expression p.dot(Q * p).
inline float quad(const M3& Q, float x, float y)
{
    const float r0 = Q.v[0][0] * x + Q.v[0][1] * y + Q.v[0][2];
    const float r1 = Q.v[1][0] * x + Q.v[1][1] * y + Q.v[1][2];
    const float r2 = Q.v[2][0] * x + Q.v[2][1] * y + Q.v[2][2];
    return x * r0 + y * r1 + r2;
}

// isInEllipse (EllipseGrowing.hpp:24-33)
inline bool is_in_ellipse(const Ellipse& e, float x, float y)
{
    return quad(e.Q, x, y) * (x * (e.Q.v[0][0] * e.cx + e.Q.v[0][1] * e.cy + e.Q.v[0][2]) +
                              y * (e.Q.v[1][0] * e.cx + e.Q.v[1][1] * e.cy + e.Q.v[1][2]) +
                              (e.Q.v[2][0] * e.cx + e.Q.v[2][1] * e.cy + e.Q.v[2][2])) >
           0;
}

// isInHull (EllipseGrowing.hpp:60-72)
inline bool is_in_hull(const Ellipse& qIn, const Ellipse& qOut, float x, float y)
{
    return quad(qIn.Q, x, y) * quad(qOut.Q, x, y) < 0;
}

// computeHull (EllipseGrowing.cpp:424-441)
inline void compute_hull(const Ellipse& e, float delta, Ellipse& qIn, Ellipse& qOut)
{
    qIn = ellipse_from_params(e.cx, e.cy, std::max(e.a - delta, 0.001f), std::max(e.b - delta, 0.001f), e.angle);
    qOut = ellipse_from_params(e.cx, e.cy, e.a + delta, e.b + delta, e.angle);
}

// distancePointEllipseScalar (geometry/Distance.cpp:18-43), p = (x, y, 1).
inline float distance_point_ellipse(const M3& Q, float x, float y)
{
    const float aux[6] = {x * x, 2 * x * y, 2 * x, y * y, 2 * y, 1};
    const float tmp1 = x * Q.v[0][0] + y * Q.v[0][1] + 1.f * Q.v[0][2];
    const float tmp2 = x * Q.v[0][1] + y * Q.v[1][1] + 1.f * Q.v[1][2];
    const float denom = tmp1 * tmp1 + tmp2 * tmp2;
    const float qL[6] = {Q.v[0][0], Q.v[0][1], Q.v[0][2], Q.v[1][1], Q.v[1][2], Q.v[2][2]};
    float dot = 0.f;
    for (int k = 0; k < 6; ++k) dot = k == 0 ? aux[0] * qL[0] : dot + aux[k] * qL[k];
    return dot * dot / denom;
}

// intersectEllipseWithLine (EllipseFromPoints.cpp:157-196): the roots along
// y = const (horizontal) or x = const.
inline std::vector<float> intersect_with_line(const Ellipse& e, float y, bool horizontal)
{
    std::vector<float> res;
    const M3& C = e.Q;
    float a, b, c;
    if (horizontal) {
        a = C.v[0][0];
        b = 2 * (y * C.v[0][1] + C.v[0][2]);
        c = C.v[1][1] * (y * y) + 2 * y * C.v[2][1] + C.v[2][2];
    } else {
        a = C.v[1][1];
        b = 2 * (y * C.v[0][1] + C.v[1][2]);
        c = C.v[0][0] * (y * y) + 2 * y * C.v[0][2] + C.v[2][2];
    }
    const float discriminant = (b * b) / 4.0f - a * c;
    if (discriminant > 0.f) {
        const float sq = std::sqrt(discriminant);
        res.push_back((-b / 2.0f - sq) / a);
        res.push_back((-b / 2.0f + sq) / a);
    } else if (discriminant == 0.f) {
        res.push_back(-b / (2.0f * a));
    }
    return res;
}

// ellipsePoint (EllipseFromPoints.cpp:66-74)
inline void ellipse_point(const Ellipse& e, float theta, float& px, float& py)
{
    const float x = e.a * cos_cr(theta);
    const float y = e.b * sin_cr(theta);
    px = x * cos_cr(e.angle) - y * sin_cr(e.angle) + e.cx;
    py = x * sin_cr(e.angle) + y * cos_cr(e.angle) + e.cy;
}

// computeIntermediatePoints + rasterizeEllipsePerimeter
// (EllipseFromPoints.cpp:76-105, 230-266).
inline int rasterize_perimeter(const Ellipse& e)
{
    float a = -e.b * sin_cr(e.angle) - e.b * cos_cr(e.angle);
    float b = -e.a * cos_cr(e.angle) + e.a * sin_cr(e.angle);
    const float t11 = atan2_cr(-a, b);
    const float t12 = t11 + kPi;
    a = -e.b * sin_cr(e.angle) + e.b * cos_cr(e.angle);
    b = -e.a * cos_cr(e.angle) - e.a * sin_cr(e.angle);
    const float t21 = atan2_cr(-a, b);
    const float t22 = t21 + kPi;
    float v11x, v11y, v12x, v12y, v22x, v22y;
    ellipse_point(e, t11, v11x, v11y);
    ellipse_point(e, t12, v12x, v12y);
    ellipse_point(e, t22, v22x, v22y);
    const int p11x = int(std::round(v11x)), p11y = int(std::round(v11y));
    const int p12x = int(std::round(v12x)), p12y = int(std::round(v12y));
    const int p22x = int(std::round(v22x)), p22y = int(std::round(v22y));
    float diff1, diff2;
    {
        const float mx = float(std::abs(p22x - p11x)), my = float(std::abs(p22y - p11y));
        diff1 = mx > my ? mx : my;
    }
    {
        const float mx = float(std::abs(p12x - p22x)), my = float(std::abs(p12y - p22y));
        diff2 = mx > my ? mx : my;
    }
    return int(size_t((diff1 + diff2) * 2.f));
}

// medianRef (Statistic.hpp:141-145): sort, take the element at size / 2.
inline float median_ref(std::vector<float> v)
{
    std::sort(v.begin(), v.end(), [](float x, float y) {
        if (std::isnan(x)) return false;
        if (std::isnan(y)) return true;
        return x < y;
    });
    return v[v.size() / 2];
}

// pcg32 (utils/pcg_random.hpp, O'Neill's XSH-RR 64/32 with a selectable
// stream), with the bounded draw by rejection of its operator()(n).
struct Pcg {
    uint64_t state, inc;
    static constexpr uint64_t kMult = 6364136223846793005ULL;
    Pcg(uint64_t seed, uint64_t stream)
    {
        inc = (stream << 1) | 1u;
        state = (seed + inc) * kMult + inc;
    }
    uint32_t operator()()
    {
        const uint64_t s = state;
        state = s * kMult + inc;
        const uint32_t xorshifted = uint32_t(((s >> 18u) ^ s) >> 27u);
        const uint32_t rot = uint32_t(s >> 59u);
        return (xorshifted >> rot) | (xorshifted << ((-rot) & 31u));
    }
    uint32_t operator()(uint32_t n)
    {
        const uint32_t threshold = uint32_t(0u - n) % n;
        for (;;) {
            const uint32_t r = (*this)();
            if (r >= threshold) return r % n;
        }
    }
};

// rand_5_k (Statistic.cpp:16-29)
inline void rand_5_k(int perm[5], size_t N, Pcg& rng)
{
    for (int i = 0; i < 5; ++i) {
        int r;
        do {
            r = int(rng(uint32_t(N)));
        } while (std::find(perm, perm + i, r) != perm + i);
        perm[i] = r;
    }
}

// Random streams of the candidate stage (the determinism choice of the
// restatement, seed 271828 as Statistic.cpp:18): loop 2 and loop 3 of
// candidate `index` on level `level`, and the level-0 re-fit of marker `mi`.
inline Pcg candidate_stream(int level, size_t index, int loop)
{
    return Pcg(271828u, (uint64_t(level) << 32) | (uint64_t(index) << 1) | uint64_t(loop));
}
inline Pcg refit_stream(size_t mi) { return Pcg(271828u, (uint64_t(1) << 62) | uint64_t(mi)); }

// The LMedS conic solve: A t = b for a 5x5 system in FP64 by Gaussian
// elimination with partial pivoting; false when a pivot column is all zero.
inline bool solve_5x5(double A[5][5], double b[5], double t[5])
{
    for (int col = 0; col < 5; ++col) {
        int best = col;
        for (int r = col + 1; r < 5; ++r)
            if (std::fabs(A[r][col]) > std::fabs(A[best][col])) best = r;
        if (std::fabs(A[best][col]) == 0.0) return false;
        if (best != col) {
            for (int k = 0; k < 5; ++k) std::swap(A[best][k], A[col][k]);
            std::swap(b[best], b[col]);
        }
        for (int r = col + 1; r < 5; ++r) {
            const double f = A[r][col] / A[col][col];
            for (int k = col; k < 5; ++k) A[r][k] -= f * A[col][k];
            b[r] -= f * b[col];
        }
    }
    for (int r = 4; r >= 0; --r) {
        double s = b[r];
        for (int k = r + 1; k < 5; ++k) s -= A[r][k] * t[k];
        t[r] = s / A[r][r];
    }
    return true;
}

struct P2 {
    float x, y;
};

// fitEllipse (Fitting.cpp:89-239): throws std::domain_error as the reference.
inline Ellipse fit_ellipse(const std::vector<P2>& p)
{
    if (p.size() < 5) throw std::domain_error("fitEllipse: at least 5 points are needed");
    float cx, cy, a, b, angle;
    const int st = cctagb::geo::fit_ellipse_core(
        [&p](size_t i, float& x, float& y) {
            x = p[i].x;
            y = p[i].y;
        },
        p.size(), cx, cy, a, b, angle);
    if (st != cctagb::geo::kFitOk) throw std::domain_error("fitEllipse: degenerate point set");
    return ellipse_from_params(cx, cy, a, b, angle);
}

// circleFitting (Fitting.cpp:329-360)
inline Ellipse fit_circle(const std::vector<P2>& p)
{
    double xc, yc, r;
    const bool ok = cctagb::geo::fit_circle_core(
        [&p](size_t i, float& x, float& y) {
            x = p[i].x;
            y = p[i].y;
        },
        p.size(), xc, yc, r);
    if (!ok) throw std::domain_error("Degenerate circle in circleFitting");
    return ellipse_from_params(float(xc), float(yc), float(r), float(r), 0.f);
}

}  // namespace gm
}  // namespace orc
