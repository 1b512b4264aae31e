// Host geometry for the candidate and identification stages: conics, ellipse
// parameters, point-conic distance, rasterised perimeter, ellipse and circle
// fitting, and the PCG32 generator used by the robust fits.  FP32 where the
// reference computes in FP32 (so thresholds behave the same), with FP64 only
// inside the small linear-algebra solves that the reference does with Eigen.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "cctag_b200/portable/pmath.hpp"

namespace cctagb {
namespace geo {

struct Mat3 {
    float m[3][3];
    CCTAGB_HD float& operator()(int r, int c) { return m[r][c]; }
    CCTAGB_HD float operator()(int r, int c) const { return m[r][c]; }
    CCTAGB_HD static Mat3 zero()
    {
        Mat3 z;
        for (auto& r : z.m)
            for (float& v : r) v = 0.f;
        return z;
    }
    CCTAGB_HD static Mat3 eye()
    {
        Mat3 z = zero();
        z.m[0][0] = z.m[1][1] = z.m[2][2] = 1.f;
        return z;
    }
};

CCTAGB_HD inline Mat3 mul(const Mat3& a, const Mat3& b)
{
    Mat3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j] + a.m[i][2] * b.m[2][j];
    return r;
}

CCTAGB_HD inline Mat3 transpose(const Mat3& a)
{
    Mat3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[j][i];
    return r;
}

// 3x3 inverse by cofactors (FP64 internally).  Throws when singular.
inline Mat3 inverse(const Mat3& a)
{
    double m[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) m[i][j] = a.m[i][j];
    const double c00 = m[1][1] * m[2][2] - m[1][2] * m[2][1];
    const double c01 = m[1][2] * m[2][0] - m[1][0] * m[2][2];
    const double c02 = m[1][0] * m[2][1] - m[1][1] * m[2][0];
    const double det = m[0][0] * c00 + m[0][1] * c01 + m[0][2] * c02;
    if (det == 0.0 || !std::isfinite(det)) throw std::domain_error("singular 3x3 matrix");
    const double id = 1.0 / det;
    Mat3 r;
    r.m[0][0] = float(c00 * id);
    r.m[0][1] = float((m[0][2] * m[2][1] - m[0][1] * m[2][2]) * id);
    r.m[0][2] = float((m[0][1] * m[1][2] - m[0][2] * m[1][1]) * id);
    r.m[1][0] = float(c01 * id);
    r.m[1][1] = float((m[0][0] * m[2][2] - m[0][2] * m[2][0]) * id);
    r.m[1][2] = float((m[0][2] * m[1][0] - m[0][0] * m[1][2]) * id);
    r.m[2][0] = float(c02 * id);
    r.m[2][1] = float((m[0][1] * m[2][0] - m[0][0] * m[2][1]) * id);
    r.m[2][2] = float((m[0][0] * m[1][1] - m[0][1] * m[1][0]) * id);
    return r;
}

inline void apply_h(const Mat3& H, float x, float y, float& ox, float& oy)
{
    // Identification.hpp:102-113
    const float u = H.m[0][0] * x + H.m[0][1] * y + H.m[0][2];
    const float v = H.m[1][0] * x + H.m[1][1] * y + H.m[1][2];
    const float w = H.m[2][0] * x + H.m[2][1] * y + H.m[2][2];
    ox = u / w;
    oy = v / w;
}

// ------------------------------------------------------------------ ellipse --
// Ellipse.cpp:223-241: Q = R^-T diag(1/a^2, 1/b^2, -1) R^-1 with R the rigid
// transform of the ellipse frame.
CCTAGB_HD inline Mat3 conic_of_params(float cx, float cy, float a, float b, float angle)
{
    const float c = pm::cosf_(angle), s = pm::sinf_(angle);
    Mat3 Ri;  // inverse of [c -s cx; s c cy; 0 0 1]
    Ri.m[0][0] = c;  Ri.m[0][1] = s; Ri.m[0][2] = -(c * cx + s * cy);
    Ri.m[1][0] = -s; Ri.m[1][1] = c; Ri.m[1][2] = s * cx - c * cy;
    Ri.m[2][0] = 0;  Ri.m[2][1] = 0; Ri.m[2][2] = 1;
    Mat3 D = Mat3::zero();
    D.m[0][0] = 1.f / (a * a);
    D.m[1][1] = 1.f / (b * b);
    D.m[2][2] = -1.f;
    return mul(transpose(Ri), mul(D, Ri));
}

// Ellipse.cpp:103-159: center, semi axes and angle of the conic Q.  All zero
// when the conic is degenerate (Auu or Avv zero); returns false when a semi
// axis comes out negative (the reference throws).
CCTAGB_HD inline bool params_of_conic(const Mat3& Q, float& cx, float& cy, float& a, float& b, float& angle)
{
    const float p0 = Q.m[0][0], p1 = 2.f * Q.m[0][1], p2 = Q.m[1][1], p3 = 2.f * Q.m[0][2],
                p4 = 2.f * Q.m[1][2], p5 = Q.m[2][2];
    const float th = 0.5f * pm::atan2f_(p1, p0 - p2);
    const float ct = pm::cosf_(th), st = pm::sinf_(th);
    const float s2 = st * st, c2 = ct * ct, cs = st * ct;
    const float Ao = p5;
    const float Au = p3 * ct + p4 * st;
    const float Av = -p3 * st + p4 * ct;
    const float Auu = p0 * c2 + p2 * s2 + p1 * cs;
    const float Avv = p0 * s2 + p2 * c2 - p1 * cs;
    if (Auu == 0.f || Avv == 0.f) {
        cx = cy = a = b = angle = 0.f;
        return true;
    }
    const float tu = -Au / (2.f * Auu);
    const float tv = -Av / (2.f * Avv);
    const float wc = Ao - Auu * tu * tu - Avv * tv * tv;
    cx = tu * ct - tv * st;
    cy = tu * st + tv * ct;
    const float Ru = -wc / Auu, Rv = -wc / Avv;
    const float aa = ::sqrtf(::fabsf(Ru)) * float((Ru > 0) - (Ru < 0));
    const float bb = ::sqrtf(::fabsf(Rv)) * float((Rv > 0) - (Rv < 0));
    if (aa < 0.f || bb < 0.f) return false;
    a = aa;
    b = bb;
    angle = th;
    return true;
}

// geometry/Ellipse.cpp: an ellipse is held both as parameters (center, semi
// axes, angle) and as its conic matrix Q (x^T Q x = 0, negative inside).
struct Ellipse {
    float cx = 0.f, cy = 0.f, a = 0.f, b = 0.f, angle = 0.f;
    Mat3 Q = Mat3::zero();

    static Ellipse from_params(float cx, float cy, float a, float b, float angle)
    {
        if (a < 0.f || b < 0.f) throw std::invalid_argument("Semi axes must be real positive!");
        Ellipse e;
        e.cx = cx;
        e.cy = cy;
        e.a = a;
        e.b = b;
        e.angle = angle;
        e.compute_matrix();
        return e;
    }
    static Ellipse from_matrix(const Mat3& Q)
    {
        Ellipse e;
        e.Q = Q;
        e.compute_parameters();
        return e;
    }
    void compute_matrix() { Q = conic_of_params(cx, cy, a, b, angle); }
    void compute_parameters()
    {
        if (!params_of_conic(Q, cx, cy, a, b, angle)) throw std::invalid_argument("Semi axes must be real positive!");
    }
    // Ellipse.cpp:89-94: conic of the transformed ellipse, mT^T Q mT.
    Ellipse transform(const Mat3& mT) const { return from_matrix(mul(transpose(mT), mul(Q, mT))); }

    // Ellipse.cpp:161-214: the conic in its canonical frame (rotated, centred)
    // with the primal and dual frame transforms.
    void canonic_form(Mat3& C, Mat3& Tp, Mat3& Td) const
    {
        const float q1 = Q.m[0][0], q2 = Q.m[0][1], q3 = Q.m[0][2], q4 = Q.m[1][1], q5 = Q.m[1][2], q6 = Q.m[2][2];
        const float par1 = q1, par2 = 2 * q2, par3 = q4, par4 = 2 * q3, par5 = 2 * q5;
        const float th = 0.5f * pm::atan2f_(par2, par1 - par3);
        const float ct = pm::cosf_(th), st = pm::sinf_(th);
        const float s2 = st * st, c2 = ct * ct, cs = st * ct;
        const float Au = par4 * ct + par5 * st;
        const float Av = -par4 * st + par5 * ct;
        const float Auu = par1 * c2 + par3 * s2 + par2 * cs;
        const float Avv = par1 * s2 + par3 * c2 - par2 * cs;
        const float tu = -Au / (2 * Auu);
        const float tv = -Av / (2 * Avv);
        const float uc = tu * ct - tv * st;
        const float vc = tu * st + tv * ct;
        const float t1 = ct * (ct * q1 + q2 * st) + st * (ct * q2 + q4 * st);
        const float t2 = ct * (ct * q2 + q4 * st) - st * (ct * q1 + q2 * st);
        const float t3 = ct * q3 + q5 * st + uc * (ct * q1 + q2 * st) + vc * (ct * q2 + q4 * st);
        const float t4 = ct * (ct * q4 - q2 * st) - st * (ct * q2 - q1 * st);
        const float t5 = ct * q5 - q3 * st + uc * (ct * q2 - q1 * st) + vc * (ct * q4 - q2 * st);
        const float t6 = q6 + uc * (q3 + q1 * uc + q2 * vc) + vc * (q5 + q2 * uc + q4 * vc) + q3 * uc + q5 * vc;
        C.m[0][0] = t1; C.m[0][1] = t2; C.m[0][2] = t3;
        C.m[1][0] = t2; C.m[1][1] = t4; C.m[1][2] = t5;
        C.m[2][0] = t3; C.m[2][1] = t5; C.m[2][2] = t6;
        Tp.m[0][0] = ct;  Tp.m[0][1] = st; Tp.m[0][2] = -ct * uc - st * vc;
        Tp.m[1][0] = -st; Tp.m[1][1] = ct; Tp.m[1][2] = st * uc - ct * vc;
        Tp.m[2][0] = 0;   Tp.m[2][1] = 0;  Tp.m[2][2] = ct * ct + st * st;
        Td.m[0][0] = ct;  Td.m[0][1] = -st; Td.m[0][2] = uc;
        Td.m[1][0] = st;  Td.m[1][1] = ct;  Td.m[1][2] = vc;
        Td.m[2][0] = 0;   Td.m[2][1] = 0;   Td.m[2][2] = 1.f;
    }
};

// Quadratic form p^T Q p for p = (x, y, 1).
CCTAGB_HD inline float qform(const Mat3& Q, float x, float y)
{
    const float r0 = Q.m[0][0] * x + Q.m[0][1] * y + Q.m[0][2];
    const float r1 = Q.m[1][0] * x + Q.m[1][1] * y + Q.m[1][2];
    const float r2 = Q.m[2][0] * x + Q.m[2][1] * y + Q.m[2][2];
    return x * r0 + y * r1 + r2;
}

// EllipseGrowing.hpp:24-33: p and the center on the same side of the conic.
inline bool is_in_ellipse(const Ellipse& e, float x, float y)
{
    return qform(e.Q, x, y) * qform(e.Q, e.cx, e.cy) > 0.f;
}

// EllipseGrowing.hpp:60-72: strictly between the two conics.
CCTAGB_HD inline bool is_in_hull_q(const Mat3& qIn, const Mat3& qOut, float x, float y)
{
    return qform(qIn, x, y) * qform(qOut, x, y) < 0.f;
}
inline bool is_in_hull(const Ellipse& qIn, const Ellipse& qOut, float x, float y)
{
    return is_in_hull_q(qIn.Q, qOut.Q, x, y);
}

// EllipseGrowing.cpp:424-441
inline void compute_hull(const Ellipse& e, float delta, Ellipse& qIn, Ellipse& qOut)
{
    qIn = Ellipse::from_params(e.cx, e.cy, std::max(e.a - delta, 0.001f), std::max(e.b - delta, 0.001f), e.angle);
    qOut = Ellipse::from_params(e.cx, e.cy, e.a + delta, e.b + delta, e.angle);
}

// geometry/Distance.cpp:18-43 (the scalar path): squared algebraic distance
// normalised by the squared gradient norm of the conic at p.
CCTAGB_HD inline float dist_point_ellipse(const Mat3& Q, float x, float y)
{
    const float aux0 = x * x, aux1 = 2 * x * y, aux2 = 2 * x, aux3 = y * y, aux4 = 2 * y;
    const float t1 = x * Q.m[0][0] + y * Q.m[0][1] + Q.m[0][2];
    const float t2 = x * Q.m[0][1] + y * Q.m[1][1] + Q.m[1][2];
    const float denom = t1 * t1 + t2 * t2;
    const float dot = aux0 * Q.m[0][0] + aux1 * Q.m[0][1] + aux2 * Q.m[0][2] + aux3 * Q.m[1][1] +
                      aux4 * Q.m[1][2] + Q.m[2][2];
    return dot * dot / denom;
}

// EllipseFromPoints.cpp:124-154: intersections of the conic with y = const
// (horizontal) or x = const (vertical).
CCTAGB_HD inline int intersect_line_q(const Mat3& C, float y, bool horizontal, float out[2])
{
    out[0] = out[1] = 0.f;
    float a, b, c;
    if (horizontal) {
        a = C.m[0][0];
        b = 2 * (y * C.m[0][1] + C.m[0][2]);
        c = C.m[1][1] * (y * y) + 2 * y * C.m[2][1] + C.m[2][2];  // pow<2>(y) first
    } else {
        a = C.m[1][1];
        b = 2 * (y * C.m[0][1] + C.m[1][2]);
        c = C.m[0][0] * (y * y) + 2 * y * C.m[0][2] + C.m[2][2];
    }
    const float disc = b * b / 4.0f - a * c;
    if (disc > 0.f) {
        const float sd = ::sqrtf(disc);
        out[0] = (-b / 2.0f - sd) / a;
        out[1] = (-b / 2.0f + sd) / a;
        return 2;
    }
    if (disc == 0.f) {
        out[0] = -b / (2.0f * a);
        return 1;
    }
    return 0;
}

inline int intersect_line(const Ellipse& e, float y, bool horizontal, float out[2])
{
    return intersect_line_q(e.Q, y, horizontal, out);
}

CCTAGB_HD inline float round_half_away(float v) { return ::roundf(v); }

// EllipseFromPoints.cpp:64-99 (computeIntermediatePoints) and :193-230
// (rasterizeEllipsePerimeter): pixel length of the rasterised perimeter of
// the ellipse (center, semi axes, angle).
CCTAGB_HD inline int rasterize_perimeter_p(float ecx, float ecy, float ea, float eb, float eangle)
{
    struct {
        float cx, cy, a, b, angle;
    } e{ecx, ecy, ea, eb, eangle};
    auto pt = [&](float t, float& x, float& y) {
        const float ex = e.a * pm::cosf_(t), ey = e.b * pm::sinf_(t);
        x = ex * pm::cosf_(e.angle) - ey * pm::sinf_(e.angle) + e.cx;
        y = ex * pm::sinf_(e.angle) + ey * pm::cosf_(e.angle) + e.cy;
    };
    const float pi = 3.14159265358979323846f;
    float a = -e.b * pm::sinf_(e.angle) - e.b * pm::cosf_(e.angle);
    float b = -e.a * pm::cosf_(e.angle) + e.a * pm::sinf_(e.angle);
    const float t11 = pm::atan2f_(-a, b), t12 = t11 + pi;
    a = -e.b * pm::sinf_(e.angle) + e.b * pm::cosf_(e.angle);
    b = -e.a * pm::cosf_(e.angle) - e.a * pm::sinf_(e.angle);
    const float t21 = pm::atan2f_(-a, b), t22 = t21 + pi;
    float x11, y11, x12, y12, x22, y22;
    (void)t21;
    pt(t11, x11, y11);
    pt(t12, x12, y12);
    pt(t22, x22, y22);
    const int p11x = int(round_half_away(x11)), p11y = int(round_half_away(y11));
    const int p12x = int(round_half_away(x12)), p12y = int(round_half_away(y12));
    const int p22x = int(round_half_away(x22)), p22y = int(round_half_away(y22));
    float d1, d2;
    {
        const float mx = float(::abs(p22x - p11x)), my = float(::abs(p22y - p11y));
        d1 = mx > my ? mx : my;
    }
    {
        const float mx = float(::abs(p12x - p22x)), my = float(::abs(p12y - p22y));
        d2 = mx > my ? mx : my;
    }
    return int((d1 + d2) * 2.f);
}
inline int rasterize_perimeter(const Ellipse& e) { return rasterize_perimeter_p(e.cx, e.cy, e.a, e.b, e.angle); }

// EllipseFromPoints.cpp:29-48: radial projection of p onto the ellipse.
inline void point_on_ellipse(const Ellipse& e, float px, float py, float& ox, float& oy)
{
    const float x = px - e.cx, y = py - e.cy;
    const float c = pm::cosf_(e.angle), s = pm::sinf_(e.angle);
    float tx = x * c + y * s;
    float ty = -x * s + y * c;
    const float cs = std::sqrt(tx * tx / (e.a * e.a) + ty * ty / (e.b * e.b));
    tx /= cs;
    ty /= cs;
    ox = tx * c - ty * s + e.cx;
    oy = tx * s + ty * c + e.cy;
}

// ---------------------------------------------------------------- fitting --
struct Pt {
    float x, y;
};

// Direct least-squares ellipse fit with the constraint 4ac - b^2 = 1
// (Fitting.cpp:89-200, the Halir-Flusser split of the scatter matrix), points
// centred on their mean.  The 3x3 eigenproblem and the 2x2 SVD are solved in
// FP64.  Throws std::domain_error on degenerate input as the reference.
Ellipse fit_ellipse(const Pt* p, size_t n);
// Algebraic circle fit (Fitting.cpp:329-360): smallest right singular vector
// of [x y 1 x^2+y^2].
Ellipse fit_circle(const Pt* p, size_t n);

// ------------------------------------------------------------------- PCG32 --
// O'Neill's PCG32 (XSH-RR 64/32), default stream; bounded draws by rejection
// of the low range, as the reference's rand_5_k (Statistic.cpp:16-29) uses
// with seed 271828.
struct Pcg32 {
    uint64_t state = 0;
    static constexpr uint64_t kMul = 6364136223846793005ULL;
    static constexpr uint64_t kInc = 1442695040888963407ULL;
    uint64_t inc = kInc;
    CCTAGB_HD explicit Pcg32(uint64_t seed = 271828) { reseed(seed); }
    // Stream `stream` of the generator (PCG's selectable increment).
    CCTAGB_HD Pcg32(uint64_t seed, uint64_t stream) : inc((stream << 1) | 1u)
    {
        state = 0;
        state = state * kMul + inc;
        state += seed;
        state = state * kMul + inc;
    }
    CCTAGB_HD void reseed(uint64_t seed)
    {
        inc = kInc;
        state = (seed + kInc) * kMul + kInc;
    }
    CCTAGB_HD uint32_t next()
    {
        const uint64_t old = state;
        state = old * kMul + inc;
        return output(old);
    }
    // Output of the generator at state s (XSH-RR).
    CCTAGB_HD static uint32_t output(uint64_t s)
    {
        const uint32_t xs = uint32_t(((s >> 18) ^ s) >> 27);
        const uint32_t rot = uint32_t(s >> 59);
        return (xs >> rot) | (xs << ((32u - rot) & 31u));
    }
    // Skips `delta` outputs in O(log delta): the LCG jump of F. Brown,
    // "Random number generation with arbitrary strides" (1994), as PCG's
    // advance function.
    CCTAGB_HD void advance(uint64_t delta)
    {
        uint64_t curMul = kMul, curPlus = inc, accMul = 1u, accPlus = 0u;
        while (delta > 0) {
            if (delta & 1u) {
                accMul *= curMul;
                accPlus = accPlus * curMul + curPlus;
            }
            curPlus = (curMul + 1u) * curPlus;
            curMul *= curMul;
            delta >>= 1;
        }
        state = accMul * state + accPlus;
    }
    CCTAGB_HD uint32_t bounded(uint32_t n)
    {
        const uint32_t threshold = uint32_t(-n) % n;
        for (;;) {
            const uint32_t r = next();
            if (r >= threshold) return r % n;
        }
    }
    // Five distinct indices in [0, n) (Statistic.cpp:16-29).
    CCTAGB_HD void rand5(int perm[5], size_t n)
    {
        for (int i = 0; i < 5; ++i) perm[i] = -1;
        for (int i = 0; i < 5; ++i) {
            int r;
            bool seen;
            do {
                r = int(bounded(uint32_t(n)));
                seen = false;
                for (int j = 0; j < i; ++j) seen = seen || perm[j] == r;
            } while (seen);
            perm[i] = r;
        }
    }
};

// Order key of a float with every NaN above +inf: the total order the
// medians use, so that an array holding NaNs has one well-defined median on
// every platform (the reference's nth_element leaves it unspecified).
CCTAGB_HD inline uint32_t order_key(float v)
{
    uint32_t u;
    memcpy(&u, &v, 4);
    if (v != v) return 0xffffffffu;
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Statistic.hpp:112-117 (medianRef): the element at index size/2 of the
// sorted values (NaN last); nth_element yields it without a full sort.  The
// vector is reordered.
inline float median_ref(std::vector<float>& v)
{
    std::nth_element(v.begin(), v.begin() + v.size() / 2, v.end(),
                     [](float a, float b) { return order_key(a) < order_key(b); });
    return v[v.size() / 2];
}

}  // namespace geo
}  // namespace cctagb
