// Portable sine, cosine and arctangent for the candidate stage, which runs on
// the host (C++) and on the GPU (CUDA) and must give the same bits on both.
// Each function is evaluated in double precision -- argument reduction by a
// three-part pi/2 (Cody-Waite) and a polynomial fitted by gen_pmath.py -- and
// rounded once to float, so the float results are correctly rounded except
// within ~1e-16 of a rounding boundary.  Only IEEE +, -, *, / and floor are
// used, with no fused multiply-add (host: -ffp-contract=off; device: the
// translation units that include this are built with --fmad=false), so both
// compilers perform the same operations in the same order.
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define CCTAGB_HD __host__ __device__
#else
#define CCTAGB_HD
#endif

namespace cctagb {
namespace pm {

// Polynomials fitted by gen_pmath.py, in Horner form.
CCTAGB_HD inline double sin_p(double u)
{
    return -0.16666666666666666 + u * (0.008333333333333331 + u * (-0.00019841269841265065 + u * (2.7557319219339963e-06 + u * (-2.505210623269685e-08 + u * (1.605853165490743e-10 + u * (-7.586699058841919e-13))))));
}
CCTAGB_HD inline double cos_q(double u)
{
    return 0.041666666666666664 + u * (-0.0013888888888888887 + u * (2.480158730158465e-05 + u * (-2.755731922140322e-07 + u * (2.0876755791205128e-09 + u * (-1.1470460905580259e-11 + u * (4.745872873139979e-14))))));
}
CCTAGB_HD inline double atan_r(double u)
{
    return -0.3333333333333333 + u * (0.19999999999995652 + u * (-0.14285714284691378 + u * (0.11111111017100195 + u * (-0.0909090464769147 + u * (0.07692184699290894 + u * (-0.06664531368831207 + u * (0.05858311803098606 + u * (-0.05086254851324164 + u * (0.03925369542082372 + u * (-0.0192025282626767))))))))));
}

static constexpr double kPio2Hi = 1.5707963267341256, kPio2Mid = 6.07710050359346e-11,
                        kPio2Lo = 2.912732056093356e-20;
static constexpr double kPi = 3.141592653589793, kPio2 = 1.5707963267948966, kPio4 = 0.7853981633974483,
                        kTanPio8 = 0.41421356237309503, k2OverPi = 0.6366197723675814;

CCTAGB_HD inline bool sign_bit(double x) { return ::copysign(1.0, x) < 0.0; }

// x - k pi/2 with k the nearest integer to x 2/pi; q = k mod 4.
CCTAGB_HD inline double reduce_pio2(double x, int& q)
{
    const double k = ::floor(x * k2OverPi + 0.5);
    q = int(static_cast<long long>(k) & 3);
    return ((x - k * kPio2Hi) - k * kPio2Mid) - k * kPio2Lo;
}

CCTAGB_HD inline double sin_poly(double r)
{
    const double u = r * r;
    return r + r * (u * sin_p(u));
}

CCTAGB_HD inline double cos_poly(double r)
{
    const double u = r * r;
    return (1.0 - 0.5 * u) + (u * u) * cos_q(u);
}

CCTAGB_HD inline double sin_d(double x)
{
    int q;
    const double r = reduce_pio2(x, q);
    switch (q) {
    case 0: return sin_poly(r);
    case 1: return cos_poly(r);
    case 2: return -sin_poly(r);
    default: return -cos_poly(r);
    }
}

CCTAGB_HD inline double cos_d(double x)
{
    int q;
    const double r = reduce_pio2(x, q);
    switch (q) {
    case 0: return cos_poly(r);
    case 1: return -sin_poly(r);
    case 2: return -cos_poly(r);
    default: return sin_poly(r);
    }
}

// atan t for t in [0, 1]
CCTAGB_HD inline double atan_unit(double t)
{
    double base = 0.0, u = t;
    if (t > kTanPio8) {
        u = (t - 1.0) / (t + 1.0);
        base = kPio4;
    }
    const double z = u * u;
    return base + (u + u * (z * atan_r(z)));
}

// atan2 with the IEEE special cases of the zeros' signs.
CCTAGB_HD inline double atan2_d(double y, double x)
{
    if (x != x || y != y) return x + y;
    const double ax = ::fabs(x), ay = ::fabs(y);
    double r;
    if (ay == 0.0) r = 0.0;
    else if (ax == ay) r = kPio4;
    else if (ay < ax) r = atan_unit(ay / ax);
    else r = kPio2 - atan_unit(ax / ay);
    if (sign_bit(x)) r = kPi - r;
    return ::copysign(r, y);
}

// x / d, correctly rounded, for a small positive integer d given with its
// correctly rounded reciprocal y = RN(1 / d): q = RN(x y) is within one ulp of
// x / d, the remainder r = x - q d is exact as one fused multiply-add, and
// RN(q + r y) = RN(x / d) (Markstein's correction theorem: P. W. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34(1), 1990).  Valid while x, q and r stay
// normal; checked exhaustively over a binade of x for every d in [1, 256].
// Three dependent operations instead of a full division.
CCTAGB_HD inline float div_small(float x, float d, float y)
{
#ifdef __CUDA_ARCH__
    const float q = __fmul_rn(x, y);
    const float r = __fmaf_rn(-q, d, x);
    return __fmaf_rn(r, y, q);
#else
    const float q = x * y;
    const float r = std::fma(-q, d, x);
    return std::fma(r, y, q);
#endif
}

CCTAGB_HD inline float sinf_(float x) { return float(sin_d(double(x))); }
CCTAGB_HD inline float cosf_(float x) { return float(cos_d(double(x))); }
CCTAGB_HD inline float atan2f_(float y, float x) { return float(atan2_d(double(y), double(x))); }

}  // namespace pm
}  // namespace cctagb
