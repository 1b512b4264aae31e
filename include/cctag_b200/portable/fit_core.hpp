// FP64 cores of the two point fits of the candidate stage, written once for
// the host and the GPU, and the arithmetic that pins them: the reference
// solves their small eigen / singular-value problems with Eigen, whose last
// bits depend on the platform, so this header fixes one sequence of IEEE
// operations for them.  The library and the CPU oracle both use it; each
// restates the algorithm around it (point selection, conic parameters,
// thresholds) on its own.
//
// Direct least-squares ellipse fit (Fitting.cpp:89-200 of the reference: the
// Halir-Flusser reduction of Fitzgibbon's fit, eigen decomposition of the 3x3
// reduced scatter matrix).  The characteristic cubic is solved in real
// arithmetic (Cardano with a portable cube root, or the trigonometric form for
// three real roots), each root polished by Newton, and the eigenvectors taken
// from cross products of (M - lambda I), in complex arithmetic for a complex
// pair (the real part, as Eigen's eigenvectors().real()).
//
// Algebraic circle fit (Fitting.cpp:329-360): the smallest right singular
// vector of [x y 1 x^2+y^2], as the eigenvector of the smallest eigenvalue of
// the 4x4 normal matrix, by cyclic Jacobi rotations.
//
// Only +, -, *, /, sqrt and the portable pmath functions are used.
#pragma once

#include <cfloat>
#include <cmath>
#include <cstddef>
#if defined(__SSE2__) && !defined(__CUDA_ARCH__)
#include <emmintrin.h>
#endif

#include "pmath.hpp"

namespace cctagb {
namespace geo {

enum FitStatus {
    kFitOk = 0,
    kFitTooFewPoints,      // fewer than 5 points
    kFitDependent,         // the points appear to be linearly dependent
    kFitDegenerate,        // no eigenvector satisfies the ellipse constraint
    kFitSingular1,         // to_ellipse: singularity 1
    kFitSingular2,         // to_ellipse: singularity 2
    kFitLineOrPoint,       // degenerate ellipse (line or point)
};

struct FitCplx {
    double re, im;
};

CCTAGB_HD inline FitCplx cx_mul(FitCplx a, FitCplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
CCTAGB_HD inline FitCplx cx_sub(FitCplx a, FitCplx b) { return {a.re - b.re, a.im - b.im}; }
CCTAGB_HD inline FitCplx cx_add(FitCplx a, FitCplx b) { return {a.re + b.re, a.im + b.im}; }
CCTAGB_HD inline double cx_norm(FitCplx a) { return a.re * a.re + a.im * a.im; }
CCTAGB_HD inline FitCplx cx_div(FitCplx a, FitCplx b)
{
    const double d = b.re * b.re + b.im * b.im;
    return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}

// Real cube root (sign kept): Newton's iteration from 2^k, k = floor(log8 a)
// (the power of two whose cube brings a into [1, 8)), until an iterate
// repeats, at most 60 steps.  When the iterates settle into two alternating
// values the 60th is known without running the rest.
CCTAGB_HD inline double cbrt_d(double y)
{
    if (y == 0.0 || !(y == y) || ::fabs(y) > DBL_MAX) return y;
    const double a = ::fabs(y);
    const int e = ::ilogb(a);  // floor(log2 a)
    const int k = e >= 0 ? e / 3 : -((2 - e) / 3);
    double x = ::ldexp(1.0, k), prev = 0.0;
    for (int it = 0; it < 60; ++it) {
        const double nx = x - (x * x * x - a) / (3.0 * x * x);
        if (nx == x) break;
        if (it > 0 && nx == prev) {  // x_(it+1) == x_(it-1): x_60 is x_(it-1) or x_it
            x = (61 - it) % 2 == 0 ? prev : x;
            break;
        }
        prev = x;
        x = nx;
    }
    return y < 0.0 ? -x : x;
}

// Roots of x^3 + a x^2 + b x + c: three real, or one real and a complex pair.
CCTAGB_HD inline void cubic_roots_real(double a, double b, double c, FitCplx r[3])
{
    const double p = b - a * a / 3.0;
    const double q = 2.0 * a * a * a / 27.0 - a * b / 3.0 + c;
    const double disc = q * q / 4.0 + p * p * p / 27.0;
    const double shift = a / 3.0;
    if (disc > 0.0) {
        const double s = ::sqrt(disc);
        const double u = cbrt_d(-q / 2.0 + s), v = cbrt_d(-q / 2.0 - s);
        r[0] = {u + v - shift, 0.0};
        const double re = -(u + v) / 2.0 - shift, im = (u - v) * 0.8660254037844386;
        r[1] = {re, im};
        r[2] = {re, -im};
    } else if (p == 0.0) {
        r[0] = r[1] = r[2] = {-shift, 0.0};
    } else {
        const double m = 2.0 * ::sqrt(-p / 3.0);
        double arg = 3.0 * q / (p * m);
        arg = arg > 1.0 ? 1.0 : (arg < -1.0 ? -1.0 : arg);
        const double th = pm::atan2_d(::sqrt((1.0 - arg) * (1.0 + arg)), arg) / 3.0;
        for (int k = 0; k < 3; ++k) r[k] = {m * pm::cos_d(th - 2.0943951023931957 * double(k)) - shift, 0.0};
    }
    // Newton polish on the original cubic (complex arithmetic for a complex root)
    for (int k = 0; k < 3; ++k) {
        for (int it = 0; it < 3; ++it) {
            const FitCplx x = r[k];
            const FitCplx f = cx_add(cx_mul(cx_add(cx_mul(cx_add(x, {a, 0.0}), x), {b, 0.0}), x), {c, 0.0});
            const FitCplx df = cx_add(cx_mul(cx_add({3.0 * x.re, 3.0 * x.im}, {2.0 * a, 0.0}), x), {b, 0.0});
            if (!(cx_norm(df) > 0.0)) break;
            r[k] = cx_sub(x, cx_div(f, df));
        }
    }
}

// Unit eigenvector of M for eigenvalue lam: the largest cross product of two
// rows of (M - lam I), phase fixed so that its largest component is real, real
// part returned (Eigen's EigenSolver().eigenvectors().real() convention).
CCTAGB_HD inline void eigvec_real(const double M[3][3], FitCplx lam, double out[3])
{
    FitCplx A[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) A[i][j] = {M[i][j] - (i == j ? lam.re : 0.0), i == j ? -lam.im : 0.0};
    FitCplx best[3] = {{0, 0}, {0, 0}, {0, 0}};
    double bn = -1.0;
    for (int i = 0; i < 3; ++i)
        for (int j = i + 1; j < 3; ++j) {
            const FitCplx c0 = cx_sub(cx_mul(A[i][1], A[j][2]), cx_mul(A[i][2], A[j][1]));
            const FitCplx c1 = cx_sub(cx_mul(A[i][2], A[j][0]), cx_mul(A[i][0], A[j][2]));
            const FitCplx c2 = cx_sub(cx_mul(A[i][0], A[j][1]), cx_mul(A[i][1], A[j][0]));
            const double n = cx_norm(c0) + cx_norm(c1) + cx_norm(c2);
            if (n > bn) {
                bn = n;
                best[0] = c0;
                best[1] = c1;
                best[2] = c2;
            }
        }
    const double nrm = ::sqrt(bn > 0.0 ? bn : 0.0);
    if (!(nrm > 0.0)) {
        out[0] = out[1] = out[2] = 0.0;
        return;
    }
    int kmax = 0;
    for (int k = 1; k < 3; ++k)
        if (cx_norm(best[k]) > cx_norm(best[kmax])) kmax = k;
    const double am = ::sqrt(cx_norm(best[kmax]));
    const FitCplx ph = am > 0.0 ? FitCplx{best[kmax].re / am, -best[kmax].im / am} : FitCplx{1.0, 0.0};
    for (int k = 0; k < 3; ++k) out[k] = cx_mul(best[k], ph).re / nrm;
}

CCTAGB_HD inline bool inv3_d(const double a[3][3], double r[3][3])
{
    const double c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1];
    const double c01 = a[1][2] * a[2][0] - a[1][0] * a[2][2];
    const double c02 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
    const double det = a[0][0] * c00 + a[0][1] * c01 + a[0][2] * c02;
    double scale = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) scale = ::fmax(scale, ::fabs(a[i][j]));
    if (det == 0.0 || !(::fabs(det) <= DBL_MAX) || ::fabs(det) <= 1e-14 * scale * scale * scale) return false;
    const double id = 1.0 / det;
    r[0][0] = c00 * id;
    r[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) * id;
    r[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) * id;
    r[1][0] = c01 * id;
    r[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) * id;
    r[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) * id;
    r[2][0] = c02 * id;
    r[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) * id;
    r[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) * id;
    return true;
}

// Symmetric 2x2 eigen decomposition by Jacobi rotations, eigenvectors in columns.
CCTAGB_HD inline void jacobi2(double A[2][2], double V[2][2], double d[2])
{
    V[0][0] = V[1][1] = 1.0;
    V[0][1] = V[1][0] = 0.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        if (A[0][1] * A[0][1] < 1e-300) break;
        if (::fabs(A[0][1]) < 1e-300) break;
        const double theta = (A[1][1] - A[0][0]) / (2.0 * A[0][1]);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (::fabs(theta) + ::sqrt(theta * theta + 1.0));
        const double c = 1.0 / ::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 2; ++k) {
            const double akp = A[k][0], akq = A[k][1];
            A[k][0] = c * akp - s * akq;
            A[k][1] = s * akp + c * akq;
        }
        for (int k = 0; k < 2; ++k) {
            const double apk = A[0][k], aqk = A[1][k];
            A[0][k] = c * apk - s * aqk;
            A[1][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 2; ++k) {
            const double vkp = V[k][0], vkq = V[k][1];
            V[k][0] = c * vkp - s * vkq;
            V[k][1] = s * vkp + c * vkq;
        }
    }
    d[0] = A[0][0];
    d[1] = A[1][1];
}

// The fit on n points (x[i], y[i]) read through `pt(i, x, y)`; on success the
// ellipse parameters (center, semi axes, angle) as the reference's
// Ellipse(center, r0, r1, angle) receives them.  The sums run in point order.
template <class PointAt>
CCTAGB_HD inline int fit_ellipse_core(PointAt pt, size_t n, float& ocx, float& ocy, float& oa, float& ob,
                                      float& oangle)
{
    if (n < 5) return kFitTooFewPoints;
    // Fitting.cpp:37-45 offset (mean), :47-71 scatter matrices
    double ox = 0, oy = 0;
    for (size_t i = 0; i < n; ++i) {
        float x, y;
        pt(i, x, y);
        ox += x;
        oy += y;
    }
    ox /= double(n);
    oy /= double(n);
    // S1 = sum q q^T, S2 = sum q l^T, S3 = sum l l^T with q = (x^2, xy, y^2) and
    // l = (x, y, 1): the symmetric entries once (a product and its transpose
    // are the same double), the products by 1 left out (exact).
    double a00 = 0, a01 = 0, a02 = 0, a11 = 0, a12 = 0, a22 = 0;  // S1
    double b00 = 0, b01 = 0, b02 = 0, b10 = 0, b11 = 0, b12 = 0, b20 = 0, b21 = 0, b22 = 0;  // S2
    double c00 = 0, c01 = 0, c02 = 0, c11 = 0, c12 = 0, c22 = 0;  // S3
#if defined(__SSE2__) && !defined(__CUDA_ARCH__)
    // The same products and sums, two accumulators per SSE2 operation (IEEE
    // double multiplies and adds; each accumulator is still summed in point
    // order, so the results are the same bits).  S3's x x, x y, y y are the
    // q0, q1, q2 products.
    {
        const __m128d z = _mm_setzero_pd(), vo = _mm_set_pd(oy, ox);
        __m128d A0 = z, A1 = z, A2 = z;                // (a00 a01) (a02 a11) (a12 a22)
        __m128d B0 = z, B1 = z, B2 = z, B3 = z, B4 = z;  // (b00 b01) (b10 b11) (b20 b21) (b02 b12) (b22 c00)
        __m128d C0 = z, C1 = z;                        // (c01 c11) (c02 c12)
        for (size_t i = 0; i < n; ++i) {
            float xf, yf;
            pt(i, xf, yf);
            const __m128d xy = _mm_sub_pd(_mm_set_pd(double(yf), double(xf)), vo);  // (x, y)
            const __m128d q01 = _mm_mul_pd(_mm_unpacklo_pd(xy, xy), xy);            // (q0, q1)
            const __m128d yy = _mm_unpackhi_pd(xy, xy);
            const __m128d q22 = _mm_mul_pd(yy, yy);                                 // (q2, q2)
            const __m128d q00 = _mm_unpacklo_pd(q01, q01), q11 = _mm_unpackhi_pd(q01, q01);
            const __m128d q12 = _mm_shuffle_pd(q01, q22, 1);                        // (q1, q2)
            A0 = _mm_add_pd(A0, _mm_mul_pd(q00, q01));
            A1 = _mm_add_pd(A1, _mm_mul_pd(q01, _mm_shuffle_pd(q22, q01, 2)));     // (q0 q2, q1 q1)
            A2 = _mm_add_pd(A2, _mm_mul_pd(q12, q22));
            B0 = _mm_add_pd(B0, _mm_mul_pd(q00, xy));
            B1 = _mm_add_pd(B1, _mm_mul_pd(q11, xy));
            B2 = _mm_add_pd(B2, _mm_mul_pd(q22, xy));
            B3 = _mm_add_pd(B3, q01);
            B4 = _mm_add_pd(B4, _mm_shuffle_pd(q22, q01, 0));                      // (q2, q0)
            C0 = _mm_add_pd(C0, q12);
            C1 = _mm_add_pd(C1, xy);
            c22 += 1.0;
        }
        double v[2];
        _mm_storeu_pd(v, A0), a00 = v[0], a01 = v[1];
        _mm_storeu_pd(v, A1), a02 = v[0], a11 = v[1];
        _mm_storeu_pd(v, A2), a12 = v[0], a22 = v[1];
        _mm_storeu_pd(v, B0), b00 = v[0], b01 = v[1];
        _mm_storeu_pd(v, B1), b10 = v[0], b11 = v[1];
        _mm_storeu_pd(v, B2), b20 = v[0], b21 = v[1];
        _mm_storeu_pd(v, B3), b02 = v[0], b12 = v[1];
        _mm_storeu_pd(v, B4), b22 = v[0], c00 = v[1];
        _mm_storeu_pd(v, C0), c01 = v[0], c11 = v[1];
        _mm_storeu_pd(v, C1), c02 = v[0], c12 = v[1];
    }
#else
    for (size_t i = 0; i < n; ++i) {
        float xf, yf;
        pt(i, xf, yf);
        const double x = xf - ox, y = yf - oy;
        const double q0 = x * x, q1 = x * y, q2 = y * y;
        a00 += q0 * q0;
        a01 += q0 * q1;
        a02 += q0 * q2;
        a11 += q1 * q1;
        a12 += q1 * q2;
        a22 += q2 * q2;
        b00 += q0 * x;
        b01 += q0 * y;
        b02 += q0;
        b10 += q1 * x;
        b11 += q1 * y;
        b12 += q1;
        b20 += q2 * x;
        b21 += q2 * y;
        b22 += q2;
        c00 += x * x;
        c01 += x * y;
        c02 += x;
        c11 += y * y;
        c12 += y;
        c22 += 1.0;
    }
#endif
    const double S1[3][3] = {{a00, a01, a02}, {a01, a11, a12}, {a02, a12, a22}};
    const double S2[3][3] = {{b00, b01, b02}, {b10, b11, b12}, {b20, b21, b22}};
    const double S3[3][3] = {{c00, c01, c02}, {c01, c11, c12}, {c02, c12, c22}};
    double S3i[3][3];
    if (!inv3_d(S3, S3i)) return kFitDependent;
    // T = -S3^-1 S2^T ; M = C1^-1 (S1 + S2 T), C1^-1 = [0 0 .5; 0 -1 0; .5 0 0]
    double T[3][3], R[3][3], M[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += S3i[r][k] * S2[c][k];
            T[r][c] = -s;
        }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double s = S1[r][c];
            for (int k = 0; k < 3; ++k) s += S2[r][k] * T[k][c];
            R[r][c] = s;
        }
    for (int c = 0; c < 3; ++c) {
        M[0][c] = 0.5 * R[2][c];
        M[1][c] = -R[1][c];
        M[2][c] = 0.5 * R[0][c];
    }
    // eigenvector with the smallest positive 4 v0 v2 - v1^2 (Fitting.cpp:102-128)
    const double tr = M[0][0] + M[1][1] + M[2][2];
    const double m2 = M[0][0] * M[1][1] - M[0][1] * M[1][0] + M[0][0] * M[2][2] - M[0][2] * M[2][0] +
                      M[1][1] * M[2][2] - M[1][2] * M[2][1];
    const double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) -
                       M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                       M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
    FitCplx lam[3];
    cubic_roots_real(-tr, m2, -det, lam);
    const double eps = double(FLT_EPSILON);
    int imin = -1;
    double minv = DBL_MAX;
    double vecs[3][3];
    for (int i = 0; i < 3; ++i) {
        eigvec_real(M, lam[i], vecs[i]);
        const double cond = 4 * vecs[i][0] * vecs[i][2] - vecs[i][1] * vecs[i][1];
        if (cond > eps && cond < minv) {
            imin = i;
            minv = cond;
        }
    }
    if (imin < 0) return kFitDegenerate;
    double coef[6];
    for (int k = 0; k < 3; ++k) coef[k] = vecs[imin][k];
    for (int k = 0; k < 3; ++k) coef[3 + k] = T[k][0] * coef[0] + T[k][1] * coef[1] + T[k][2] * coef[2];
    // to_ellipse, Fitting.cpp:131-169
    double idet = coef[0] * coef[2] - coef[1] * coef[1] / 4;
    idet = idet > eps ? 1.0 / idet : 0.0;
    const double scale = ::sqrt(idet / 4);
    if (scale < eps) return kFitSingular1;
    for (double& v : coef) v *= scale;
    const double aa = coef[0], bb = coef[1], cc = coef[2], dd = coef[3], ee = coef[4];
    double ff = coef[5];
    const double cxo = 2 * (-dd * cc + ee * bb / 2), cyo = 2 * (-aa * ee + dd * bb / 2);
    ff += aa * cxo * cxo + bb * cxo * cyo + cc * cyo * cyo + dd * cxo + ee * cyo;
    if (::fabs(ff) < eps) return kFitSingular2;
    double S[2][2] = {{aa / -ff, bb / 2 / -ff}, {bb / 2 / -ff, cc / -ff}};
    double V[2][2], d[2];
    jacobi2(S, V, d);
    // singular values in decreasing order, with their left singular vectors
    const int i0 = ::fabs(d[0]) >= ::fabs(d[1]) ? 0 : 1, i1 = 1 - i0;
    const double s0 = ::fabs(d[i0]), s1 = ::fabs(d[i1]);
    const double u01 = V[0][i1], u11 = V[1][i1];
    const double r0 = ::sqrt(1.0 / s0), r1 = ::sqrt(1.0 / s1);
    const double angle = pm::kPi - pm::atan2_d(u01, u11);
    if (!(r0 > 0) || !(r1 > 0) || !(r0 <= DBL_MAX) || !(r1 <= DBL_MAX)) return kFitLineOrPoint;
    ocx = float(cxo + ox);
    ocy = float(cyo + oy);
    oa = float(r0);
    ob = float(r1);
    oangle = float(angle);
    return kFitOk;
}

// Symmetric Jacobi eigen decomposition (n <= 4), eigenvectors in columns:
// cyclic sweeps over (p, q) in row order until the off-diagonal mass is below
// 1e-28 of the diagonal's (or 1e-300), at most 100 sweeps.
template <int N>
CCTAGB_HD inline void jacobi_sym(double A[N][N], double V[N][N], double d[N])
{
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) V[i][j] = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, diag = 0.0;
        for (int i = 0; i < N; ++i) {
            diag += A[i][i] * A[i][i];
            for (int j = i + 1; j < N; ++j) off += A[i][j] * A[i][j];
        }
        // converged: off-diagonal below 1e-14 of the diagonal (the absolute
        // test alone never fires once rounding noise is all that is left)
        if (off < 1e-300 || off <= 1e-28 * diag) break;
        for (int p = 0; p < N; ++p)
            for (int q = p + 1; q < N; ++q) {
                if (::fabs(A[p][q]) < 1e-300) continue;
                const double theta = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (::fabs(theta) + ::sqrt(theta * theta + 1.0));
                const double c = 1.0 / ::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < N; ++k) {
                    const double akp = A[k][p], akq = A[k][q];
                    A[k][p] = c * akp - s * akq;
                    A[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < N; ++k) {
                    const double apk = A[p][k], aqk = A[q][k];
                    A[p][k] = c * apk - s * aqk;
                    A[q][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < N; ++k) {
                    const double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = c * vkp - s * vkq;
                    V[k][q] = s * vkp + c * vkq;
                }
            }
    }
    for (int i = 0; i < N; ++i) d[i] = A[i][i];
}

// The circle fit on n points read through `pt(i, x, y)`: center and radius in
// FP64; false when the radius is not positive (the reference throws).  The
// normal matrix is summed in point order.
template <class PointAt>
CCTAGB_HD inline bool fit_circle_core(PointAt pt, size_t n, double& xc, double& yc, double& r)
{
    double A[4][4] = {};
    for (size_t i = 0; i < n; ++i) {
        float xf, yf;
        pt(i, xf, yf);
        const double row[4] = {xf, yf, 1.0, double(xf) * xf + double(yf) * yf};
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) A[a][b] += row[a] * row[b];
    }
    double V[4][4], d[4];
    jacobi_sym<4>(A, V, d);
    int k = 0;
    for (int i = 1; i < 4; ++i)
        if (d[i] < d[k]) k = i;
    const double v0 = V[0][k], v1 = V[1][k], v2 = V[2][k], v3 = V[3][k];
    xc = -0.5 * v0 / v3;
    yc = -0.5 * v1 / v3;
    r = ::sqrt(xc * xc + yc * yc - v2 / v3);
    return r > 0.0;
}

}  // namespace geo
}  // namespace cctagb
