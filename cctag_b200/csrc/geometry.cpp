// Ellipse and circle fits of the host candidate stage (Fitting.cpp of the
// reference, restated without Eigen: the small eigen/singular problems are
// solved in FP64 here).
#include "geometry.hpp"

#include <complex>
#include <limits>

namespace cctagb {
namespace geo {

namespace {

using cd = std::complex<double>;

// Roots of x^3 + a x^2 + b x + c (complex arithmetic, Cardano).
void cubic_roots(double a, double b, double c, cd r[3])
{
    const double p = b - a * a / 3.0;
    const double q = 2.0 * a * a * a / 27.0 - a * b / 3.0 + c;
    const cd disc = cd(q * q / 4.0 + p * p * p / 27.0, 0.0);
    const cd sq = std::sqrt(disc);
    cd u = std::pow(-q / 2.0 + sq, 1.0 / 3.0);
    if (std::abs(u) < 1e-300) u = std::pow(-q / 2.0 - sq, 1.0 / 3.0);
    const cd w(-0.5, std::sqrt(3.0) / 2.0);
    for (int k = 0; k < 3; ++k) {
        cd uk = u;
        for (int j = 0; j < k; ++j) uk *= w;
        const cd vk = std::abs(uk) < 1e-300 ? cd(0.0) : -p / (3.0 * uk);
        r[k] = uk + vk - a / 3.0;
    }
    // One Newton polish per root on the original cubic.
    for (int k = 0; k < 3; ++k) {
        for (int it = 0; it < 3; ++it) {
            const cd x = r[k];
            const cd f = ((x + a) * x + b) * x + c;
            const cd df = (3.0 * x + 2.0 * a) * x + b;
            if (std::abs(df) < 1e-300) break;
            r[k] = x - f / df;
        }
    }
}

// Unit eigenvector of M for eigenvalue lam: the largest cross product of two
// rows of (M - lam I).  Real part returned, as Eigen's EigenSolver().real().
void eigvec(const double M[3][3], cd lam, double out[3])
{
    cd A[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) A[i][j] = cd(M[i][j]) - (i == j ? lam : cd(0.0));
    cd best[3] = {cd(0), cd(0), cd(0)};
    double bn = -1.0;
    for (int i = 0; i < 3; ++i)
        for (int j = i + 1; j < 3; ++j) {
            const cd c[3] = {A[i][1] * A[j][2] - A[i][2] * A[j][1], A[i][2] * A[j][0] - A[i][0] * A[j][2],
                             A[i][0] * A[j][1] - A[i][1] * A[j][0]};
            const double n = std::norm(c[0]) + std::norm(c[1]) + std::norm(c[2]);
            if (n > bn) {
                bn = n;
                for (int k = 0; k < 3; ++k) best[k] = c[k];
            }
        }
    const double nrm = std::sqrt(std::max(bn, 0.0));
    if (!(nrm > 0.0)) {
        out[0] = out[1] = out[2] = 0.0;
        return;
    }
    // Fix the phase so that the largest component is real, then normalise.
    int kmax = 0;
    for (int k = 1; k < 3; ++k)
        if (std::abs(best[k]) > std::abs(best[kmax])) kmax = k;
    const cd ph = std::abs(best[kmax]) > 0 ? std::conj(best[kmax]) / std::abs(best[kmax]) : cd(1.0);
    for (int k = 0; k < 3; ++k) out[k] = (best[k] * ph / nrm).real();
}

// Symmetric Jacobi eigen decomposition (n <= 4), eigenvectors in columns.
template <int N>
void jacobi(double A[N][N], double V[N][N], double d[N])
{
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) V[i][j] = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int i = 0; i < N; ++i)
            for (int j = i + 1; j < N; ++j) off += A[i][j] * A[i][j];
        if (off < 1e-300) break;
        for (int p = 0; p < N; ++p)
            for (int q = p + 1; q < N; ++q) {
                if (std::fabs(A[p][q]) < 1e-300) continue;
                const double theta = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
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

bool inv3(const double a[3][3], double r[3][3])
{
    const double c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1];
    const double c01 = a[1][2] * a[2][0] - a[1][0] * a[2][2];
    const double c02 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
    const double det = a[0][0] * c00 + a[0][1] * c01 + a[0][2] * c02;
    double scale = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) scale = std::max(scale, std::fabs(a[i][j]));
    if (det == 0.0 || !std::isfinite(det) || std::fabs(det) <= 1e-14 * scale * scale * scale) return false;
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

}  // namespace

Ellipse fit_ellipse(const Pt* p, size_t n)
{
    if (n < 5) throw std::domain_error("fitEllipse: at least 5 points are needed");
    // Fitting.cpp:37-45 offset (mean), :47-71 scatter matrices.
    double ox = 0, oy = 0;
    for (size_t i = 0; i < n; ++i) {
        ox += p[i].x;
        oy += p[i].y;
    }
    ox /= double(n);
    oy /= double(n);
    double S1[3][3] = {}, S2[3][3] = {}, S3[3][3] = {};
    for (size_t i = 0; i < n; ++i) {
        const double x = p[i].x - ox, y = p[i].y - oy;
        const double q[3] = {x * x, x * y, y * y};
        const double l[3] = {x, y, 1.0};
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                S1[r][c] += q[r] * q[c];
                S2[r][c] += q[r] * l[c];
                S3[r][c] += l[r] * l[c];
            }
    }
    double S3i[3][3];
    if (!inv3(S3, S3i)) throw std::domain_error("fit_solver: the input points appear to be linearly dependent");
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
    // Eigen decomposition of M; keep the eigenvector with the smallest
    // positive 4 v0 v2 - v1^2 (the ellipse constraint), Fitting.cpp:102-128.
    const double tr = M[0][0] + M[1][1] + M[2][2];
    const double m2 = M[0][0] * M[1][1] - M[0][1] * M[1][0] + M[0][0] * M[2][2] - M[0][2] * M[2][0] +
                      M[1][1] * M[2][2] - M[1][2] * M[2][1];
    const double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) -
                       M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                       M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
    cd lam[3];
    cubic_roots(-tr, m2, -det, lam);
    const double eps = double(std::numeric_limits<float>::epsilon());
    int imin = -1;
    double minv = std::numeric_limits<double>::max();
    double vecs[3][3];
    for (int i = 0; i < 3; ++i) {
        eigvec(M, lam[i], vecs[i]);
        const double cond = 4 * vecs[i][0] * vecs[i][2] - vecs[i][1] * vecs[i][1];
        if (cond > eps && cond < minv) {
            imin = i;
            minv = cond;
        }
    }
    if (imin < 0) throw std::domain_error("fit_solver: degeneracy");
    double coef[6];
    for (int k = 0; k < 3; ++k) coef[k] = vecs[imin][k];
    for (int k = 0; k < 3; ++k) coef[3 + k] = T[k][0] * coef[0] + T[k][1] * coef[1] + T[k][2] * coef[2];
    // to_ellipse, Fitting.cpp:131-169
    double idet = coef[0] * coef[2] - coef[1] * coef[1] / 4;
    idet = idet > eps ? 1.0 / idet : 0.0;
    const double scale = std::sqrt(idet / 4);
    if (scale < eps) throw std::domain_error("to_ellipse_2: singularity 1");
    for (double& v : coef) v *= scale;
    const double aa = coef[0], bb = coef[1], cc = coef[2], dd = coef[3], ee = coef[4];
    double ff = coef[5];
    const double cxo = 2 * (-dd * cc + ee * bb / 2), cyo = 2 * (-aa * ee + dd * bb / 2);
    ff += aa * cxo * cxo + bb * cxo * cyo + cc * cyo * cyo + dd * cxo + ee * cyo;
    if (std::fabs(ff) < eps) throw std::domain_error("to_ellipse_2: singularity 2");
    double S[2][2] = {{aa / -ff, bb / 2 / -ff}, {bb / 2 / -ff, cc / -ff}};
    double V[2][2], d[2];
    jacobi<2>(S, V, d);
    // singular values in decreasing order, with their left singular vectors
    int i0 = std::fabs(d[0]) >= std::fabs(d[1]) ? 0 : 1, i1 = 1 - i0;
    const double s0 = std::fabs(d[i0]), s1 = std::fabs(d[i1]);
    const double u01 = V[0][i1], u11 = V[1][i1];
    const double r0 = std::sqrt(1.0 / s0), r1 = std::sqrt(1.0 / s1);
    const double angle = 3.14159265358979323846 - std::atan2(u01, u11);
    if (!(r0 > 0) || !(r1 > 0) || !std::isfinite(r0) || !std::isfinite(r1))
        throw std::domain_error("Degenerate ellipse after fitEllipse => line or point.");
    return Ellipse::from_params(float(cxo + ox), float(cyo + oy), float(r0), float(r1), float(angle));
}

Ellipse fit_circle(const Pt* p, size_t n)
{
    // Normal matrix of [x y 1 x^2+y^2]; its smallest eigenvector is the
    // smallest right singular vector of the design matrix.
    double A[4][4] = {};
    for (size_t i = 0; i < n; ++i) {
        const double r[4] = {p[i].x, p[i].y, 1.0, double(p[i].x) * p[i].x + double(p[i].y) * p[i].y};
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) A[a][b] += r[a] * r[b];
    }
    double V[4][4], d[4];
    jacobi<4>(A, V, d);
    int k = 0;
    for (int i = 1; i < 4; ++i)
        if (d[i] < d[k]) k = i;
    const double v0 = V[0][k], v1 = V[1][k], v2 = V[2][k], v3 = V[3][k];
    const double xc = -0.5 * v0 / v3, yc = -0.5 * v1 / v3;
    const double r = std::sqrt(xc * xc + yc * yc - v2 / v3);
    if (!(r > 0.0)) throw std::domain_error("Degenerate circle in circleFitting");
    return Ellipse::from_params(float(xc), float(yc), float(r), float(r), 0.f);
}

}  // namespace geo
}  // namespace cctagb
