// Ellipse and circle fits of the host candidate stage (Fitting.cpp of the
// reference, restated without Eigen: the small eigen/singular problems are
// solved in FP64 here).
#include "geometry.hpp"
#include "fit_core.hpp"

#include <limits>

namespace cctagb {
namespace geo {

namespace {

// Symmetric Jacobi eigen decomposition (n <= 4), eigenvectors in columns.
template <int N>
void jacobi(double A[N][N], double V[N][N], double d[N])
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

}  // namespace

Ellipse fit_ellipse(const Pt* p, size_t n)
{
    float cx = 0.f, cy = 0.f, a = 0.f, b = 0.f, angle = 0.f;
    const int st = fit_ellipse_core(
        [p](size_t i, float& x, float& y) {
            x = p[i].x;
            y = p[i].y;
        },
        n, cx, cy, a, b, angle);
    switch (st) {
    case kFitOk: break;
    case kFitTooFewPoints: throw std::domain_error("fitEllipse: at least 5 points are needed");
    case kFitDependent: throw std::domain_error("fit_solver: the input points appear to be linearly dependent");
    case kFitDegenerate: throw std::domain_error("fit_solver: degeneracy");
    case kFitSingular1: throw std::domain_error("to_ellipse_2: singularity 1");
    case kFitSingular2: throw std::domain_error("to_ellipse_2: singularity 2");
    default: throw std::domain_error("Degenerate ellipse after fitEllipse => line or point.");
    }
    return Ellipse::from_params(cx, cy, a, b, angle);
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
