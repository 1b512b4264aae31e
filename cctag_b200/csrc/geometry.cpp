// Ellipse and circle fits of the host candidate stage (Fitting.cpp of the
// reference, restated without Eigen: the small eigen/singular problems are
// solved in FP64 here).
#include "geometry.hpp"
#include "cctag_b200/portable/fit_core.hpp"

#include <limits>

namespace cctagb {
namespace geo {

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
    double xc, yc, r;
    const bool ok = fit_circle_core(
        [p](size_t i, float& x, float& y) {
            x = p[i].x;
            y = p[i].y;
        },
        n, xc, yc, r);
    if (!ok) throw std::domain_error("Degenerate circle in circleFitting");
    return Ellipse::from_params(float(xc), float(yc), float(r), float(r), 0.f);
}

}  // namespace geo
}  // namespace cctagb
