// TEST INFRASTRUCTURE ONLY -- FP64 oracle for the batched identification
// calls (cctagb_identify_tasks, cctagb_cut_cost).
//
// Restates in double precision, for one candidate given as a cctagb_cut_task:
//  - the trial homography of an imaged center (Ellipse.cpp:161-214 canonic
//    form, Identification.cpp:739-798), here templated so that a dual number
//    carries d/dcenter through it;
//  - the cut signals (Identification.cpp:216-280 extractSignalUsingHomography:
//    stop point back-projected through H^-1, samples on [beginSig, 1] of the
//    ray, forward through H, bilinear / 2, Identification.hpp:197-219; a sample
//    outside the candidate's rectangle drops its cut);
//  - the cost (Identification.cpp:1122-1158 costFunctionGlob: mean over cut
//    pairs of the summed squared differences);
//  - its analytic gradient with respect to H and the center (the adjoint of
//    the steps above);
//  - the grid refinement (Identification.cpp:813-965, 1071-1109) continued to
//    a caller-chosen step, the FP64 localisation reference.
// Only the tests and the bench's accuracy check call it.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "cctag_b200.h"

namespace {

// value and derivatives along the two center coordinates
struct Dd {
    double v, a, b;
};
inline Dd cst(double v) { return Dd{v, 0, 0}; }
inline Dd operator+(Dd p, Dd q) { return Dd{p.v + q.v, p.a + q.a, p.b + q.b}; }
inline Dd operator-(Dd p, Dd q) { return Dd{p.v - q.v, p.a - q.a, p.b - q.b}; }
inline Dd operator*(Dd p, Dd q) { return Dd{p.v * q.v, p.a * q.v + p.v * q.a, p.b * q.v + p.v * q.b}; }
inline Dd operator/(Dd p, Dd q)
{
    const double r = p.v / q.v;
    return Dd{r, (p.a - r * q.a) / q.v, (p.b - r * q.b) / q.v};
}
inline Dd sqrt_(Dd p)
{
    const double r = std::sqrt(p.v);
    return Dd{r, p.a / (2 * r), p.b / (2 * r)};
}
inline double sqrt_(double p) { return std::sqrt(p); }
inline double val(double x) { return x; }
inline double val(Dd x) { return x.v; }
template <class T>
T lift(double v);
template <>
double lift<double>(double v)
{
    return v;
}
template <>
Dd lift<Dd>(double v)
{
    return cst(v);
}

struct M3 {
    double m[9];
};

M3 mul(const M3& a, const M3& b)
{
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i * 3 + j] = a.m[i * 3] * b.m[j] + a.m[i * 3 + 1] * b.m[3 + j] + a.m[i * 3 + 2] * b.m[6 + j];
    return r;
}

bool inv(const M3& a, M3& r)
{
    const double* m = a.m;
    const double c00 = m[4] * m[8] - m[5] * m[7], c01 = m[5] * m[6] - m[3] * m[8], c02 = m[3] * m[7] - m[4] * m[6];
    const double det = m[0] * c00 + m[1] * c01 + m[2] * c02;
    if (det == 0 || !std::isfinite(det)) return false;
    const double id = 1 / det;
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

// Ellipse.cpp:161-214
void canonic(const double* Q, M3& C, M3& Tp, M3& Td)
{
    const double q1 = Q[0], q2 = Q[1], q3 = Q[2], q4 = Q[4], q5 = Q[5], q6 = Q[8];
    const double par1 = q1, par2 = 2 * q2, par3 = q4, par4 = 2 * q3, par5 = 2 * q5;
    const double th = 0.5 * std::atan2(par2, par1 - par3);
    const double ct = std::cos(th), st = std::sin(th);
    const double s2 = st * st, c2 = ct * ct, cs = st * ct;
    const double Au = par4 * ct + par5 * st, Av = -par4 * st + par5 * ct;
    const double Auu = par1 * c2 + par3 * s2 + par2 * cs, Avv = par1 * s2 + par3 * c2 - par2 * cs;
    const double tu = -Au / (2 * Auu), tv = -Av / (2 * Avv);
    const double uc = tu * ct - tv * st, vc = tu * st + tv * ct;
    const double t1 = ct * (ct * q1 + q2 * st) + st * (ct * q2 + q4 * st);
    const double t2 = ct * (ct * q2 + q4 * st) - st * (ct * q1 + q2 * st);
    const double t3 = ct * q3 + q5 * st + uc * (ct * q1 + q2 * st) + vc * (ct * q2 + q4 * st);
    const double t4 = ct * (ct * q4 - q2 * st) - st * (ct * q2 - q1 * st);
    const double t5 = ct * q5 - q3 * st + uc * (ct * q2 - q1 * st) + vc * (ct * q4 - q2 * st);
    const double t6 = q6 + uc * (q3 + q1 * uc + q2 * vc) + vc * (q5 + q2 * uc + q4 * vc) + q3 * uc + q5 * vc;
    C = M3{{t1, t2, t3, t2, t4, t5, t3, t5, t6}};
    Tp = M3{{ct, st, -ct * uc - st * vc, -st, ct, st * uc - ct * vc, 0, 0, ct * ct + st * st}};
    Td = M3{{ct, -st, uc, st, ct, vc, 0, 0, 1}};
}

// Identification.cpp:739-798, on a scalar that may carry d/dcenter.
template <class T>
void homography(const M3& C, const M3& Tp, const M3& Td, T x, T y, T H[9])
{
    const T u = x * lift<T>(Tp.m[0]) + y * lift<T>(Tp.m[1]) + lift<T>(Tp.m[2]);
    const T v = x * lift<T>(Tp.m[3]) + y * lift<T>(Tp.m[4]) + lift<T>(Tp.m[5]);
    const T w = x * lift<T>(Tp.m[6]) + y * lift<T>(Tp.m[7]) + lift<T>(Tp.m[8]);
    const T xc = u / w, yc = v / w;
    const T Q11 = lift<T>(C.m[0]), Q22 = lift<T>(C.m[4]), Q33 = lift<T>(C.m[8]);
    T h[9] = {Q33,           Q22 * xc * yc,  lift<T>(0) - Q33 * xc,
              lift<T>(0),    lift<T>(0) - Q11 * xc * xc - Q33, lift<T>(0) - Q33 * yc,
              lift<T>(0) - Q11 * xc, Q22 * yc, lift<T>(0) - Q33};
    const T d0 = sqrt_(Q22 * Q33 / Q11 * (Q11 * xc * xc + Q22 * yc * yc + Q33));
    const T d2 = sqrt_(lift<T>(0) - Q22 * (Q11 * xc * xc + Q33));
    for (int i = 0; i < 3; ++i) {
        h[i * 3 + 0] = h[i * 3 + 0] * d0;
        h[i * 3 + 1] = h[i * 3 + 1] * Q33;
        h[i * 3 + 2] = h[i * 3 + 2] * d2;
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            H[i * 3 + j] = h[j] * lift<T>(Td.m[i * 3]) + h[3 + j] * lift<T>(Td.m[i * 3 + 1]) +
                           h[6 + j] * lift<T>(Td.m[i * 3 + 2]);
}

struct Img {
    const uint8_t* p;
    size_t pitch;
    int x0, y0, x1, y1;
    bool inside(double x, double y) const { return x >= x0 && x < x1 - 1 && y >= y0 && y < y1 - 1; }
    // Identification.hpp:197-219 and its gradient
    double sample(double x, double y, double* gx = nullptr, double* gy = nullptr) const
    {
        const int px = int(x), py = int(y);
        const uint8_t* q = p + px + size_t(py) * pitch;
        const double fx = x - px, fy = y - py;
        const double p1 = q[0], p2 = q[1], p3 = q[pitch], p4 = q[pitch + 1];
        if (gx) *gx = ((p2 - p1) * (1 - fy) + (p4 - p3) * fy) / 2;
        if (gy) *gy = ((p3 - p1) * (1 - fx) + (p4 - p2) * fx) / 2;
        return (p1 * (1 - fx) * (1 - fy) + p2 * fx * (1 - fy) + p3 * (1 - fx) * fy + p4 * fx * fy) / 2;
    }
};

Img image_of(const uint8_t* img, size_t pitch, const cctagb_cut_task& t)
{
    if (t.local)  // coordinates relative to the rectangle's corner
        return Img{img + size_t(t.roi[1]) * pitch + size_t(t.roi[0]), pitch, 0, 0, t.roi[2], t.roi[3]};
    return Img{img, pitch, t.roi[0], t.roi[1], t.roi[0] + t.roi[2], t.roi[1] + t.roi[3]};
}

// Cost at homography H; with grad_h (9) the analytic gradient with respect to
// the entries of H.  Returns false when fewer than two cuts stay inside (or H
// is singular).
bool cost_at(const Img& I, const cctagb_cut_task& t, const M3& H, int nS, double bs, double& cost, double* grad_h,
             std::vector<char>* sticky = nullptr)
{
    M3 Hi;
    if (!inv(H, Hi)) return false;
    const int nc = t.ncuts;
    std::vector<double> sig(size_t(nc) * nS), bxv(nc), byv(nc), z2v(nc);
    std::vector<char> ok(nc, 1);
    for (int c = 0; c < nc; ++c) {
        if (sticky && (*sticky)[c]) {
            ok[c] = 0;
            continue;
        }
        const double px = t.stop[c][0], py = t.stop[c][1];
        const double z0 = Hi.m[0] * px + Hi.m[1] * py + Hi.m[2];
        const double z1 = Hi.m[3] * px + Hi.m[4] * py + Hi.m[5];
        const double z2 = Hi.m[6] * px + Hi.m[7] * py + Hi.m[8];
        const double bx = z0 / z2, by = z1 / z2;
        bxv[c] = bx;
        byv[c] = by;
        z2v[c] = z2;
        const double xs = bx * bs, ys = by * bs;
        const double sx = (bx - xs) / (nS - 1), sy = (by - ys) / (nS - 1);
        for (int k = 0; k < nS; ++k) {
            const double x = xs + k * sx, y = ys + k * sy;
            const double u = H.m[0] * x + H.m[1] * y + H.m[2];
            const double v = H.m[3] * x + H.m[4] * y + H.m[5];
            const double w = H.m[6] * x + H.m[7] * y + H.m[8];
            const double qx = u / w, qy = v / w;
            if (!I.inside(qx, qy)) {
                ok[c] = 0;
                if (sticky) (*sticky)[c] = 1;
                break;
            }
            sig[size_t(c) * nS + k] = I.sample(qx, qy);
        }
    }
    int n = 0;
    for (int c = 0; c < nc; ++c) n += ok[c];
    if (n < 2) return false;
    const double pairs = 0.5 * n * (n - 1);
    std::vector<double> mean(nS);
    double acc = 0;
    for (int k = 0; k < nS; ++k) {
        double s1 = 0, s2 = 0;
        for (int c = 0; c < nc; ++c)
            if (ok[c]) {
                const double v = sig[size_t(c) * nS + k];
                s1 += v;
                s2 += v * v;
            }
        mean[k] = s1 / n;
        acc += n * s2 - s1 * s1;
    }
    cost = acc / pairs;
    if (!grad_h) return true;
    double G[9] = {}, GHi[9] = {};
    const double coef = 2.0 * n / pairs;
    for (int c = 0; c < nc; ++c) {
        if (!ok[c]) continue;
        const double bx = bxv[c], by = byv[c], z2 = z2v[c];
        const double xs = bx * bs, ys = by * bs;
        const double sx = (bx - xs) / (nS - 1), sy = (by - ys) / (nS - 1);
        double gbx = 0, gby = 0;
        for (int k = 0; k < nS; ++k) {
            const double x = xs + k * sx, y = ys + k * sy;
            const double u = H.m[0] * x + H.m[1] * y + H.m[2];
            const double v = H.m[3] * x + H.m[4] * y + H.m[5];
            const double w = H.m[6] * x + H.m[7] * y + H.m[8];
            const double qx = u / w, qy = v / w;
            double gx, gy;
            I.sample(qx, qy, &gx, &gy);
            const double lam = coef * (sig[size_t(c) * nS + k] - mean[k]);
            const double fx = lam * gx, fy = lam * gy, fw = -(fx * qx + fy * qy);
            const double y3[3] = {x, y, 1};
            for (int j = 0; j < 3; ++j) {
                G[j] += fx * y3[j] / w;
                G[3 + j] += fy * y3[j] / w;
                G[6 + j] += fw * y3[j] / w;
            }
            const double fX = (fx * (H.m[0] - qx * H.m[6]) + fy * (H.m[3] - qy * H.m[6])) / w;
            const double fY = (fx * (H.m[1] - qx * H.m[7]) + fy * (H.m[4] - qy * H.m[7])) / w;
            const double tk = bs + k * (1 - bs) / (nS - 1);
            gbx += tk * fX;
            gby += tk * fY;
        }
        const double dz[3] = {gbx / z2, gby / z2, -(gbx * bx + gby * by) / z2};
        const double p3[3] = {t.stop[c][0], t.stop[c][1], 1};
        for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q) GHi[r * 3 + q] += dz[r] * p3[q];
    }
    // d/dH through Hi = H^-1: -Hi^T GHi Hi^T
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double a = 0;
            for (int p = 0; p < 3; ++p)
                for (int q = 0; q < 3; ++q) a += Hi.m[p * 3 + i] * GHi[p * 3 + q] * Hi.m[j * 3 + q];
            G[i * 3 + j] -= a;
        }
    for (int j = 0; j < 9; ++j) grad_h[j] = G[j];
    return true;
}

}  // namespace

extern "C" {

/* Cost of the task at homography H (row-major 9); returns 0 and FLT_MAX when
 * fewer than two cuts stay inside.  grad_h (9, may be null): d cost / d H. */
int orc_cut_cost_h(const uint8_t* img, size_t pitch, const cctagb_cut_task* t, const double* H, int nS,
                   double beginSig, double* cost, double* grad_h)
{
    M3 Hm;
    std::memcpy(Hm.m, H, sizeof(Hm.m));
    double c = 0;
    const bool ok = cost_at(image_of(img, pitch, *t), *t, Hm, nS, beginSig, c, grad_h);
    *cost = ok ? c : DBL_MAX;
    if (!ok && grad_h) std::fill(grad_h, grad_h + 9, 0.0);
    return ok ? 1 : 0;
}

/* Cost at imaged center (cx, cy) and out[12] = cost, d/dcenter (2), d/dH (9);
 * H_out (9, may be null) receives the trial homography. */
int orc_cut_cost(const uint8_t* img, size_t pitch, const cctagb_cut_task* t, double cx, double cy, int nS,
                 double beginSig, double* out, double* H_out)
{
    double Q[9];
    for (int k = 0; k < 9; ++k) Q[k] = t->Q[k];
    M3 C, Tp, Td;
    canonic(Q, C, Tp, Td);
    Dd Hd[9];
    homography<Dd>(C, Tp, Td, Dd{cx, 1, 0}, Dd{cy, 0, 1}, Hd);
    M3 H;
    for (int k = 0; k < 9; ++k) H.m[k] = Hd[k].v;
    if (H_out) std::memcpy(H_out, H.m, sizeof(H.m));
    double g[9];
    double c = 0;
    const bool ok = cost_at(image_of(img, pitch, *t), *t, H, nS, beginSig, c, g);
    std::fill(out, out + 12, 0.0);
    if (!ok) {
        out[0] = DBL_MAX;
        return 0;
    }
    out[0] = c;
    for (int j = 0; j < 9; ++j) {
        out[1] += g[j] * Hd[j].a;
        out[2] += g[j] * Hd[j].b;
        out[3 + j] = g[j];
    }
    return 1;
}

/* The reference's grid refinement in FP64 (5x5 by default, conditioned by
 * the ellipse, shrinking by (grid-1)/2, cuts leaving the rectangle dropped
 * for good), continued until the grid step times the larger semi-axis
 * falls to `stop_width` (0.02 px in the reference).  out[3] = x, y, cost.
 * Returns 0 when no trial was readable. */
int orc_refine_grid(const uint8_t* img, size_t pitch, const cctagb_cut_task* t, int nS, double beginSig, int gridN,
                    double neighbourSize, double stop_width, double* out)
{
    double Q[9];
    for (int k = 0; k < 9; ++k) Q[k] = t->Q[k];
    M3 C, Tp, Td;
    canonic(Q, C, Tp, Td);
    const double sqrt2 = std::sqrt(2.0), meanAB = (double(t->a) + double(t->b)) / 2;
    const M3 mT{{sqrt2 / meanAB, 0, -sqrt2 * t->cx / meanAB, 0, sqrt2 / meanAB, -sqrt2 * t->cy / meanAB, 0, 0, 1}};
    M3 mTi;
    inv(mT, mTi);
    M3 mTiT;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) mTiT.m[i * 3 + j] = mTi.m[j * 3 + i];
    M3 Qm;
    std::memcpy(Qm.m, Q, sizeof(Q));
    const M3 Qc = mul(mTiT, mul(Qm, mTi));
    // semi axes of the conditioned conic (Ellipse.cpp:103-159)
    double ca, cb;
    {
        const double* q = Qc.m;
        const double p0 = q[0], p1 = 2 * q[1], p2 = q[4], p3 = 2 * q[2], p4 = 2 * q[5], p5 = q[8];
        const double th = 0.5 * std::atan2(p1, p0 - p2);
        const double ct = std::cos(th), st = std::sin(th);
        const double Au = p3 * ct + p4 * st, Av = -p3 * st + p4 * ct;
        const double Auu = p0 * ct * ct + p2 * st * st + p1 * st * ct, Avv = p0 * st * st + p2 * ct * ct - p1 * st * ct;
        const double tu = -Au / (2 * Auu), tv = -Av / (2 * Avv);
        const double wc = p5 - Auu * tu * tu - Avv * tv * tv;
        ca = std::sqrt(std::fabs(-wc / Auu));
        cb = std::sqrt(std::fabs(-wc / Avv));
    }
    const Img I = image_of(img, pitch, *t);
    std::vector<char> sticky(size_t(std::max(t->ncuts, 1)), 0);
    double cx = t->x0, cy = t->y0, best = DBL_MAX;
    double ns = neighbourSize;
    const double maxSemi = std::max(double(t->a), double(t->b));
    bool any = false;
    for (int round = 0; ns * maxSemi > stop_width && round < 64; ++round) {  // 64: the kernel's bound
        const double size = ns * std::max(ca, cb);
        const double half = size / 2, step = size / (gridN - 1);
        const double ccx = mT.m[0] * cx + mT.m[1] * cy + mT.m[2];
        const double ccy = mT.m[3] * cx + mT.m[4] * cy + mT.m[5];
        double rb = DBL_MAX, bx = cx, by = cy;
        bool has = false;
        for (int i = 0; i < gridN; ++i)
            for (int j = 0; j < gridN; ++j) {
                const double qx = ccx - half + i * step, qy = ccy - half + j * step;
                const double w = mTi.m[6] * qx + mTi.m[7] * qy + mTi.m[8];
                const double px = (mTi.m[0] * qx + mTi.m[1] * qy + mTi.m[2]) / w;
                const double py = (mTi.m[3] * qx + mTi.m[4] * qy + mTi.m[5]) / w;
                double H[9];
                homography<double>(C, Tp, Td, px, py, H);
                M3 Hm;
                std::memcpy(Hm.m, H, sizeof(H));
                double c;
                if (cost_at(I, *t, Hm, nS, beginSig, c, nullptr, &sticky)) {
                    has = true;
                    if (c < rb) {
                        rb = c;
                        bx = px;
                        by = py;
                    }
                }
            }
        if (!has) break;
        any = true;
        cx = bx;
        cy = by;
        best = rb;
        ns /= double((gridN - 1) / 2);
    }
    out[0] = cx;
    out[1] = cy;
    out[2] = best;
    return any ? 1 : 0;
}

}  // extern "C"
