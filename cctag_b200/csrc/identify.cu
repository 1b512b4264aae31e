// Identification on sm_100a: imaged-center refinement and ID reading, one
// thread block per marker (Identification.cpp:813-1158 refineConicFamilyGlob /
// imageCenterOptimizationGlob / costFunctionGlob / getSignals, and
// :50-193 orazioDistanceRobust, :1408-1436 ID vote).
//
// Grid refinement: each round evaluates a gridN x gridN set of trial centres
// (getNearbyPoints, conditioned by the ellipse) with one warp per trial.  A
// trial's homography maps the unit circle to the outer ellipse and the origin
// to the trial centre (computeHomographyFromEllipseAndImagedCenter); every cut
// is resampled in the marker plane along the ray to its back-projected end.
//
// The reference marks a cut "out of bounds" the first time any of its samples
// leaves the image, for every later trial and round (the flag lives in the cut
// object).  This kernel reproduces that order: the flags of all trials of a
// round are computed first (a cut's samples lie on the image of a segment, so
// its two end samples decide), then a prefix OR in trial order gives each
// trial the set of cuts the reference would still use.
//
// Cost: the reference's mean over cut pairs of sum_k (s_i[k] - s_j[k])^2, here
// in the equivalent form n * sum_i (s_i[k] - mean_k)^2 summed over k, divided
// by the n(n-1)/2 pairs (shifted FP32 sums per sample, FP64 over samples).
// The sample loop avoids the XU pipe (conversions, divisions), which bounds
// a straightforward version of it.
#include <cfloat>
#include <cstdint>

#include <cooperative_groups.h>

#include "common.hpp"
#include "ident_host.hpp"
#include "cctag_b200/portable/pmath.hpp"

namespace cctagb {

namespace {

constexpr int kMaxTrials = 25;
constexpr int kThreads = 32 * kMaxTrials;
constexpr int kWarps = kThreads / 32;
// The samples along a cut come in chunks of 32 (one per lane).  A marker is
// either one thread block doing every chunk, or a cluster of kCluster blocks,
// block r doing chunk r, whose per-chunk sums meet through distributed shared
// memory: few markers per launch spread over four SMs each, many markers
// keep one SM each.  Per-chunk sums are formed the same way in both, and
// added in chunk order, so both give the same bits.
constexpr int kChunk = 32;
constexpr int kMaxChunks = kMaxSamples / kChunk;
constexpr int kCluster = kMaxChunks;

__device__ __forceinline__ void mat_mul(const float* a, const float* b, float* r)
{
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r[i * 3 + j] = a[i * 3] * b[j] + a[i * 3 + 1] * b[3 + j] + a[i * 3 + 2] * b[6 + j];
}

__device__ __forceinline__ bool mat_inv(const float* a, float* r)
{
    const float c00 = a[4] * a[8] - a[5] * a[7];
    const float c01 = a[5] * a[6] - a[3] * a[8];
    const float c02 = a[3] * a[7] - a[4] * a[6];
    const float det = a[0] * c00 + a[1] * c01 + a[2] * c02;
    if (det == 0.f || !isfinite(det)) return false;
    const float id = 1.f / det;
    r[0] = c00 * id;
    r[1] = (a[2] * a[7] - a[1] * a[8]) * id;
    r[2] = (a[1] * a[5] - a[2] * a[4]) * id;
    r[3] = c01 * id;
    r[4] = (a[0] * a[8] - a[2] * a[6]) * id;
    r[5] = (a[2] * a[3] - a[0] * a[5]) * id;
    r[6] = c02 * id;
    r[7] = (a[1] * a[6] - a[0] * a[7]) * id;
    r[8] = (a[0] * a[4] - a[1] * a[3]) * id;
    return true;
}

__device__ __forceinline__ void apply_h(const float* H, float x, float y, float& ox, float& oy, float& w)
{
    const float u = H[0] * x + H[1] * y + H[2];
    const float v = H[3] * x + H[4] * y + H[5];
    w = H[6] * x + H[7] * y + H[8];
    ox = u / w;
    oy = v / w;
}

// The image a candidate is read from: a device image with its row pitch and
// the candidate's rectangle [x0, x1) x [y0, y1) (the whole frame in a
// detection; one crop of an atlas in the batched form).
struct Roi {
    const uint8_t* img;
    size_t pitch;
    int x0, y0, x1, y1;
};

__device__ __forceinline__ Roi make_roi(const uint8_t* img, size_t pitch, const IdentTask& T)
{
    if (T.local)  // coordinates relative to the rectangle's corner
        return Roi{img + size_t(T.roi[1]) * pitch + size_t(T.roi[0]), pitch, 0, 0, T.roi[2], T.roi[3]};
    return Roi{img, pitch, T.roi[0], T.roi[1], T.roi[0] + T.roi[2], T.roi[1] + T.roi[3]};
}

// Identification.hpp:197-219
__device__ __forceinline__ float bilinear(const Roi& R, float x, float y)
{
    const int px = int(x), py = int(y);
    const uint8_t* p0 = R.img + px + size_t(py) * R.pitch;
    const float fx = x - float(px), fy = y - float(py);
    const float fx1 = 1.0f - fx, fy1 = 1.0f - fy;
    const float p1 = __ldg(p0), p2 = __ldg(p0 + 1), p3 = __ldg(p0 + R.pitch), p4 = __ldg(p0 + R.pitch + 1);
    return (p1 * (fx1 * fy1) + p2 * (fx * fy1) + p3 * (fx1 * fy) + p4 * (fx * fy)) / 2;
}

// The reference's test "x >= 0 && x < cols - 1 && y >= 0 && y < rows - 1",
// on the candidate's rectangle.
__device__ __forceinline__ bool inside(const Roi& R, float x, float y)
{
    return x >= float(R.x0) && x < float(R.x1 - 1) && y >= float(R.y0) && y < float(R.y1 - 1);
}

// Ellipse.cpp:103-159 semi axes of a conic (for the conditioned ellipse).
__device__ void conic_axes(const float* Q, float& a, float& b)
{
    const float p0 = Q[0], p1 = 2.f * Q[1], p2 = Q[4], p3 = 2.f * Q[2], p4 = 2.f * Q[5], p5 = Q[8];
    const float th = 0.5f * atan2f(p1, p0 - p2);
    float st, ct;
    sincosf(th, &st, &ct);
    const float s2 = st * st, c2 = ct * ct, cs = st * ct;
    const float Au = p3 * ct + p4 * st, Av = -p3 * st + p4 * ct;
    const float Auu = p0 * c2 + p2 * s2 + p1 * cs, Avv = p0 * s2 + p2 * c2 - p1 * cs;
    if (Auu == 0.f || Avv == 0.f) {
        a = b = 0.f;
        return;
    }
    const float tu = -Au / (2.f * Auu), tv = -Av / (2.f * Avv);
    const float wc = p5 - Auu * tu * tu - Avv * tv * tv;
    a = sqrtf(fabsf(-wc / Auu));
    b = sqrtf(fabsf(-wc / Avv));
}

// Ellipse.cpp:161-214 canonic form: C (canonical conic), Tp (primal), Td (dual).
__device__ void canonic_form(const float* Q, float* C, float* Tp, float* Td)
{
    const float q1 = Q[0], q2 = Q[1], q3 = Q[2], q4 = Q[4], q5 = Q[5], q6 = Q[8];
    const float par1 = q1, par2 = 2 * q2, par3 = q4, par4 = 2 * q3, par5 = 2 * q5;
    const float th = 0.5f * atan2f(par2, par1 - par3);
    const float ct = cosf(th), st = sinf(th);
    const float s2 = st * st, c2 = ct * ct, cs = st * ct;
    const float Au = par4 * ct + par5 * st, Av = -par4 * st + par5 * ct;
    const float Auu = par1 * c2 + par3 * s2 + par2 * cs, Avv = par1 * s2 + par3 * c2 - par2 * cs;
    const float tu = -Au / (2 * Auu), tv = -Av / (2 * Avv);
    const float uc = tu * ct - tv * st, vc = tu * st + tv * ct;
    const float t1 = ct * (ct * q1 + q2 * st) + st * (ct * q2 + q4 * st);
    const float t2 = ct * (ct * q2 + q4 * st) - st * (ct * q1 + q2 * st);
    const float t3 = ct * q3 + q5 * st + uc * (ct * q1 + q2 * st) + vc * (ct * q2 + q4 * st);
    const float t4 = ct * (ct * q4 - q2 * st) - st * (ct * q2 - q1 * st);
    const float t5 = ct * q5 - q3 * st + uc * (ct * q2 - q1 * st) + vc * (ct * q4 - q2 * st);
    const float t6 = q6 + uc * (q3 + q1 * uc + q2 * vc) + vc * (q5 + q2 * uc + q4 * vc) + q3 * uc + q5 * vc;
    C[0] = t1; C[1] = t2; C[2] = t3; C[3] = t2; C[4] = t4; C[5] = t5; C[6] = t3; C[7] = t5; C[8] = t6;
    Tp[0] = ct;  Tp[1] = st; Tp[2] = -ct * uc - st * vc;
    Tp[3] = -st; Tp[4] = ct; Tp[5] = st * uc - ct * vc;
    Tp[6] = 0;   Tp[7] = 0;  Tp[8] = ct * ct + st * st;
    Td[0] = ct; Td[1] = -st; Td[2] = uc;
    Td[3] = st; Td[4] = ct;  Td[5] = vc;
    Td[6] = 0;  Td[7] = 0;   Td[8] = 1.f;
}

// Identification.cpp:739-798: homography (plane -> image) sending the unit
// circle to the ellipse and the origin to (x, y).
__device__ void homography_from_center(const float* C, const float* Tp, const float* Td, float x, float y, float* H)
{
    float xc, yc, w;
    apply_h(Tp, x, y, xc, yc, w);
    const float Q11 = C[0], Q22 = C[4], Q33 = C[8];
    float h[9];
    h[0] = Q33;      h[1] = Q22 * xc * yc;           h[2] = -Q33 * xc;
    h[3] = 0.f;      h[4] = -Q11 * xc * xc - Q33;    h[5] = -Q33 * yc;
    h[6] = -Q11 * xc; h[7] = Q22 * yc;               h[8] = -Q33;
    const float d0 = sqrtf((Q22 * Q33 / Q11 * (Q11 * xc * xc + Q22 * yc * yc + Q33)));
    const float d1 = Q33;
    const float d2 = sqrtf(-Q22 * (Q11 * xc * xc + Q33));
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        h[i * 3 + 0] *= d0;
        h[i * 3 + 1] *= d1;
        h[i * 3 + 2] *= d2;
    }
    mat_mul(Td, h, H);
}

struct Shared {
    float C[9], Tp[9], Td[9];
    float mT[9], mTi[9];
    float nsScale;                 // max semi axis of the conditioned ellipse
    float cx, cy;                  // current center
    float Hopt[9];
    float minRes;
    uint32_t oob;                  // sticky out-of-bounds cut mask
    int rounds;
    int fail;
    float trialH[kMaxTrials][9];
    float trialPt[kMaxTrials][2];
    union {
        float cutp[kMaxTrials][kMaxCuts][6];  // grid: image line of the cut's samples, U0 dU V0 dV W0 dW
        struct {                              // Gauss-Newton: one chunk of samples
            float s[kMaxCuts][kChunk];        // value
            float dx[kMaxCuts][kChunk];       // d value / d center x
            float dy[kMaxCuts][kChunk];       // d value / d center y
        } gn;
    } u;
    // Gauss-Newton state
    float gH[9], gHi[9], gdH[2][9], gdHi[2][9];  // homography at the trial center, inverse, center derivatives
    float gTry[2];                               // trial center
    uint32_t gOob;                               // cuts whose end samples leave the rectangle at the trial
    double gPart[2][kMaxChunks][6];              // per-chunk sums (cost, J^T r, J^T J) by parity
    double gSum[6];
    double gA[3], gG[2], gBest, gLambda;         // normal equations at the best center, its cost, damping
    int gHave, gStop, iterations;
    uint32_t trialOob[kMaxTrials];
    uint32_t valid[kMaxTrials];
    float cost[kMaxTrials];
    double part[2][kMaxChunks][kMaxTrials];  // per-chunk shares of each trial's cost (by round parity)
    float sig[kMaxCuts][kMaxSamples];
    float barcode[kMaxSamples];
    int winner[kMaxCuts];
    float vwin[kMaxCuts];
};

// Per trial (one warp): homography, the image line of each cut's samples and
// the cuts whose end samples leave the rectangle.
__device__ void setup_trial(Shared& S, const IdentTask& T, int t, float px, float py, const IdentParams& ip,
                            const Roi& R, int lane)
{
    float Hm[9], Hi[9];
    homography_from_center(S.C, S.Tp, S.Td, px, py, Hm);
    const bool ok = mat_inv(Hm, Hi);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 9; ++k) S.trialH[t][k] = Hm[k];
        S.trialPt[t][0] = px;
        S.trialPt[t][1] = py;
    }
    bool bad = false;
    if (lane < T.ncuts) {
        float bx, by, w;
        if (ok) apply_h(Hi, T.stop[lane][0], T.stop[lane][1], bx, by, w);
        else bx = by = NAN;
        const float xs = bx * ip.beginSig, ys = by * ip.beginSig;
        const float sx = (bx - xs) / (float(ip.nSamples) - 1.f), sy = (by - ys) / (float(ip.nSamples) - 1.f);
        // sample k is (xs + k sx, ys + k sy) in the marker plane; its image in
        // homogeneous coordinates is linear in k: H (xs, ys, 1) + k H (sx, sy, 0)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            S.u.cutp[t][lane][2 * i] = __fmaf_rn(Hm[3 * i], xs, __fmaf_rn(Hm[3 * i + 1], ys, Hm[3 * i + 2]));
            S.u.cutp[t][lane][2 * i + 1] = __fmaf_rn(Hm[3 * i], sx, __fmul_rn(Hm[3 * i + 1], sy));
        }
        // end samples, with the sample loop's own arithmetic
        const float* cp = S.u.cutp[t][lane];
        const float kl = float(ip.nSamples - 1);
        const float w0 = cp[4], w1 = __fmaf_rn(kl, cp[5], cp[4]);
        const float r0 = __fdividef(1.0f, w0), r1 = __fdividef(1.0f, w1);
        const float x0 = __fmul_rn(cp[0], r0), y0 = __fmul_rn(cp[2], r0);
        const float x1 = __fmul_rn(__fmaf_rn(kl, cp[1], cp[0]), r1), y1 = __fmul_rn(__fmaf_rn(kl, cp[3], cp[2]), r1);
        bad = !(w0 > 0.f && w1 > 0.f) && !(w0 < 0.f && w1 < 0.f);
        bad = bad || !inside(R, x0, y0) || !inside(R, x1, y1);
    }
    const uint32_t m = __ballot_sync(0xffffffffu, bad);
    if (lane == 0) S.trialOob[t] = m & ((T.ncuts >= 32) ? 0xffffffffu : ((1u << T.ncuts) - 1u));
}

// Byte -> float without a conversion instruction (exponent 2^23 trick).
__device__ __forceinline__ float byte_to_float(uint32_t b) { return __uint_as_float(0x4B000000u | b) - 8388608.f; }

// floor(x) for 0 <= x < 2^22 without a conversion instruction: adding 2^23
// with round-toward-zero leaves floor(x) in the mantissa.  Returns the
// integer and stores its float value in fl.
__device__ __forceinline__ int floor_small(float x, float& fl)
{
    const float t = __fadd_rz(x, 8388608.f);
    fl = t - 8388608.f;
    return __float_as_int(t) - 0x4B000000;
}

// The four pixels around a sample known to lie inside the rectangle (the
// integer corner is clamped so that rounding at the border never reads
// outside it), and the fractional offsets.
__device__ __forceinline__ void bilinear_taps(const Roi& R, float x, float y, float p[4], float& fx, float& fy)
{
    float fpx, fpy;
    int px = floor_small(fmaxf(x, 0.f), fpx);
    int py = floor_small(fmaxf(y, 0.f), fpy);
    fx = x - fpx;
    fy = y - fpy;
    px = min(max(px, R.x0), R.x1 - 2);
    py = min(max(py, R.y0), R.y1 - 2);
    const uint8_t* p0 = R.img + px + size_t(py) * R.pitch;
    p[0] = byte_to_float(__ldg(p0));
    p[1] = byte_to_float(__ldg(p0 + 1));
    p[2] = byte_to_float(__ldg(p0 + R.pitch));
    p[3] = byte_to_float(__ldg(p0 + R.pitch + 1));
}

// Identification.hpp:197-219 for a sample inside the rectangle (explicit
// roundings, so that every caller gets the same bits).
__device__ __forceinline__ float bilinear_value(const float p[4], float fx, float fy)
{
    const float fx1 = __fsub_rn(1.0f, fx), fy1 = __fsub_rn(1.0f, fy);
    float a = __fmul_rn(p[0], __fmul_rn(fx1, fy1));
    a = __fmaf_rn(p[1], __fmul_rn(fx, fy1), a);
    a = __fmaf_rn(p[2], __fmul_rn(fx1, fy), a);
    a = __fmaf_rn(p[3], __fmul_rn(fx, fy), a);
    return __fmul_rn(a, 0.5f);
}

__device__ __forceinline__ float bilinear_in(const Roi& R, float x, float y)
{
    float p[4], fx, fy;
    bilinear_taps(R, x, y, p, fx, fy);
    return bilinear_value(p, fx, fy);
}

// Same value and its gradient in x and y (the derivative of the bilinear
// patch the sample falls in).
__device__ __forceinline__ float bilinear_grad(const Roi& R, float x, float y, float& gx, float& gy)
{
    float p[4], fx, fy;
    bilinear_taps(R, x, y, p, fx, fy);
    const float fx1 = 1.0f - fx, fy1 = 1.0f - fy;
    gx = ((p[1] - p[0]) * fy1 + (p[3] - p[2]) * fy) * 0.5f;
    gy = ((p[2] - p[0]) * fx1 + (p[3] - p[1]) * fx) * 0.5f;
    return bilinear_value(p, fx, fy);
}

// Row i of H applied to (x, y, 1), explicit roundings.
__device__ __forceinline__ float hrow(const float* Hm, int i, float x, float y)
{
    return __fmaf_rn(Hm[3 * i], x, __fmaf_rn(Hm[3 * i + 1], y, Hm[3 * i + 2]));
}

// One sample of cut c of trial t: its point on the cut's image line, then a
// bilinear read (fast reciprocal: one MUFU op, no IEEE fix-up).
__device__ __forceinline__ float cut_sample(const Shared& S, const Roi& R, int t, int c, float kf)
{
    const float* cp = S.u.cutp[t][c];
    const float u = __fmaf_rn(kf, cp[1], cp[0]);
    const float v = __fmaf_rn(kf, cp[3], cp[2]);
    const float w = __fmaf_rn(kf, cp[5], cp[4]);
    const float r = __fdividef(1.0f, w);
    return bilinear_in(R, __fmul_rn(u, r), __fmul_rn(v, r));
}

// Sum over the 32 lanes (the same butterfly, so the same bits, everywhere).
__device__ __forceinline__ double lane_sum(double v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Per-chunk shares of the cost of trial t (one warp): chunks j0 .. j0+NCH-1
// (those below nch), lane = sample within the chunk, over the valid cuts in
// order, a few cuts at a time so that their reads overlap.  Per sample the
// cut values are shifted by the first valid cut's value before the FP32 sums
// (the term n * sum(d^2) - (sum d)^2 does not change under a common shift,
// and the shifted sums stay small); out[q] is the chunk's FP64 lane sum.
template <int NCH>
__device__ void trial_partial(const Shared& S, const Roi& R, int t, uint32_t valid, int j0, int nch, int nS,
                              int lane, double out[NCH])
{
    constexpr int G = NCH == 1 ? 4 : 2;  // cuts per step
    const int n = __popc(valid);
    float v0[NCH], s1[NCH], s2[NCH], kf[NCH];
    bool act[NCH];
#pragma unroll
    for (int q = 0; q < NCH; ++q) {
        const int k = (j0 + q) * kChunk + lane;
        act[q] = j0 + q < nch && k < nS;
        // lanes past the last sample read the last one again (in bounds, no
        // branch) and their terms are dropped below
        kf[q] = float(min(k, nS - 1));
        v0[q] = s1[q] = s2[q] = 0.f;
    }
    if (n >= 2) {
        uint32_t m = valid;
        bool first = true;  // the same in every lane: a uniform branch
        while (m) {
            int c[G];
            float keep[G];
#pragma unroll
            for (int g = 0; g < G; ++g) {
                // past the last valid cut: repeat it, with weight 0
                c[g] = m ? __ffs(m) - 1 : c[g > 0 ? g - 1 : 0];
                keep[g] = m ? 1.f : 0.f;
                m &= m - 1;
            }
            float val[G][NCH];
#pragma unroll
            for (int g = 0; g < G; ++g)
#pragma unroll
                for (int q = 0; q < NCH; ++q) val[g][q] = cut_sample(S, R, t, c[g], kf[q]);
            if (first) {
#pragma unroll
                for (int q = 0; q < NCH; ++q) v0[q] = val[0][q];  // first valid cut: the shift
                first = false;
            }
#pragma unroll
            for (int g = 0; g < G; ++g) {
#pragma unroll
                for (int q = 0; q < NCH; ++q) {
                    const float d = __fmul_rn(__fsub_rn(val[g][q], v0[q]), keep[g]);
                    s1[q] = __fadd_rn(s1[q], d);
                    s2[q] = __fmaf_rn(d, d, s2[q]);
                }
            }
        }
    }
#pragma unroll
    for (int q = 0; q < NCH; ++q) {
        const double term =
            (n >= 2 && act[q]) ? double(__fsub_rn(__fmul_rn(float(n), s2[q]), __fmul_rn(s1[q], s1[q]))) : 0.0;
        out[q] = lane_sum(term);
    }
}

// Identification.hpp:373-384, with val = +1 (white: even ratio count) or -1
// and the division by 2 var done as a product with rvar2 = 1 / double(2 var).
__device__ __forceinline__ float dis_r(float sig, bool white, float mub, float muw, double rvar2)
{
    const float d = white ? fminf(__fsub_rn(sig, muw), 0.f) : fmaxf(__fsub_rn(sig, mub), 0.f);
    return float(double(__fmul_rn(d, d)) * rvar2);
}


// ------------------------------------------------------- center derivatives --
// A value with its derivatives along the two imaged-center coordinates
// (forward mode), for the homography of a trial center.
struct D2 {
    float v, a, b;
};
__device__ __forceinline__ D2 d2c(float v) { return D2{v, 0.f, 0.f}; }
__device__ __forceinline__ D2 operator+(D2 p, D2 q) { return D2{p.v + q.v, p.a + q.a, p.b + q.b}; }
__device__ __forceinline__ D2 operator*(D2 p, float s) { return D2{p.v * s, p.a * s, p.b * s}; }
__device__ __forceinline__ D2 operator+(D2 p, float s) { return D2{p.v + s, p.a, p.b}; }
__device__ __forceinline__ D2 operator*(D2 p, D2 q) { return D2{p.v * q.v, p.a * q.v + p.v * q.a, p.b * q.v + p.v * q.b}; }
__device__ __forceinline__ D2 operator/(D2 p, D2 q)
{
    const float r = p.v / q.v;
    return D2{r, (p.a - r * q.a) / q.v, (p.b - r * q.b) / q.v};
}
__device__ __forceinline__ D2 dsqrt(D2 p)
{
    const float r = sqrtf(p.v);
    const float h = 0.5f / r;
    return D2{r, p.a * h, p.b * h};
}

// homography_from_center and its derivatives with respect to (x, y).
__device__ void homography_center_derivs(const float* C, const float* Tp, const float* Td, float x, float y,
                                         float* H, float* dHx, float* dHy)
{
    const D2 X{x, 1.f, 0.f}, Y{y, 0.f, 1.f};
    const D2 u = X * Tp[0] + Y * Tp[1] + Tp[2];
    const D2 v = X * Tp[3] + Y * Tp[4] + Tp[5];
    const D2 w = X * Tp[6] + Y * Tp[7] + Tp[8];
    const D2 xc = u / w, yc = v / w;
    const float Q11 = C[0], Q22 = C[4], Q33 = C[8];
    D2 h[9];
    h[0] = d2c(Q33);        h[1] = xc * yc * Q22;          h[2] = xc * (-Q33);
    h[3] = d2c(0.f);        h[4] = xc * xc * (-Q11) + (-Q33); h[5] = yc * (-Q33);
    h[6] = xc * (-Q11);     h[7] = yc * Q22;               h[8] = d2c(-Q33);
    const D2 e0 = dsqrt((xc * xc * Q11 + yc * yc * Q22 + Q33) * (Q22 * Q33 / Q11));
    const D2 e2 = dsqrt((xc * xc * Q11 + Q33) * (-Q22));
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        h[i * 3 + 0] = h[i * 3 + 0] * e0;
        h[i * 3 + 1] = h[i * 3 + 1] * Q33;
        h[i * 3 + 2] = h[i * 3 + 2] * e2;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const D2 r = h[j] * Td[i * 3] + h[3 + j] * Td[i * 3 + 1] + h[6 + j] * Td[i * 3 + 2];
            H[i * 3 + j] = r.v;
            dHx[i * 3 + j] = r.a;
            dHy[i * 3 + j] = r.b;
        }
}

// Back-projected end of a cut (stop point through Hi, normalised) and its
// derivatives along the center, given dHi for both center coordinates.
__device__ __forceinline__ void back_project(const float* Hi, const float* dHi0, const float* dHi1, float px, float py,
                                             float& bx, float& by, float db[2][2])
{
    const float z0 = Hi[0] * px + Hi[1] * py + Hi[2];
    const float z1 = Hi[3] * px + Hi[4] * py + Hi[5];
    const float z2 = Hi[6] * px + Hi[7] * py + Hi[8];
    bx = z0 / z2;
    by = z1 / z2;
    const float* d[2] = {dHi0, dHi1};
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const float e0 = d[q][0] * px + d[q][1] * py + d[q][2];
        const float e1 = d[q][3] * px + d[q][4] * py + d[q][5];
        const float e2 = d[q][6] * px + d[q][7] * py + d[q][8];
        db[q][0] = (e0 - bx * e2) / z2;
        db[q][1] = (e1 - by * e2) / z2;
    }
}

// dHi = -Hi dH Hi
__device__ __forceinline__ void inverse_derivative(const float* Hi, const float* dH, float* dHi)
{
    float t[9];
    mat_mul(dH, Hi, t);
    mat_mul(Hi, t, dHi);
#pragma unroll
    for (int k = 0; k < 9; ++k) dHi[k] = -dHi[k];
}

// Sample k of a cut for Gauss-Newton at the trial homography S.gH: its value
// and, in ds, its derivatives along the two center coordinates (through H, and
// through the back-projected cut end (bx, by) whose derivatives are db).
__device__ __forceinline__ float gn_sample(const Shared& S, const Roi& roi, float bs, float den, float bx, float by,
                                          const float db[2][2], int k, float ds[2])
{
    const float xs = bx * bs, ys = by * bs;
    const float sx = (bx - xs) / den, sy = (by - ys) / den;
    const float kf = float(k);
    const float x = __fmaf_rn(kf, sx, xs), y = __fmaf_rn(kf, sy, ys);
    const float t = bs + kf * (1.f - bs) / den;
    const float* Hm = S.gH;
    const float u = hrow(Hm, 0, x, y), v = hrow(Hm, 1, x, y), w = hrow(Hm, 2, x, y);
    const float r = __frcp_rn(w);
    const float qx = __fmul_rn(u, r), qy = __fmul_rn(v, r);
    float gx, gy;
    const float val = bilinear_grad(roi, qx, qy, gx, gy);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const float* dH = S.gdH[q];
        const float dxq = __fmul_rn(t, db[q][0]), dyq = __fmul_rn(t, db[q][1]);
        const float du = __fmaf_rn(Hm[0], dxq, __fmaf_rn(Hm[1], dyq, hrow(dH, 0, x, y)));
        const float dv = __fmaf_rn(Hm[3], dxq, __fmaf_rn(Hm[4], dyq, hrow(dH, 1, x, y)));
        const float dw = __fmaf_rn(Hm[6], dxq, __fmaf_rn(Hm[7], dyq, hrow(dH, 2, x, y)));
        const float ex = __fmul_rn(__fmaf_rn(-qx, dw, du), r);
        const float ey = __fmul_rn(__fmaf_rn(-qy, dw, dv), r);
        ds[q] = __fmaf_rn(gx, ex, __fmul_rn(gy, ey));
    }
    return val;
}

// The Gauss-Newton sums of one chunk (lane = sample): cost, J^T r and J^T J
// of the residuals s_ik - mean_k, from per-lane shifted FP32 sums over the
// valid cuts in cut order, then FP64 over the lanes.  at(c, v, a, b) reads
// sample value v and its center derivatives a, b of cut c.
template <class At>
__device__ __forceinline__ void gn_chunk_sums(uint32_t valid, int n, bool live, double acc[6], At at)
{
#pragma unroll
    for (int q = 0; q < 6; ++q) acc[q] = 0.0;
    if (live && n >= 2) {
        float v0 = 0.f, s1 = 0.f, s2 = 0.f, a1 = 0.f, b1 = 0.f, aa = 0.f, ab = 0.f, bb = 0.f, ad = 0.f, bd = 0.f;
        bool first = true;
        uint32_t m = valid;
        while (m) {
            const int c = __ffs(m) - 1;
            m &= m - 1;
            float v, a, b;
            at(c, v, a, b);
            if (first) {
                v0 = v;
                first = false;
            }
            const float d = __fsub_rn(v, v0);
            s1 = __fadd_rn(s1, d);
            s2 = __fmaf_rn(d, d, s2);
            a1 = __fadd_rn(a1, a);
            b1 = __fadd_rn(b1, b);
            aa = __fmaf_rn(a, a, aa);
            ab = __fmaf_rn(a, b, ab);
            bb = __fmaf_rn(b, b, bb);
            ad = __fmaf_rn(a, d, ad);
            bd = __fmaf_rn(b, d, bd);
        }
        const float fn = float(n);
        acc[0] = double(__fsub_rn(__fmul_rn(fn, s2), __fmul_rn(s1, s1)));
        acc[1] = double(__fsub_rn(ad, __fdiv_rn(__fmul_rn(a1, s1), fn)));
        acc[2] = double(__fsub_rn(bd, __fdiv_rn(__fmul_rn(b1, s1), fn)));
        acc[3] = double(__fsub_rn(aa, __fdiv_rn(__fmul_rn(a1, a1), fn)));
        acc[4] = double(__fsub_rn(ab, __fdiv_rn(__fmul_rn(a1, b1), fn)));
        acc[5] = double(__fsub_rn(bb, __fdiv_rn(__fmul_rn(b1, b1), fn)));
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) acc[q] = lane_sum(acc[q]);
}

// Levenberg-Marquardt on the cut-consistency cost (CCTAGB_REFINE_GAUSS_NEWTON):
// residuals r_ik = s_ik - mean_k over the valid cuts i and samples k, whose
// sum of squares is the reference's pair cost up to the factor n / pairs;
// Jacobian d r_ik / d center from the forward derivatives of the trial
// homography, its inverse (which moves the back-projected cut ends) and the
// bilinear patch.  Each block of the cluster sums its samples; the sums meet
// through distributed shared memory and every block takes the same step.
// Starts from the grid's center; a step that raises the cost is rejected and
// the damping raised.  Stops when a step is below 1e-3 px, or after
// gnIterations cost evaluations.
template <int CL>
__device__ void gn_refine(Shared& S, const IdentTask& T, const Roi& roi, const IdentParams& ip, uint32_t cutMask,
                          int crank)
{
    namespace cg = cooperative_groups;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nS = ip.nSamples;
    const int nch = (nS + kChunk - 1) / kChunk;
    const float bs = ip.beginSig;
    const float den = float(nS) - 1.f;
    // chunks of this block: all of them, or chunk `crank` in a cluster
    const int j0 = CL == 1 ? 0 : crank;
    const int j1 = CL == 1 ? nch : min(crank + 1, nch);
    if (tid == 0) {
        S.gTry[0] = S.cx;
        S.gTry[1] = S.cy;
        S.gHave = 0;
        S.gStop = 0;
        S.gLambda = 1e-3;
    }
    __syncthreads();
    for (int it = 0; it < ip.gnIterations; ++it) {
        if (tid == 0) {
            homography_center_derivs(S.C, S.Tp, S.Td, S.gTry[0], S.gTry[1], S.gH, S.gdH[0], S.gdH[1]);
            if (!mat_inv(S.gH, S.gHi)) {
                S.gStop = 1;
            } else {
                inverse_derivative(S.gHi, S.gdH[0], S.gdHi[0]);
                inverse_derivative(S.gHi, S.gdH[1], S.gdHi[1]);
            }
        }
        __syncthreads();
        if (S.gStop) break;
        // cuts whose end samples leave the rectangle at this center
        if (warp == 0) {
            bool bad = false;
            if (lane < T.ncuts) {
                float bx, by, w;
                apply_h(S.gHi, T.stop[lane][0], T.stop[lane][1], bx, by, w);
                const float xs = bx * bs, ys = by * bs;
                const float sx = (bx - xs) / den, sy = (by - ys) / den;
                float x0, y0, w0, x1, y1, w1;
                apply_h(S.gH, xs, ys, x0, y0, w0);
                apply_h(S.gH, xs + den * sx, ys + den * sy, x1, y1, w1);
                bad = !(w0 > 0.f && w1 > 0.f) && !(w0 < 0.f && w1 < 0.f);
                bad = bad || !inside(roi, x0, y0) || !inside(roi, x1, y1);
            }
            const uint32_t m = __ballot_sync(0xffffffffu, bad);
            if (lane == 0) S.gOob = m & cutMask;
        }
        __syncthreads();
        const uint32_t valid = ~(S.oob | S.gOob) & cutMask;
        const int n = __popc(valid);
        const int par = it & 1;
        // One block doing every chunk, with room for all samples: each warp
        // computes its cuts' samples of every chunk (the back-projected end
        // once per cut), then warp j sums chunk j.  The per-chunk sums are
        // the same operations in the same order as the chunk-at-a-time path,
        // so both give the same bits.
        const bool whole = CL == 1 && 2 * T.ncuts * nS <= int(sizeof(S.u) / sizeof(float));
        if (whole) {
            float* gdx = reinterpret_cast<float*>(&S.u);
            float* gdy = gdx + T.ncuts * nS;
            for (int c = warp; c < T.ncuts; c += kWarps) {
                if (!((valid >> c) & 1u)) continue;
                float bx, by, db[2][2];
                back_project(S.gHi, S.gdHi[0], S.gdHi[1], T.stop[c][0], T.stop[c][1], bx, by, db);
                for (int k = lane; k < nS; k += kChunk) {
                    float ds[2];
                    S.sig[c][k] = gn_sample(S, roi, bs, den, bx, by, db, k, ds);
                    gdx[c * nS + k] = ds[0];
                    gdy[c * nS + k] = ds[1];
                }
            }
            __syncthreads();
            if (warp < nch) {
                const int k = warp * kChunk + lane;
                double acc[6];
                gn_chunk_sums(valid, n, k < nS, acc, [&](int c, float& v, float& a, float& b) {
                    v = S.sig[c][k];
                    a = gdx[c * nS + k];
                    b = gdy[c * nS + k];
                });
                if (lane == 0)
#pragma unroll
                    for (int q = 0; q < 6; ++q) S.gPart[par][warp][q] = acc[q];
            }
            __syncthreads();
        } else {
            for (int j = j0; j < j1; ++j) {
                // this chunk's samples: value and its derivatives along the center
                const int k = j * kChunk + lane;
                for (int c = warp; c < T.ncuts; c += kWarps) {
                    if (!((valid >> c) & 1u) || k >= nS) continue;
                    float bx, by, db[2][2];
                    back_project(S.gHi, S.gdHi[0], S.gdHi[1], T.stop[c][0], T.stop[c][1], bx, by, db);
                    float ds[2];
                    S.u.gn.s[c][lane] = gn_sample(S, roi, bs, den, bx, by, db, k, ds);
                    S.u.gn.dx[c][lane] = ds[0];
                    S.u.gn.dy[c][lane] = ds[1];
                }
                __syncthreads();
                if (warp == 0) {
                    double acc[6];
                    gn_chunk_sums(valid, n, k < nS, acc, [&](int c, float& v, float& a, float& b) {
                        v = S.u.gn.s[c][lane];
                        a = S.u.gn.dx[c][lane];
                        b = S.u.gn.dy[c][lane];
                    });
                    if (lane == 0)
#pragma unroll
                        for (int q = 0; q < 6; ++q) S.gPart[par][j][q] = acc[q];
                }
                __syncthreads();
            }
        }
        // every chunk's sums are in; a parity's array is rewritten two
        // evaluations later, past the next barrier of the cluster
        if constexpr (CL > 1) cg::this_cluster().sync();
        if (warp == 0 && lane < 6) {
            double a = 0.0;
            for (int j = 0; j < nch; ++j) {
                const double* src = &S.gPart[par][j][0];
                if constexpr (CL > 1) src = cg::this_cluster().map_shared_rank(src, j);
                a += src[lane];
            }
            S.gSum[lane] = a;
        }
        __syncthreads();
        if (tid == 0) {
            const double cost = n >= 2 ? S.gSum[0] / (0.5 * double(n) * double(n - 1)) : DBL_MAX;
            ++S.iterations;
            if (n >= 2 && (!S.gHave || cost < S.gBest)) {
                S.gHave = 1;
                S.gBest = cost;
                S.cx = S.gTry[0];
                S.cy = S.gTry[1];
                S.oob |= S.gOob;
                for (int q = 0; q < 9; ++q) S.Hopt[q] = S.gH[q];
                S.minRes = float(cost);
                S.gG[0] = S.gSum[1];
                S.gG[1] = S.gSum[2];
                S.gA[0] = S.gSum[3];
                S.gA[1] = S.gSum[4];
                S.gA[2] = S.gSum[5];
                S.gLambda = fmax(S.gLambda * 0.1, 1e-7);
            } else {
                S.gLambda *= 10.0;
            }
            if (!S.gHave) {
                S.gStop = 1;
            } else {
                const double a = S.gA[0] * (1.0 + S.gLambda), b = S.gA[1], c = S.gA[2] * (1.0 + S.gLambda);
                const double det = a * c - b * b;
                if (!(det > 0.0)) {
                    S.gStop = 1;
                } else {
                    const double dx = -(c * S.gG[0] - b * S.gG[1]) / det;
                    const double dy = -(a * S.gG[1] - b * S.gG[0]) / det;
                    if (dx * dx + dy * dy < 1e-6) S.gStop = 1;
                    S.gTry[0] = float(double(S.cx) + dx);
                    S.gTry[1] = float(double(S.cy) + dy);
                }
            }
        }
        __syncthreads();
        if (S.gStop) break;
    }
}

}  // namespace

// CL = 1: one block per marker; CL = kCluster: a cluster of blocks per marker
// (launched with that cluster dimension), block r on sample chunk r.  MB:
// blocks per SM the registers are budgeted for (2 suits Gauss-Newton, whose
// steps leave most warps waiting; the grid keeps every warp busy and prefers
// the registers).  The register caps follow from the 25 warps of a block
// spread over the SM's four 16 K-register partitions (7 warps on one): 72 for
// one block per SM, 32 for two; 64 for the cluster form (the detection's),
// which needs no spill at 64 and so leaves room in every partition for a
// block of another stream's kernel.
template <int CL, int MB>
__global__ void __maxnreg__(CL > 1 ? 64 : (MB == 1 ? 72 : 32))
    k_identify(const uint8_t* __restrict__ img, size_t pitch, const IdentTask* __restrict__ tasks, IdentResult* res,
               const float* __restrict__ bankInv, IdentParams ip)
{
    namespace cg = cooperative_groups;
    __shared__ Shared S;
    int crank = 0;
    if constexpr (CL > 1) crank = int(cg::this_cluster().block_rank());
    const int marker = blockIdx.x / CL;
    const IdentTask& T = tasks[marker];
    const Roi roi = make_roi(img, pitch, T);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nS = ip.nSamples;
    const int nch = (nS + kChunk - 1) / kChunk;
    // chunks this block evaluates (all, or chunk `crank` in a cluster), NCH
    // per pass (fewer live registers when two blocks share an SM)
    constexpr int NCH = CL == 1 ? (MB == 1 ? kMaxChunks : kMaxChunks / 2) : 1;
    const int j0 = CL == 1 ? 0 : crank;
    const int jEnd = CL == 1 ? nch : j0 + 1;
    const int gridN = ip.gridN;
    const int nTrials = gridN * gridN;
    const uint32_t cutMask = (T.ncuts >= 32) ? 0xffffffffu : ((1u << T.ncuts) - 1u);
    if (T.ncuts <= 0) {  // nothing to refine or read (identify_step_1 stopped it)
        if (tid == 0 && crank == 0) {
            IdentResult& R0 = res[marker];
            R0 = IdentResult{};
            R0.x = T.x0;
            R0.y = T.y0;
            R0.id = -1;
            R0.status = CCTAGB_NO_SELECTED_CUTS;
        }
        return;
    }

    if (tid == 0) {
        canonic_form(T.Q, S.C, S.Tp, S.Td);
        // conditionerFromEllipse (conditioner.hpp:22-44) with meanAB of this ellipse
        const float sqrt2 = sqrtf(2.f);
        const float meanAB = (T.a + T.b) / 2.f;
        float mT[9] = {sqrt2 / meanAB, 0.f, -sqrt2 * T.cx / meanAB, 0.f, sqrt2 / meanAB, -sqrt2 * T.cy / meanAB,
                       0.f, 0.f, 1.f};
        float mTi[9];
        mat_inv(mT, mTi);
        float tq[9], Qc[9], mTiT[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) mTiT[i * 3 + j] = mTi[j * 3 + i];
        mat_mul(T.Q, mTi, tq);
        mat_mul(mTiT, tq, Qc);
        float ca, cb;
        conic_axes(Qc, ca, cb);
        S.nsScale = fmaxf(ca, cb);
        for (int k = 0; k < 9; ++k) {
            S.mT[k] = mT[k];
            S.mTi[k] = mTi[k];
        }
        S.cx = T.x0;
        S.cy = T.y0;
        S.minRes = FLT_MAX;
        S.oob = 0u;
        S.fail = 0;
        // refineConicFamilyGlob loop bound (Identification.cpp:869-885)
        const float maxSemiAxis = fmaxf(T.a, T.b);
        float ns = ip.neighbourSize;
        int r = 0;
        while (ns * maxSemiAxis > 0.02f && r < 64) {
            ++r;
            ns /= float((gridN - 1) / 2);
        }
        if (ip.refineMode == CCTAGB_REFINE_GAUSS_NEWTON) r = min(r, ip.coarseRounds);
        S.rounds = r;
        S.iterations = r;
    }
    __syncthreads();
    float ns = ip.neighbourSize;
    for (int round = 0; round < S.rounds; ++round) {
        // getNearbyPoints (Identification.cpp:1071-1109)
        if (warp < nTrials) {
            const float size = ns * S.nsScale;
            const float half = size / 2.f, step = size / float(gridN - 1);
            const float ccx = S.mT[0] * S.cx + S.mT[1] * S.cy + S.mT[2];
            const float ccy = S.mT[3] * S.cx + S.mT[4] * S.cy + S.mT[5];
            const int i = warp / gridN, j = warp % gridN;
            const float qx = ccx - half + float(i) * step, qy = ccy - half + float(j) * step;
            float px, py, w;
            apply_h(S.mTi, qx, qy, px, py, w);
            setup_trial(S, T, warp, px, py, ip, roi, lane);
        }
        __syncthreads();
        // sticky out-of-bounds flags in trial order: inclusive OR scan
        if (warp == 0) {
            uint32_t m = lane < nTrials ? S.trialOob[lane] : 0u;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t v = __shfl_up_sync(0xffffffffu, m, o);
                if (lane >= o) m |= v;
            }
            m |= S.oob;
            if (lane < nTrials) S.valid[lane] = ~m & cutMask;
            const uint32_t last = __shfl_sync(0xffffffffu, m, nTrials - 1);
            __syncwarp();
            if (lane == 0) S.oob = last;
        }
        __syncthreads();
        const int par = round & 1;
        if (warp < nTrials) {
            for (int jp = j0; jp < jEnd; jp += NCH) {
                double c[NCH];
                trial_partial<NCH>(S, roi, warp, S.valid[warp], jp, nch, nS, lane, c);
                if (lane == 0)
#pragma unroll
                    for (int q = 0; q < NCH; ++q)
                        if (jp + q < nch) S.part[par][jp + q][warp] = c[q];
            }
        }
        // All chunks of the marker are in; a block rewrites this parity's
        // array two rounds later, after the next cluster barrier, when every
        // block has finished reading it.
        if constexpr (CL > 1) cg::this_cluster().sync();
        else __syncthreads();
        if (warp == 0) {
            double acc = 0.0;
            if (lane < nTrials)
                for (int j = 0; j < nch; ++j) {
                    const double* src = &S.part[par][j][0];
                    if constexpr (CL > 1) src = cg::this_cluster().map_shared_rank(src, j);
                    acc += src[lane];
                }
            const int n = lane < nTrials ? __popc(S.valid[lane]) : 0;
            const float cost = n >= 2 ? float(acc / (0.5 * double(n) * double(n - 1))) : FLT_MAX;
            if (lane < nTrials) S.cost[lane] = cost;
            // imageCenterOptimizationGlob: first strict minimum in trial order
            // (costs below FLT_MAX; key = orderable cost bits, then index)
            unsigned long long key = ~0ull;
            if (lane < nTrials && cost < FLT_MAX) {
                const uint32_t b = __float_as_uint(cost);
                const uint32_t ord = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
                key = (static_cast<unsigned long long>(ord) << 32) | unsigned(lane);
            }
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                const unsigned long long k2 = __shfl_xor_sync(0xffffffffu, key, o);
                key = k2 < key ? k2 : key;
            }
            const bool readable = __any_sync(0xffffffffu, n >= 2);
            __syncwarp();
            if (lane == 0) {
                if (!readable || key == ~0ull) {
                    S.fail = 1;
                } else {
                    const int bi = int(key & 0xffffffffull);
                    S.cx = S.trialPt[bi][0];
                    S.cy = S.trialPt[bi][1];
                    for (int k = 0; k < 9; ++k) S.Hopt[k] = S.trialH[bi][k];
                    S.minRes = S.cost[bi];
                }
            }
        }
        __syncthreads();
        if (S.fail) break;
        ns /= float((gridN - 1) / 2);
    }
    if (ip.refineMode == CCTAGB_REFINE_GAUSS_NEWTON && !S.fail && S.rounds > 0)
        gn_refine<CL>(S, T, roi, ip, cutMask, crank);
    // No block leaves while another may still read its shared memory; the
    // rest of the identification runs in the first block of the cluster.
    if constexpr (CL > 1) {
        cg::this_cluster().sync();
        if (crank != 0) return;
    }
    IdentResult& R = res[marker];
    if (S.fail || S.rounds == 0) {
        if (tid == 0) {
            R.status = CCTAGB_OPTI_HAS_DIVERGED;
            R.id = -1;
            R.x = S.cx;
            R.y = S.cy;
            for (int k = 0; k < 9; ++k) R.H[k] = 0.f;
            R.residual = FLT_MAX;
            R.score = 0.f;
            R.nvalid = 0;
            R.iterations = S.iterations;
        }
        return;
    }
    // Final signals with the optimal homography (getSignals, Identification.cpp:901).
    for (int c = warp; c < T.ncuts; c += kWarps) {
        float Hi[9];
        mat_inv(S.Hopt, Hi);
        float bx, by, w;
        apply_h(Hi, T.stop[c][0], T.stop[c][1], bx, by, w);
        const float xs = bx * ip.beginSig, ys = by * ip.beginSig;
        const float sx = (bx - xs) / (float(nS) - 1.f), sy = (by - ys) / (float(nS) - 1.f);
        bool bad = false;
        for (int k = lane; k < nS; k += 32) {
            const float x = xs + float(k) * sx, y = ys + float(k) * sy;
            float xr, yr;
            apply_h(S.Hopt, x, y, xr, yr, w);
            if (inside(roi, xr, yr)) S.sig[c][k] = bilinear(roi, xr, yr);
            else bad = true;
        }
        const uint32_t any = __ballot_sync(0xffffffffu, bad);
        if (lane == 0 && any) atomicOr(&S.oob, 1u << c);
    }
    __syncthreads();
    const uint32_t valid = ~S.oob & cutMask;
    const int nValid = __popc(valid);
    // Median barcode over the valid cuts (computeMedian, Identification.hpp:351-371).
    if (tid < nS) {
        float v[kMaxCuts];
        int n = 0;
        uint32_t m = valid;
        while (m) {
            const int c = __ffs(m) - 1;
            m &= m - 1;
            const float x = S.sig[c][tid];
            int j = n++;
            while (j > 0 && v[j - 1] > x) {
                v[j] = v[j - 1];
                --j;
            }
            v[j] = x;
        }
        float med = 0.f;
        if (n > 0) med = (n & 1) ? v[n / 2] : float((double(v[n / 2]) + double(v[n / 2 - 1])) / 2.0);
        S.barcode[tid] = med;
    }
    __syncthreads();
    // Orazio distance per valid cut: lane = bank id (Identification.cpp:77-190).
    for (int c = warp; c < T.ncuts; c += kWarps) {
        if (!((valid >> c) & 1u)) continue;
        const float* sg = S.sig[c];
        // statistics over samples [30, n): Boost immediate mean / variance
        // (the divisions by the counts correctly rounded by div_small)
        float mean = 0.f, var = 0.f;
        {
            int cnt = 0;
            float rprev = 1.f;
            for (int k = 30; k < nS; ++k) {
                ++cnt;
                const float x = sg[k];
                const float fc = float(cnt), fc1 = float(cnt - 1), rc = __frcp_rn(fc);
                mean = pm::div_small(__fmaf_rn(mean, fc1, x), fc, rc);
                if (cnt > 1) {
                    const float t = __fsub_rn(x, mean);
                    var = __fadd_rn(pm::div_small(__fmul_rn(var, fc1), fc, rc),
                                    pm::div_small(__fmul_rn(t, t), fc1, rprev));
                }
                rprev = rc;
            }
        }
        float mub = 0.f, muw = 0.f;
        {
            int ni = 0, nsup = 0;
            bool acc = false;
            for (int k = 0; k < nS; ++k) {
                const float x = sg[k];
                if (!acc && x < mean) acc = true;
                if (acc) {
                    if (x < mean) {
                        ++ni;
                        mub = pm::div_small(__fmaf_rn(mub, float(ni - 1), x), float(ni), __frcp_rn(float(ni)));
                    } else {
                        ++nsup;
                        muw = pm::div_small(__fmaf_rn(muw, float(nsup - 1), x), float(nsup),
                                            __frcp_rn(float(nsup)));
                    }
                }
            }
        }
        // dis()'s division by 2 var: a float quotient through the double
        // reciprocal is correctly rounded for a normal result (its relative
        // error, 2^-52, is below the 2^-49 that separates a quotient of floats
        // from a float rounding midpoint), so each term is the IEEE quotient.
        const double rvar2 = 1.0 / double(2.0f * var);
        const float stepX = (1.f - ip.beginSig) / (float(nS) - 1.f);
        // std::map<float, id> keeps, for equal keys, the id inserted last: the
        // winner is the largest v, ties to the largest id.  v >= 0, so its bit
        // pattern orders like the value; (bits << 32 | id) orders like the map.
        unsigned long long best = 0ull;
        for (int base = 0; base < ip.nIds; base += 32) {
            const int idc = base + lane;
            unsigned long long key = 0ull;
            if (idc < ip.nIds) {
                // this lane's bank row (1 / ratio), padded with +inf
                float inv[kMaxBankRatios];
#pragma unroll
                for (int r = 0; r < kMaxBankRatios; ++r)
                    inv[r] = r < ip.nRatios ? __ldg(&bankInv[idc * kMaxBankRatios + r]) : FLT_MAX;
                float x = ip.beginSig, dist = 0.f;
#pragma unroll 4
                for (int k = 0; k < nS; ++k) {
                    int ldum = 0;
#pragma unroll
                    for (int r = 0; r < kMaxBankRatios; ++r) ldum += (inv[r] <= x) ? 1 : 0;
                    dist += dis_r(sg[k], (ldum & 1) == 0, mub, muw, rvar2);
                    x += stepX;
                }
                const float v = expf(-dist);
                key = (static_cast<unsigned long long>(__float_as_uint(v)) << 32) | unsigned(idc);
            }
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                const unsigned long long ok = __shfl_xor_sync(0xffffffffu, key, o);
                key = ok > key ? ok : key;
            }
            best = key > best ? key : best;
        }
        const int bestId = int(best & 0xffffffffull);
        const float bestV = __uint_as_float(unsigned(best >> 32));
        if (lane == 0) {
            S.winner[c] = bestId;
            S.vwin[c] = bestV;
        }
    }
    __syncthreads();
    if (tid == 0) {
        // ID vote (Identification.cpp:1408-1431): most-voted id (first on ties),
        // score = mean probability of its votes.
        int counts[kMaxBankIds];
        for (int i = 0; i < ip.nIds; ++i) counts[i] = 0;
        for (int c = 0; c < T.ncuts; ++c)
            if ((valid >> c) & 1u) counts[S.winner[c]]++;
        int iMax = 0, maxSize = 0;
        for (int i = 0; i < ip.nIds; ++i)
            if (counts[i] > maxSize) {
                iMax = i;
                maxSize = counts[i];
            }
        float score = 0.f;
        for (int c = 0; c < T.ncuts; ++c)
            if (((valid >> c) & 1u) && S.winner[c] == iMax) score += S.vwin[c];
        score /= float(maxSize);
        float vmin = FLT_MAX, vmax = -FLT_MAX;
        for (int k = 0; k < nS; ++k) {
            vmin = fminf(vmin, S.barcode[k]);
            vmax = fmaxf(vmax, S.barcode[k]);
        }
        const float residual = sqrtf(S.minRes) / (vmax - vmin);
        R.x = S.cx;
        R.y = S.cy;
        for (int k = 0; k < 9; ++k) R.H[k] = S.Hopt[k];
        R.residual = residual;
        R.nvalid = nValid;
        R.iterations = S.iterations;
        if (residual > 2.7f || !(residual == residual)) {
            R.status = CCTAGB_OPTI_HAS_DIVERGED;
            R.id = -1;
            R.score = 0.f;
        } else {
            R.id = iMax;
            R.score = score;
            R.status = score > ip.minIdentProba ? CCTAGB_ID_RELIABLE : CCTAGB_ID_NOT_RELIABLE;
        }
    }
}


namespace {

struct CostShared {
    float C[9], Tp[9], Td[9];
    float H[9], Hi[9], dH[2][9];
    float sig[kMaxCuts][kMaxSamples];
    float mean[kMaxSamples];
    float dz[kMaxCuts][3];        // d cost / d (Hi p) of each cut's back-projected end
    double red[kThreads / 32][10];
    uint32_t oob;
    int bad;
};

__device__ void write_cost(float* o, float cost)
{
    o[0] = cost;
    for (int j = 1; j < 12; ++j) o[j] = 0.f;
}

}  // namespace

// Cut-consistency cost of one task at a given center and its adjoints (one
// block per task).  Pass 1 reads every sample (a sample outside the
// rectangle drops its cut, as extractSignalUsingHomography does); pass 2
// sends d cost / d s_ik = 2 n / pairs (s_ik - mean_k) back through the
// bilinear patch to the image position, from there to H directly and to the
// sample's marker-plane position, whose cut end is H^-1 applied to the stop
// point; the inverse's adjoint is -H^-T G H^-T.  The center gradient is the
// H gradient contracted with dH/dcenter (forward derivatives).
__global__ void __launch_bounds__(kThreads) k_cut_cost(const uint8_t* __restrict__ img, size_t pitch,
                                                       const IdentTask* __restrict__ tasks,
                                                       const float* __restrict__ centers, float* out, IdentParams ip)
{
    __shared__ CostShared S;
    const IdentTask& T = tasks[blockIdx.x];
    const Roi roi = make_roi(img, pitch, T);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nS = ip.nSamples;
    const float bs = ip.beginSig;
    const float den = float(nS) - 1.f;
    float* o = out + 12 * size_t(blockIdx.x);
    const uint32_t cutMask = (T.ncuts >= 32) ? 0xffffffffu : ((1u << T.ncuts) - 1u);
    if (tid == 0) {
        canonic_form(T.Q, S.C, S.Tp, S.Td);
        homography_center_derivs(S.C, S.Tp, S.Td, centers[2 * blockIdx.x], centers[2 * blockIdx.x + 1], S.H,
                                 S.dH[0], S.dH[1]);
        S.bad = mat_inv(S.H, S.Hi) ? 0 : 1;
        S.oob = 0u;
    }
    if (tid < kMaxCuts * 3) S.dz[tid / 3][tid % 3] = 0.f;
    __syncthreads();
    if (S.bad) {
        if (tid == 0) write_cost(o, FLT_MAX);
        return;
    }
    for (int c = warp; c < T.ncuts; c += kWarps) {
        float bx, by, w;
        apply_h(S.Hi, T.stop[c][0], T.stop[c][1], bx, by, w);
        const float xs = bx * bs, ys = by * bs;
        const float sx = (bx - xs) / den, sy = (by - ys) / den;
        bool bad = false;
        for (int k = lane; k < nS; k += 32) {
            const float x = xs + float(k) * sx, y = ys + float(k) * sy;
            float xr, yr;
            apply_h(S.H, x, y, xr, yr, w);
            if (inside(roi, xr, yr)) S.sig[c][k] = bilinear(roi, xr, yr);
            else bad = true;
        }
        if (__ballot_sync(0xffffffffu, bad) && lane == 0) atomicOr(&S.oob, 1u << c);
    }
    __syncthreads();
    const uint32_t valid = ~S.oob & cutMask;
    const int n = __popc(valid);
    if (n < 2) {
        if (tid == 0) write_cost(o, FLT_MAX);
        return;
    }
    const double pairs = 0.5 * double(n) * double(n - 1);
    double costPart = 0.0;
    for (int k = tid; k < nS; k += kThreads) {
        double s1 = 0.0, s2 = 0.0;
        uint32_t m = valid;
        while (m) {
            const int c = __ffs(m) - 1;
            m &= m - 1;
            const double v = S.sig[c][k];
            s1 += v;
            s2 += v * v;
        }
        S.mean[k] = float(s1 / double(n));
        costPart += double(n) * s2 - s1 * s1;
    }
    __syncthreads();
    float gH[9];
#pragma unroll
    for (int j = 0; j < 9; ++j) gH[j] = 0.f;
    const float coef = float(2.0 * double(n) / pairs);
    const float* Hm = S.H;
    for (int c = warp; c < T.ncuts; c += kWarps) {
        if (!((valid >> c) & 1u)) continue;
        const float px = T.stop[c][0], py = T.stop[c][1];
        const float z0 = S.Hi[0] * px + S.Hi[1] * py + S.Hi[2];
        const float z1 = S.Hi[3] * px + S.Hi[4] * py + S.Hi[5];
        const float z2 = S.Hi[6] * px + S.Hi[7] * py + S.Hi[8];
        const float bx = z0 / z2, by = z1 / z2;
        const float xs = bx * bs, ys = by * bs;
        const float sx = (bx - xs) / den, sy = (by - ys) / den;
        float gbx = 0.f, gby = 0.f;
        for (int k = lane; k < nS; k += 32) {
            const float x = xs + float(k) * sx, y = ys + float(k) * sy;
            const float u = Hm[0] * x + Hm[1] * y + Hm[2];
            const float v = Hm[3] * x + Hm[4] * y + Hm[5];
            const float w = Hm[6] * x + Hm[7] * y + Hm[8];
            const float rw = 1.f / w;
            const float qx = u / w, qy = v / w;
            float gx, gy;
            (void)bilinear_grad(roi, qx, qy, gx, gy);
            const float lam = coef * (S.sig[c][k] - S.mean[k]);
            const float fx = lam * gx, fy = lam * gy;
            const float fw = -(fx * qx + fy * qy);
            const float y3[3] = {x, y, 1.f};
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                gH[j] = fmaf(fx * rw, y3[j], gH[j]);
                gH[3 + j] = fmaf(fy * rw, y3[j], gH[3 + j]);
                gH[6 + j] = fmaf(fw * rw, y3[j], gH[6 + j]);
            }
            const float fX = (fx * (Hm[0] - qx * Hm[6]) + fy * (Hm[3] - qy * Hm[6])) * rw;
            const float fY = (fx * (Hm[1] - qx * Hm[7]) + fy * (Hm[4] - qy * Hm[7])) * rw;
            const float t = bs + float(k) * (1.f - bs) / den;
            gbx = fmaf(t, fX, gbx);
            gby = fmaf(t, fY, gby);
        }
#pragma unroll
        for (int off = 16; off; off >>= 1) {
            gbx += __shfl_xor_sync(0xffffffffu, gbx, off);
            gby += __shfl_xor_sync(0xffffffffu, gby, off);
        }
        if (lane == 0) {
            S.dz[c][0] = gbx / z2;
            S.dz[c][1] = gby / z2;
            S.dz[c][2] = -(gbx * bx + gby * by) / z2;
        }
    }
    double red[10];
    red[0] = costPart;
#pragma unroll
    for (int j = 0; j < 9; ++j) red[1 + j] = double(gH[j]);
#pragma unroll
    for (int j = 0; j < 10; ++j) {
#pragma unroll
        for (int off = 16; off; off >>= 1) red[j] += __shfl_xor_sync(0xffffffffu, red[j], off);
    }
    if (lane == 0)
#pragma unroll
        for (int j = 0; j < 10; ++j) S.red[warp][j] = red[j];
    __syncthreads();
    if (tid == 0) {
        double cost = 0.0, G[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int w = 0; w < kWarps; ++w) {
            cost += S.red[w][0];
            for (int j = 0; j < 9; ++j) G[j] += S.red[w][1 + j];
        }
        cost /= pairs;
        // adjoint of Hi from the cut ends, then -Hi^T GHi Hi^T into G
        double GHi[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int c = 0; c < T.ncuts; ++c) {
            const double p3[3] = {T.stop[c][0], T.stop[c][1], 1.0};
            for (int r = 0; r < 3; ++r)
                for (int q = 0; q < 3; ++q) GHi[r * 3 + q] += double(S.dz[c][r]) * p3[q];
        }
        double M[9], Mt[9];
        for (int i = 0; i < 3; ++i)      // M = GHi Hi^T
            for (int j = 0; j < 3; ++j) {
                double a = 0.0;
                for (int q = 0; q < 3; ++q) a += GHi[i * 3 + q] * double(S.Hi[j * 3 + q]);
                M[i * 3 + j] = a;
            }
        for (int i = 0; i < 3; ++i)      // Mt = Hi^T M
            for (int j = 0; j < 3; ++j) {
                double a = 0.0;
                for (int q = 0; q < 3; ++q) a += double(S.Hi[q * 3 + i]) * M[q * 3 + j];
                Mt[i * 3 + j] = a;
            }
        double dc[2] = {0.0, 0.0};
        for (int j = 0; j < 9; ++j) {
            G[j] -= Mt[j];
            dc[0] += G[j] * double(S.dH[0][j]);
            dc[1] += G[j] * double(S.dH[1][j]);
        }
        o[0] = float(cost);
        o[1] = float(dc[0]);
        o[2] = float(dc[1]);
        for (int j = 0; j < 9; ++j) o[3 + j] = float(G[j]);
    }
}

namespace {

// ---------------------------------------------------- FP64 check form --
// The same cost and adjoint as k_cut_cost, every step in double precision:
// the canonic form, the trial homography with its center derivatives, the
// back-projected cut ends, the sample positions and the bilinear reads.  It
// exists to check the adjoint's derivation against central differences at a
// precision the FP32 kernel cannot reach (FP32 sample positions alone move
// the cost by ~1e-4 of itself); the refinement kernels do not use it.
struct D2d {
    double v, a, b;
};
__device__ __forceinline__ D2d operator+(D2d p, D2d q) { return D2d{p.v + q.v, p.a + q.a, p.b + q.b}; }
__device__ __forceinline__ D2d operator-(D2d p, D2d q) { return D2d{p.v - q.v, p.a - q.a, p.b - q.b}; }
__device__ __forceinline__ D2d operator*(D2d p, D2d q)
{
    return D2d{p.v * q.v, p.a * q.v + p.v * q.a, p.b * q.v + p.v * q.b};
}
__device__ __forceinline__ D2d operator/(D2d p, D2d q)
{
    const double r = p.v / q.v;
    return D2d{r, (p.a - r * q.a) / q.v, (p.b - r * q.b) / q.v};
}
__device__ __forceinline__ D2d sqrt_d2(D2d p)
{
    const double r = sqrt(p.v);
    return D2d{r, p.a / (2.0 * r), p.b / (2.0 * r)};
}
__device__ __forceinline__ D2d cst_d2(double v) { return D2d{v, 0.0, 0.0}; }

__device__ void canonic_form_d(const float* Qf, double* C, double* Tp, double* Td)
{
    const double q1 = Qf[0], q2 = Qf[1], q3 = Qf[2], q4 = Qf[4], q5 = Qf[5], q6 = Qf[8];
    const double par1 = q1, par2 = 2 * q2, par3 = q4, par4 = 2 * q3, par5 = 2 * q5;
    const double th = 0.5 * atan2(par2, par1 - par3);
    const double ct = cos(th), st = sin(th);
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
    const double c[9] = {t1, t2, t3, t2, t4, t5, t3, t5, t6};
    const double tp[9] = {ct, st, -ct * uc - st * vc, -st, ct, st * uc - ct * vc, 0, 0, ct * ct + st * st};
    const double td[9] = {ct, -st, uc, st, ct, vc, 0, 0, 1};
    for (int k = 0; k < 9; ++k) {
        C[k] = c[k];
        Tp[k] = tp[k];
        Td[k] = td[k];
    }
}

// homography_from_center in double, with d/d(x, y).
__device__ void homography_center_derivs_d(const double* C, const double* Tp, const double* Td, double x, double y,
                                           double* H, double* dHx, double* dHy)
{
    const D2d X{x, 1.0, 0.0}, Y{y, 0.0, 1.0};
    const D2d u = X * cst_d2(Tp[0]) + Y * cst_d2(Tp[1]) + cst_d2(Tp[2]);
    const D2d v = X * cst_d2(Tp[3]) + Y * cst_d2(Tp[4]) + cst_d2(Tp[5]);
    const D2d w = X * cst_d2(Tp[6]) + Y * cst_d2(Tp[7]) + cst_d2(Tp[8]);
    const D2d xc = u / w, yc = v / w;
    const D2d Q11 = cst_d2(C[0]), Q22 = cst_d2(C[4]), Q33 = cst_d2(C[8]), z = cst_d2(0.0);
    D2d h[9] = {Q33,          Q22 * xc * yc,           z - Q33 * xc,
                z,            z - Q11 * xc * xc - Q33, z - Q33 * yc,
                z - Q11 * xc, Q22 * yc,                z - Q33};
    const D2d d0 = sqrt_d2(Q22 * Q33 / Q11 * (Q11 * xc * xc + Q22 * yc * yc + Q33));
    const D2d d2 = sqrt_d2(z - Q22 * (Q11 * xc * xc + Q33));
    for (int i = 0; i < 3; ++i) {
        h[i * 3 + 0] = h[i * 3 + 0] * d0;
        h[i * 3 + 1] = h[i * 3 + 1] * Q33;
        h[i * 3 + 2] = h[i * 3 + 2] * d2;
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const D2d r = h[j] * cst_d2(Td[i * 3]) + h[3 + j] * cst_d2(Td[i * 3 + 1]) + h[6 + j] * cst_d2(Td[i * 3 + 2]);
            H[i * 3 + j] = r.v;
            dHx[i * 3 + j] = r.a;
            dHy[i * 3 + j] = r.b;
        }
}

__device__ bool mat_inv_d(const double* a, double* r)
{
    const double c00 = a[4] * a[8] - a[5] * a[7];
    const double c01 = a[5] * a[6] - a[3] * a[8];
    const double c02 = a[3] * a[7] - a[4] * a[6];
    const double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
    if (det == 0.0 || !isfinite(det)) return false;
    const double id = 1.0 / det;
    r[0] = c00 * id;
    r[1] = (a[2] * a[7] - a[1] * a[8]) * id;
    r[2] = (a[1] * a[5] - a[2] * a[4]) * id;
    r[3] = c01 * id;
    r[4] = (a[0] * a[8] - a[2] * a[6]) * id;
    r[5] = (a[2] * a[3] - a[0] * a[5]) * id;
    r[6] = c02 * id;
    r[7] = (a[1] * a[6] - a[0] * a[7]) * id;
    r[8] = (a[0] * a[4] - a[1] * a[3]) * id;
    return true;
}

__device__ __forceinline__ bool inside_d(const Roi& R, double x, double y)
{
    return x >= double(R.x0) && x < double(R.x1 - 1) && y >= double(R.y0) && y < double(R.y1 - 1);
}

// Identification.hpp:197-219 and its gradient, in double.
__device__ __forceinline__ double bilinear_d(const Roi& R, double x, double y, double& gx, double& gy)
{
    const int px = int(x), py = int(y);
    const uint8_t* p0 = R.img + px + size_t(py) * R.pitch;
    const double fx = x - double(px), fy = y - double(py);
    const double p1 = __ldg(p0), p2 = __ldg(p0 + 1), p3 = __ldg(p0 + R.pitch), p4 = __ldg(p0 + R.pitch + 1);
    gx = ((p2 - p1) * (1.0 - fy) + (p4 - p3) * fy) * 0.5;
    gy = ((p3 - p1) * (1.0 - fx) + (p4 - p2) * fx) * 0.5;
    return (p1 * (1.0 - fx) * (1.0 - fy) + p2 * fx * (1.0 - fy) + p3 * (1.0 - fx) * fy + p4 * fx * fy) * 0.5;
}

struct CostSharedD {
    double C[9], Tp[9], Td[9];
    double H[9], Hi[9], dH[2][9];
    double sig[kMaxCuts][kMaxSamples];
    double mean[kMaxSamples];
    double dz[kMaxCuts][3];
    double red[kThreads / 32][10];
    uint32_t oob;
    int bad;
};

}  // namespace

// k_cut_cost in double precision (one block per task).
__global__ void __launch_bounds__(kThreads) k_cut_cost_f64(const uint8_t* __restrict__ img, size_t pitch,
                                                           const IdentTask* __restrict__ tasks,
                                                           const float* __restrict__ centers, float* out,
                                                           IdentParams ip)
{
    __shared__ CostSharedD S;
    const IdentTask& T = tasks[blockIdx.x];
    const Roi roi = make_roi(img, pitch, T);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nS = ip.nSamples;
    const double bs = ip.beginSig;
    const double den = double(nS) - 1.0;
    float* o = out + 12 * size_t(blockIdx.x);
    const uint32_t cutMask = (T.ncuts >= 32) ? 0xffffffffu : ((1u << T.ncuts) - 1u);
    if (tid == 0) {
        canonic_form_d(T.Q, S.C, S.Tp, S.Td);
        homography_center_derivs_d(S.C, S.Tp, S.Td, centers[2 * blockIdx.x], centers[2 * blockIdx.x + 1], S.H,
                                   S.dH[0], S.dH[1]);
        S.bad = mat_inv_d(S.H, S.Hi) ? 0 : 1;
        S.oob = 0u;
    }
    if (tid < kMaxCuts * 3) S.dz[tid / 3][tid % 3] = 0.0;
    __syncthreads();
    if (S.bad) {
        if (tid == 0) write_cost(o, FLT_MAX);
        return;
    }
    for (int c = warp; c < T.ncuts; c += kWarps) {
        const double px = T.stop[c][0], py = T.stop[c][1];
        const double z0 = S.Hi[0] * px + S.Hi[1] * py + S.Hi[2];
        const double z1 = S.Hi[3] * px + S.Hi[4] * py + S.Hi[5];
        const double z2 = S.Hi[6] * px + S.Hi[7] * py + S.Hi[8];
        const double bx = z0 / z2, by = z1 / z2;
        const double xs = bx * bs, ys = by * bs;
        const double sx = (bx - xs) / den, sy = (by - ys) / den;
        bool bad = false;
        for (int k = lane; k < nS; k += 32) {
            const double x = xs + double(k) * sx, y = ys + double(k) * sy;
            const double u = S.H[0] * x + S.H[1] * y + S.H[2];
            const double v = S.H[3] * x + S.H[4] * y + S.H[5];
            const double w = S.H[6] * x + S.H[7] * y + S.H[8];
            const double qx = u / w, qy = v / w;
            double gx, gy;
            if (inside_d(roi, qx, qy)) S.sig[c][k] = bilinear_d(roi, qx, qy, gx, gy);
            else bad = true;
        }
        if (__ballot_sync(0xffffffffu, bad) && lane == 0) atomicOr(&S.oob, 1u << c);
    }
    __syncthreads();
    const uint32_t valid = ~S.oob & cutMask;
    const int n = __popc(valid);
    if (n < 2) {
        if (tid == 0) write_cost(o, FLT_MAX);
        return;
    }
    const double pairs = 0.5 * double(n) * double(n - 1);
    double costPart = 0.0;
    for (int k = tid; k < nS; k += kThreads) {
        double s1 = 0.0, s2 = 0.0;
        uint32_t m = valid;
        while (m) {
            const int c = __ffs(m) - 1;
            m &= m - 1;
            const double v = S.sig[c][k];
            s1 += v;
            s2 += v * v;
        }
        S.mean[k] = s1 / double(n);
        costPart += double(n) * s2 - s1 * s1;
    }
    __syncthreads();
    double gH[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const double coef = 2.0 * double(n) / pairs;
    const double* Hm = S.H;
    for (int c = warp; c < T.ncuts; c += kWarps) {
        if (!((valid >> c) & 1u)) continue;
        const double px = T.stop[c][0], py = T.stop[c][1];
        const double z0 = S.Hi[0] * px + S.Hi[1] * py + S.Hi[2];
        const double z1 = S.Hi[3] * px + S.Hi[4] * py + S.Hi[5];
        const double z2 = S.Hi[6] * px + S.Hi[7] * py + S.Hi[8];
        const double bx = z0 / z2, by = z1 / z2;
        const double xs = bx * bs, ys = by * bs;
        const double sx = (bx - xs) / den, sy = (by - ys) / den;
        double gbx = 0.0, gby = 0.0;
        for (int k = lane; k < nS; k += 32) {
            const double x = xs + double(k) * sx, y = ys + double(k) * sy;
            const double u = Hm[0] * x + Hm[1] * y + Hm[2];
            const double v = Hm[3] * x + Hm[4] * y + Hm[5];
            const double w = Hm[6] * x + Hm[7] * y + Hm[8];
            const double rw = 1.0 / w;
            const double qx = u / w, qy = v / w;
            double gx, gy;
            (void)bilinear_d(roi, qx, qy, gx, gy);
            const double lam = coef * (S.sig[c][k] - S.mean[k]);
            const double fx = lam * gx, fy = lam * gy;
            const double fw = -(fx * qx + fy * qy);
            const double y3[3] = {x, y, 1.0};
            for (int j = 0; j < 3; ++j) {
                gH[j] += fx * rw * y3[j];
                gH[3 + j] += fy * rw * y3[j];
                gH[6 + j] += fw * rw * y3[j];
            }
            const double fX = (fx * (Hm[0] - qx * Hm[6]) + fy * (Hm[3] - qy * Hm[6])) * rw;
            const double fY = (fx * (Hm[1] - qx * Hm[7]) + fy * (Hm[4] - qy * Hm[7])) * rw;
            const double t = bs + double(k) * (1.0 - bs) / den;
            gbx += t * fX;
            gby += t * fY;
        }
        for (int off = 16; off; off >>= 1) {
            gbx += __shfl_xor_sync(0xffffffffu, gbx, off);
            gby += __shfl_xor_sync(0xffffffffu, gby, off);
        }
        if (lane == 0) {
            S.dz[c][0] = gbx / z2;
            S.dz[c][1] = gby / z2;
            S.dz[c][2] = -(gbx * bx + gby * by) / z2;
        }
    }
    double red[10];
    red[0] = costPart;
    for (int j = 0; j < 9; ++j) red[1 + j] = gH[j];
    for (int j = 0; j < 10; ++j)
        for (int off = 16; off; off >>= 1) red[j] += __shfl_xor_sync(0xffffffffu, red[j], off);
    if (lane == 0)
        for (int j = 0; j < 10; ++j) S.red[warp][j] = red[j];
    __syncthreads();
    if (tid == 0) {
        double cost = 0.0, G[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int w = 0; w < kWarps; ++w) {
            cost += S.red[w][0];
            for (int j = 0; j < 9; ++j) G[j] += S.red[w][1 + j];
        }
        cost /= pairs;
        double GHi[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int c = 0; c < T.ncuts; ++c) {
            const double p3[3] = {T.stop[c][0], T.stop[c][1], 1.0};
            for (int r = 0; r < 3; ++r)
                for (int q = 0; q < 3; ++q) GHi[r * 3 + q] += S.dz[c][r] * p3[q];
        }
        double M[9], Mt[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double a = 0.0;
                for (int q = 0; q < 3; ++q) a += GHi[i * 3 + q] * S.Hi[j * 3 + q];
                M[i * 3 + j] = a;
            }
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double a = 0.0;
                for (int q = 0; q < 3; ++q) a += S.Hi[q * 3 + i] * M[q * 3 + j];
                Mt[i * 3 + j] = a;
            }
        double dc[2] = {0.0, 0.0};
        for (int j = 0; j < 9; ++j) {
            G[j] -= Mt[j];
            dc[0] += G[j] * S.dH[0][j];
            dc[1] += G[j] * S.dH[1][j];
        }
        o[0] = float(cost);
        o[1] = float(dc[0]);
        o[2] = float(dc[1]);
        for (int j = 0; j < 9; ++j) o[3 + j] = float(G[j]);
    }
}

void upload_bank(const std::vector<std::vector<float>>& bank, float* d_bank_inv)
{
    std::vector<float> inv(size_t(kMaxBankIds) * kMaxBankRatios, 0.f);
    if (bank.empty() || bank.size() > size_t(kMaxBankIds) || bank[0].size() > size_t(kMaxBankRatios))
        throw Error{CCTAGB_BANK_ERROR, "bank larger than the identification kernel supports"};
    for (size_t i = 0; i < bank.size(); ++i)
        for (size_t r = 0; r < bank[i].size(); ++r) inv[i * kMaxBankRatios + r] = 1.f / bank[i][r];
    CCTAGB_CUDA(cudaMemcpy(d_bank_inv, inv.data(), inv.size() * sizeof(float), cudaMemcpyHostToDevice));
}

void launch_identify(const uint8_t* d_img, size_t pitch, const IdentTask* d_tasks, IdentResult* d_res, int n,
                     const float* d_bank_inv, const IdentParams& ip, cudaStream_t s)
{
    if (n <= 0) return;
    if (ip.gridN * ip.gridN > kMaxTrials || ip.gridN < 3 || (ip.gridN & 1) == 0)
        throw Error{CCTAGB_BAD_ARG, "imagedCenterNGridSample (gnCoarseGrid in Gauss-Newton) must be 3 or 5"};
    if (ip.nSamples > kMaxSamples || ip.nSamples < 32) throw Error{CCTAGB_BAD_ARG, "sampleCutLength out of range"};
    if (ip.refineMode != CCTAGB_REFINE_GRID && ip.refineMode != CCTAGB_REFINE_GAUSS_NEWTON)
        throw Error{CCTAGB_BAD_ARG, "unknown refineMode"};
    if (ip.refineMode == CCTAGB_REFINE_GAUSS_NEWTON && (ip.gnIterations < 1 || ip.gnIterations > 100))
        throw Error{CCTAGB_BAD_ARG, "gnIterations must be in [1, 100]"};
    if (ip.refineMode == CCTAGB_REFINE_GAUSS_NEWTON && (ip.coarseRounds < 1 || ip.coarseRounds > 64))
        throw Error{CCTAGB_BAD_ARG, "gnCoarseRounds must be in [1, 64]"};
    // Few markers: a cluster of blocks each, so that a launch spreads over
    // the SMs; many (or the block layout asked for): one block each, which
    // takes about half the SM time per marker (the per-chunk sums are the
    // same bits).
    int dev = 0, sms = 0;
    CCTAGB_CUDA(cudaGetDevice(&dev));
    CCTAGB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (ip.layout != CCTAGB_IDENT_BLOCK && n * kCluster <= sms) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(unsigned(n * kCluster));
        cfg.blockDim = dim3(kThreads);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = kCluster;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CCTAGB_CUDA(cudaLaunchKernelEx(&cfg, k_identify<kCluster, 1>, d_img, pitch, d_tasks, d_res, d_bank_inv, ip));
    } else if (ip.refineMode == CCTAGB_REFINE_GAUSS_NEWTON) {
        k_identify<1, 2><<<n, kThreads, 0, s>>>(d_img, pitch, d_tasks, d_res, d_bank_inv, ip);
        CCTAGB_CUDA(cudaGetLastError());
    } else {
        k_identify<1, 1><<<n, kThreads, 0, s>>>(d_img, pitch, d_tasks, d_res, d_bank_inv, ip);
        CCTAGB_CUDA(cudaGetLastError());
    }
}

void launch_cut_cost(const uint8_t* d_img, size_t pitch, const IdentTask* d_tasks, const float* d_centers,
                     float* d_out, int n, const IdentParams& ip, cudaStream_t s, bool fp64)
{
    if (n <= 0) return;
    if (ip.nSamples > kMaxSamples || ip.nSamples < 32) throw Error{CCTAGB_BAD_ARG, "sampleCutLength out of range"};
    if (fp64) {
        k_cut_cost_f64<<<n, kThreads, 0, s>>>(d_img, pitch, d_tasks, d_centers, d_out, ip);
    } else {
        k_cut_cost<<<n, kThreads, 0, s>>>(d_img, pitch, d_tasks, d_centers, d_out, ip);
    }
    CCTAGB_CUDA(cudaGetLastError());
}

}  // namespace cctagb
