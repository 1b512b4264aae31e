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

namespace cctagb {

namespace {

constexpr int kMaxTrials = 25;
constexpr int kThreads = 32 * kMaxTrials;
// Thread blocks per marker (one cluster): each evaluates every trial on its
// quarter of the samples along the cuts, so a marker's trials run on four
// SMs; the partial costs meet through distributed shared memory.
constexpr int kCluster = 4;

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

// Identification.hpp:197-219
__device__ __forceinline__ float bilinear(const uint8_t* __restrict__ img, int W, float x, float y)
{
    const int px = int(x), py = int(y);
    const uint8_t* p0 = img + px + size_t(py) * W;
    const float fx = x - float(px), fy = y - float(py);
    const float fx1 = 1.0f - fx, fy1 = 1.0f - fy;
    const float p1 = __ldg(p0), p2 = __ldg(p0 + 1), p3 = __ldg(p0 + W), p4 = __ldg(p0 + W + 1);
    return (p1 * (fx1 * fy1) + p2 * (fx * fy1) + p3 * (fx1 * fy) + p4 * (fx * fy)) / 2;
}

__device__ __forceinline__ bool inside(float x, float y, int W, int H)
{
    return x >= 0.f && x < float(W - 1) && y >= 0.f && y < float(H - 1);
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
    float cutp[kMaxTrials][kMaxCuts][4];  // xStart, yStart, stepX, stepY (marker plane)
    uint32_t trialOob[kMaxTrials];
    uint32_t valid[kMaxTrials];
    float cost[kMaxTrials];
    double part[2][kMaxTrials];    // this block's share of each trial's cost (by round parity)
    float sig[kMaxCuts][kMaxSamples];
    float barcode[kMaxSamples];
    int winner[kMaxCuts];
    float vwin[kMaxCuts];
};

// Per trial (one warp): homography, cut parameters in the marker plane and
// the cuts whose end samples leave the image.
__device__ void setup_trial(Shared& S, const IdentTask& T, int t, float px, float py, const IdentParams& ip, int W,
                            int H, int lane)
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
        S.cutp[t][lane][0] = xs;
        S.cutp[t][lane][1] = ys;
        S.cutp[t][lane][2] = sx;
        S.cutp[t][lane][3] = sy;
        float x0, y0, w0, x1, y1, w1;
        apply_h(Hm, xs, ys, x0, y0, w0);
        const float kl = float(ip.nSamples - 1);
        apply_h(Hm, xs + kl * sx, ys + kl * sy, x1, y1, w1);
        bad = !(w0 > 0.f && w1 > 0.f) && !(w0 < 0.f && w1 < 0.f);
        bad = bad || !inside(x0, y0, W, H) || !inside(x1, y1, W, H);
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

// Identification.hpp:197-219 for a sample known to lie inside the image
// (the integer corner is clamped so that rounding at the border never reads
// outside the frame).
__device__ __forceinline__ float bilinear_in(const uint8_t* __restrict__ img, int W, int H, float x, float y)
{
    float fpx, fpy;
    int px = floor_small(fmaxf(x, 0.f), fpx);
    int py = floor_small(fmaxf(y, 0.f), fpy);
    const float fx = x - fpx, fy = y - fpy;
    px = min(px, W - 2);
    py = min(py, H - 2);
    const uint8_t* p0 = img + px + size_t(py) * W;
    const float fx1 = 1.0f - fx, fy1 = 1.0f - fy;
    const float p1 = byte_to_float(__ldg(p0)), p2 = byte_to_float(__ldg(p0 + 1));
    const float p3 = byte_to_float(__ldg(p0 + W)), p4 = byte_to_float(__ldg(p0 + W + 1));
    return (p1 * (fx1 * fy1) + p2 * (fx * fy1) + p3 * (fx1 * fy) + p4 * (fx * fy)) * 0.5f;
}

// One sample of cut c of trial t (marker plane -> image, bilinear read).
__device__ __forceinline__ float cut_sample(const Shared& S, const uint8_t* __restrict__ img, int W, int H, int t,
                                            int c, float kf, const float* Hm)
{
    const float* cp = S.cutp[t][c];
    const float x = cp[0] + kf * cp[2], y = cp[1] + kf * cp[3];
    const float u = Hm[0] * x + Hm[1] * y + Hm[2];
    const float v = Hm[3] * x + Hm[4] * y + Hm[5];
    const float w = Hm[6] * x + Hm[7] * y + Hm[8];
    const float r = __frcp_rn(w);
    return bilinear_in(img, W, H, u * r, v * r);
}

// This block's share of the cost of trial t (one warp): the samples
// k0 <= k < k1 (at most 32, one per lane) over the valid cuts, taken four
// cuts at a time so that their reads overlap.  Per sample the cut values are
// shifted by the first valid cut's value before the FP32 sums (the cost term
// n * sum(d^2) - (sum d)^2 does not change under a common shift, and the
// shifted sums stay small); the per-sample terms are summed in FP64.
__device__ double trial_partial(const Shared& S, const uint8_t* __restrict__ img, int W, int H, int t,
                               uint32_t valid, int k0, int k1, int lane)
{
    const int n = __popc(valid);
    const int k = k0 + lane;
    double acc = 0.0;
    if (n >= 2 && k < k1) {
        float Hm[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) Hm[i] = S.trialH[t][i];
        const float kf = float(k);
        float v0 = 0.f, s1 = 0.f, s2 = 0.f;
        bool first = true;
        uint32_t m = valid;
        while (m) {
            int c[4];
            int cnt = 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                c[q] = m ? __ffs(m) - 1 : c[q > 0 ? q - 1 : 0];
                if (m) {
                    m &= m - 1;
                    ++cnt;
                }
            }
            float val[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) val[q] = cut_sample(S, img, W, H, t, c[q], kf, Hm);
            if (first) {
                v0 = val[0];
                first = false;
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (q < cnt) {
                    const float d = val[q] - v0;
                    s1 += d;
                    s2 = fmaf(d, d, s2);
                }
            }
        }
        acc = double(float(n) * s2 - s1 * s1);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    return acc;
}

// Identification.hpp:373-384
__device__ __forceinline__ float dis(float sig, float val, float mub, float muw, float var)
{
    if (val == -1.f) {
        const float d = fmaxf(sig - mub, 0.f);
        return d * d / (2.0f * var);
    }
    const float d = fminf(sig - muw, 0.f);
    return d * d / (2.0f * var);
}

}  // namespace

__global__ void __cluster_dims__(kCluster, 1, 1) __launch_bounds__(kThreads)
    k_identify(const uint8_t* __restrict__ img, int W, int H, const IdentTask* __restrict__ tasks, IdentResult* res,
               const float* __restrict__ bankInv, IdentParams ip)
{
    namespace cg = cooperative_groups;
    __shared__ Shared S;
    cg::cluster_group cluster = cg::this_cluster();
    const int crank = int(cluster.block_rank());
    const int marker = blockIdx.x / kCluster;
    const IdentTask& T = tasks[marker];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nS = ip.nSamples;
    // this block's samples along every cut (at most 32: one per lane)
    const int chunk = (nS + kCluster - 1) / kCluster;
    const int k0 = min(nS, crank * chunk), k1 = min(nS, k0 + chunk);
    const int gridN = ip.gridN;
    const int nTrials = gridN * gridN;
    const uint32_t cutMask = (T.ncuts >= 32) ? 0xffffffffu : ((1u << T.ncuts) - 1u);

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
        S.rounds = r;
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
            setup_trial(S, T, warp, px, py, ip, W, H, lane);
        }
        __syncthreads();
        if (tid == 0) {
            uint32_t m = S.oob;
            for (int t = 0; t < nTrials; ++t) {
                m |= S.trialOob[t];
                S.valid[t] = ~m & cutMask;
            }
            S.oob = m;
        }
        __syncthreads();
        const int par = round & 1;
        if (warp < nTrials) {
            const double c = trial_partial(S, img, W, H, warp, S.valid[warp], k0, k1, lane);
            if (lane == 0) S.part[par][warp] = c;
        }
        // All blocks of the marker have their shares; a block reuses this
        // parity's array two rounds later, after the next cluster barrier,
        // when every block has finished reading it.
        cluster.sync();
        if (warp == 0 && lane < nTrials) {
            double acc = 0.0;
            for (int r = 0; r < kCluster; ++r) acc += cluster.map_shared_rank(&S.part[par][0], r)[lane];
            const int n = __popc(S.valid[lane]);
            S.cost[lane] = n >= 2 ? float(acc / (0.5 * double(n) * double(n - 1))) : FLT_MAX;
        }
        __syncthreads();
        if (tid == 0) {
            // imageCenterOptimizationGlob: first strict minimum in trial order.
            float best = FLT_MAX;
            int bi = -1;
            bool readable = false;
            for (int t = 0; t < nTrials; ++t) {
                if (__popc(S.valid[t]) >= 2) readable = true;
                if (S.cost[t] < best) {
                    best = S.cost[t];
                    bi = t;
                }
            }
            if (!readable || bi < 0) {
                S.fail = 1;
            } else {
                S.cx = S.trialPt[bi][0];
                S.cy = S.trialPt[bi][1];
                for (int k = 0; k < 9; ++k) S.Hopt[k] = S.trialH[bi][k];
                S.minRes = best;
            }
        }
        __syncthreads();
        if (S.fail) break;
        ns /= float((gridN - 1) / 2);
    }
    // No block leaves while another may still read its shared memory; the
    // rest of the identification runs in the first block of the cluster.
    cluster.sync();
    if (crank != 0) return;
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
        }
        return;
    }
    // Final signals with the optimal homography (getSignals, Identification.cpp:901).
    constexpr int kWarps = kThreads / 32;
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
            if (inside(xr, yr, W, H)) S.sig[c][k] = bilinear(img, W, xr, yr);
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
        float mean = 0.f, var = 0.f;
        {
            int cnt = 0;
            for (int k = 30; k < nS; ++k) {
                ++cnt;
                const float x = sg[k];
                mean = (mean * float(cnt - 1) + x) / float(cnt);
                if (cnt > 1) {
                    const float t = x - mean;
                    var = var * float(cnt - 1) / float(cnt) + t * t / float(cnt - 1);
                }
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
                        mub = (mub * float(ni - 1) + x) / float(ni);
                    } else {
                        ++nsup;
                        muw = (muw * float(nsup - 1) + x) / float(nsup);
                    }
                }
            }
        }
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
                for (int k = 0; k < nS; ++k) {
                    int ldum = 0;
#pragma unroll
                    for (int r = 0; r < kMaxBankRatios; ++r) ldum += (inv[r] <= x) ? 1 : 0;
                    dist += dis(sg[k], float(-(ldum % 2) * 2 + 1), mub, muw, var);
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

void upload_bank(const std::vector<std::vector<float>>& bank, float* d_bank_inv)
{
    std::vector<float> inv(size_t(kMaxBankIds) * kMaxBankRatios, 0.f);
    if (bank.empty() || bank.size() > size_t(kMaxBankIds) || bank[0].size() > size_t(kMaxBankRatios))
        throw Error{CCTAGB_BANK_ERROR, "bank larger than the identification kernel supports"};
    for (size_t i = 0; i < bank.size(); ++i)
        for (size_t r = 0; r < bank[i].size(); ++r) inv[i * kMaxBankRatios + r] = 1.f / bank[i][r];
    CCTAGB_CUDA(cudaMemcpy(d_bank_inv, inv.data(), inv.size() * sizeof(float), cudaMemcpyHostToDevice));
}

void launch_identify(const uint8_t* d_img, int W, int H, const IdentTask* d_tasks, IdentResult* d_res, int n,
                     const float* d_bank_inv, const IdentParams& ip, cudaStream_t s)
{
    if (n <= 0) return;
    if (ip.gridN * ip.gridN > kMaxTrials || ip.gridN < 3 || (ip.gridN & 1) == 0)
        throw Error{CCTAGB_BAD_ARG, "imagedCenterNGridSample must be 3 or 5"};
    if (ip.nSamples > kMaxSamples || ip.nSamples < 32) throw Error{CCTAGB_BAD_ARG, "sampleCutLength out of range"};
    k_identify<<<n * kCluster, kThreads, 0, s>>>(d_img, W, H, d_tasks, d_res, d_bank_inv, ip);
    CCTAGB_CUDA(cudaGetLastError());
}

}  // namespace cctagb
