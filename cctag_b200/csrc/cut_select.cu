// Cut collection and selection on the GPU (identify_step_1 after the outer
// points are sorted: Identification.cpp:396-459 cutInterpolated,
// :471-496 collectCuts, :546-601 selectCutCheapUniform, :604-709
// outerEdgeRefinement / convImageCut; EllipseFromPoints.cpp:29-48
// pointOnEllipse), one thread block per marker, one thread per outer point.
//
// Every expression is the host restatement's, evaluated with explicit IEEE
// roundings in the same order (no contraction into FMAs), so the selected
// cut ends are the same bits as the host's.  The cosine and sine of the
// ellipse angle come from the host (they are the only transcendental values).
#include <cfloat>
#include <cstdint>

#include "common.hpp"
#include "ident_host.hpp"
#include "cctag_b200/portable/pmath.hpp"

namespace cctagb {

namespace {

constexpr int kCutThreads = kMaxOuterPoints;
constexpr int kCutWarps = kCutThreads / 32;
static_assert(kCutThreads % 32 == 0, "whole warps");

__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fd(float a, float b) { return __fdiv_rn(a, b); }

// Identification.hpp:197-219, as the host: ((p0 w1 + p1 w2) + p2 w3 + p3 w4) / 2
__device__ __forceinline__ float bilinear_host(const uint8_t* img, int W, float x, float y)
{
    const int px = int(x), py = int(y);
    const uint8_t* p0 = img + px + size_t(py) * W;
    const float fx = fs(x, float(px)), fy = fs(y, float(py));
    const float fx1 = fs(1.0f, fx), fy1 = fs(1.0f, fy);
    const float w1 = fm(fx1, fy1), w2 = fm(fx, fy1), w3 = fm(fx1, fy), w4 = fm(fx, fy);
    float t = fm(float(p0[0]), w1);
    t = fa(t, fm(float(p0[1]), w2));
    t = fa(t, fm(float(p0[W]), w3));
    t = fa(t, fm(float(p0[W + 1]), w4));
    return fm(t, 0.5f);  // the division by 2, exact
}

// cutInterpolated from (sx, sy) to (ex, ey): the samples' Boost-style mean /
// variance when every sample stays in [1, W-1) x [1, H-1); sig (optional)
// receives the samples.
__device__ bool cut_stats(const uint8_t* img, int W, int H, float sx, float sy, float ex, float ey, float beginSig,
                          int n, float* var_out, float* sig)
{
    const float dX = fs(ex, sx), dY = fs(ey, sy);
    float xs = sx, ys = sy;
    if (beginSig != 0.f) {
        xs = fa(sx, fm(dX, beginSig));
        ys = fa(sy, fm(dY, beginSig));
    }
    const float den = fs(float(n), 1.f);
    const float stepX = fd(fs(ex, xs), den), stepY = fd(fs(ey, ys), den);
    float x = xs, y = ys;
    float mean = 0.f, var = 0.f, rprev = 1.f;
    // 8 samples at a time: their positions (the same running sums) and bounds
    // first, then the 8 bilinear reads, which overlap, then the running mean
    // and variance in sample order
    constexpr int kGroup = 8;
    for (int i0 = 0; i0 < n; i0 += kGroup) {
        float gx[kGroup], gy[kGroup], gv[kGroup];
        bool inside = true;
#pragma unroll
        for (int k = 0; k < kGroup; ++k)
            if (i0 + k < n) {
                gx[k] = x;
                gy[k] = y;
                inside = inside && (x >= 1.f && x < float(W - 1) && y >= 1.f && y < float(H - 1));
                x = fa(x, stepX);
                y = fa(y, stepY);
            }
        if (!inside) return false;
#pragma unroll
        for (int k = 0; k < kGroup; ++k)
            if (i0 + k < n) gv[k] = bilinear_host(img, W, gx[k], gy[k]);
#pragma unroll
        for (int k = 0; k < kGroup; ++k)
            if (i0 + k < n) {
                const float v = gv[k];
                if (sig) sig[i0 + k] = v;
                // MeanVar::add; the divisions by the counts are correctly
                // rounded (div_small: the operands here are zero or normal)
                const int c = i0 + k + 1;
                const float fc = float(c), fc1 = float(c - 1), rc = __frcp_rn(fc);
                mean = pm::div_small(fa(fm(mean, fc1), v), fc, rc);
                if (c > 1) {
                    const float t = fs(v, mean);
                    var = fa(pm::div_small(fm(var, fc1), fc, rc), pm::div_small(fm(t, t), fc1, rprev));
                }
                rprev = rc;
            }
    }
    *var_out = var;
    return true;
}

// convImageCut: (max response, first location of the max), clamped borders.
__device__ void conv_cut(const float* k, const float* sig, int n, float& best, int& loc)
{
    best = 0.f;
    loc = 0;
    for (int i = 0; i < n; ++i) {
        float t = 0.f;
        for (int j = 0; j < 9; ++j) {
            const int r = i - 4 + j;
            t = fa(t, fm(sig[r < 0 ? 0 : (r >= n ? n - 1 : r)], k[j]));
        }
        if (i == 0 || t > best) {
            best = t;
            loc = i;
        }
    }
}

// outerEdgeRefinement: the cut end moves to the strongest derivative
// response along its gradient; false when that cut leaves the image.
__device__ bool refine_stop(float& x, float& y, float dx, float dy, const uint8_t* img, int W, int H, float scale,
                            int nRefine)
{
    const float len = fm(fm(3.f, __fsqrt_rn(2.f)), scale);
    const float hw = fd(len, 2.f);
    const float gn = __fsqrt_rn(fa(fm(dx, dx), fm(dy, dy)));
    const float gx = fd(dx, gn), gy = fd(dy, gn);
    const float ax = fs(x, fm(hw, gx)), ay = fs(y, fm(hw, gy));
    const float bx = fa(x, fm(hw, gx)), by = fa(y, fm(hw, gy));
    float sig[kMaxRefineSamples];
    float unused;
    if (!cut_stats(img, W, H, ax, ay, bx, by, 0.f, nRefine, &unused, sig)) return false;
    const float kA[9] = {-0.0000f, -0.0003f, -0.1065f, -0.7863f, .0f, 0.7863f, 0.1065f, 0.0003f, 0.0000f};
    const float kB[9] = {-0.0044f, -0.0540f, -0.2376f, -0.3450f, .0f, 0.3450f, 0.2376f, 0.0540f, 0.0044f};
    const float kC[9] = {-0.0366f, -0.1113f, -0.1801f, -0.1594f, .0f, 0.1594f, 0.1801f, 0.1113f, 0.0366f};
    // std::map<float, float> insert of (A), (B), (C): the largest response
    // wins, an equal later one does not replace an earlier one.
    float best, b;
    int loc, l;
    conv_cut(kA, sig, nRefine, best, loc);
    conv_cut(kB, sig, nRefine, b, l);
    if (b > best) {
        best = b;
        loc = l;
    }
    conv_cut(kC, sig, nRefine, b, l);
    if (b > best) {
        best = b;
        loc = l;
    }
    const float step = fd(len, fs(float(nRefine), 1.f));
    x = fa(ax, fm(fm(step, float(loc)), gx));
    y = fa(ay, fm(fm(step, float(loc)), gy));
    return true;
}

}  // namespace

__global__ void __launch_bounds__(kCutThreads) k_cut_select(const uint8_t* __restrict__ img, int W, int H,
                                                            const CutSelectIn* __restrict__ ins,
                                                            const DirPoint* __restrict__ pts,
                                                            const int16_t* __restrict__ sel,
                                                            const int* __restrict__ nsel, IdentTask* tasks,
                                                            int* status, CutSelectParams cp)
{
    __shared__ float s_x[kCutThreads], s_y[kCutThreads], s_wmax[kCutWarps];
    __shared__ int s_keep[kCutThreads], s_wcnt[kCutWarps];
    const CutSelectIn in = ins[blockIdx.x];
    const int i = threadIdx.x;
    IdentTask& T = tasks[blockIdx.x];
    // the outer points sorted by angle and subsampled (k_outer_select)
    const int count = nsel[blockIdx.x];
    if (count < 5) {  // identify_step_1's TOO_FEW_OUTER_POINTS
        if (i == 0) {
            T.ncuts = 0;
            status[blockIdx.x] = CCTAGB_TOO_FEW_OUTER_POINTS;
        }
        return;
    }
    bool ok = false, ref = false;
    float var = 0.f, sx = 0.f, sy = 0.f;
    if (i < count) {
        const DirPoint op = pts[in.first + sel[size_t(blockIdx.x) * kMaxOuterPoints + i]];
        ok = cut_stats(img, W, H, in.cx, in.cy, op.x, op.y, cp.beginSig, cp.nSamples, &var, nullptr);
        if (ok) {
            // pointOnEllipse with the host's cos / sin of the angle
            const float x = fs(op.x, in.cx), y = fs(op.y, in.cy);
            float tx = fa(fm(x, in.cosA), fm(y, in.sinA));
            float ty = fa(fm(-x, in.sinA), fm(y, in.cosA));
            const float cs = __fsqrt_rn(fa(fd(fm(tx, tx), fm(in.a, in.a)), fd(fm(ty, ty), fm(in.b, in.b))));
            tx = fd(tx, cs);
            ty = fd(ty, cs);
            sx = fa(fs(fm(tx, in.cosA), fm(ty, in.sinA)), in.cx);
            sy = fa(fa(fm(tx, in.sinA), fm(ty, in.cosA)), in.cy);
            ref = refine_stop(sx, sy, op.dx, op.dy, img, W, H, in.scale, cp.nRefine);
        }
    }
    s_x[i] = sx;
    s_y[i] = sy;
    // selectCutCheapUniform over the collected (in-image) cuts, in order,
    // block-parallel.  The variances are finite and >= +0 (means and squares
    // of finite samples), so the largest one has a single bit pattern and any
    // reduction order gives the serial first-max.
    const int lane = i & 31, warp = i >> 5;
    float vm = ok ? var : -1.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) vm = fmaxf(vm, __shfl_xor_sync(0xffffffffu, vm, o));
    if (lane == 0) s_wmax[warp] = vm;
    const int nOk = __syncthreads_count(ok);
    if (nOk == 0) {
        if (i == 0) {
            T.ncuts = 0;
            status[blockIdx.x] = CCTAGB_NO_COLLECTED_CUTS;
        }
        return;
    }
    float varMax = s_wmax[0];
#pragma unroll
    for (int w = 1; w < kCutWarps; ++w) varMax = fmaxf(varMax, s_wmax[w]);
    // the kept cuts, compacted in point order: rank = kept cuts before i
    const bool kp = ok && ref && fd(var, varMax) > 0.5f;
    const unsigned kb = __ballot_sync(0xffffffffu, kp);
    if (lane == 0) s_wcnt[warp] = __popc(kb);
    __syncthreads();
    int rank = __popc(kb & ((1u << lane) - 1u)), nKeep = 0;
#pragma unroll
    for (int w = 0; w < kCutWarps; ++w) {
        rank += w < warp ? s_wcnt[w] : 0;
        nKeep += s_wcnt[w];
    }
    if (kp) s_keep[rank] = i;
    __syncthreads();
    // The serial loop's k-th pick is keep[int(k * step)] while k < selectSize
    // and that index < nKeep; the index is non-decreasing in k, so the picks
    // are the prefix of k where both hold, one thread per k.
    const int selectSize = min(cp.maxSelect, nOk);
    const float step = fmaxf(1.f, fd(float(nKeep), float(selectSize)));
    const int j = int(fm(float(i), step));
    const bool pick = i < selectSize && j < nKeep;
    if (pick) {
        T.stop[i][0] = s_x[s_keep[j]];
        T.stop[i][1] = s_y[s_keep[j]];
    }
    const int nCuts = __syncthreads_count(pick);
    if (i == 0) {
        T.ncuts = nCuts;
        status[blockIdx.x] = nCuts == 0 ? CCTAGB_NO_SELECTED_CUTS : CCTAGB_ID_RELIABLE;
    }
}

void launch_cut_select(const uint8_t* d_img, int W, int H, const CutSelectIn* d_ins, const DirPoint* d_pts,
                       const int16_t* d_sel, const int* d_nsel, IdentTask* d_tasks, int* d_status, int n,
                       const CutSelectParams& cp, cudaStream_t s)
{
    if (n <= 0) return;
    if (cp.nSamples < 2 || cp.nSamples > kMaxSamples) throw Error{CCTAGB_BAD_ARG, "sampleCutLength out of range"};
    if (cp.nRefine < 2 || cp.nRefine > kMaxRefineSamples)
        throw Error{CCTAGB_BAD_ARG, "numSamplesOuterEdgePointsRefinement out of range"};
    k_cut_select<<<n, kCutThreads, 0, s>>>(d_img, W, H, d_ins, d_pts, d_sel, d_nsel, d_tasks, d_status, cp);
    CCTAGB_CUDA(cudaGetLastError());
}

}  // namespace cctagb
