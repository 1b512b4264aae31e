// TEST INFRASTRUCTURE ONLY -- CPU oracle for the CCTag image stage and vote.
//
// This file restates, on the CPU and in plain C++, the reference CCTag CPU path
// (`Parameters::_useCuda == false`) for: the image pyramid, the 9x9
// derivative-of-Gaussian, Canny non-maximum suppression and hysteresis,
// thinning, raster edge-point collection, the Bresenham gradient walk and the
// vote with seed selection.  It exists so that tests, `__graft_entry__.smoke()`
// and the CPU-baseline leg of `bench.py` can check and time the CUDA product
// path against it.  Nothing in the product library links or calls it.
//
// Arithmetic pins:
//  * derivatives: `cv::filter2D(CV_8U -> CV_16S, BORDER_REPLICATE)` with the
//    reference kernel (filter/cvRecode.cpp:74-92).  OpenCV accumulates the 72
//    non-zero taps in row-major order with fused multiply-add, starting from
//    delta = 0, then rounds half-to-even and saturates; this file does the same
//    and is checked bit-exactly against cv2.filter2D by the test-suite.
//  * everything else in the reference is compiled without FMA contraction
//    (no -mavx2/-mfma in its CMakeLists.txt), so this file is compiled with
//    -ffp-contract=off.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "oracle.h"
#include "oracle_internal.hpp"

namespace orc {

// ---------------------------------------------------------------- pyramid --
// ImagePyramid.cpp:23-33 (floor halving), Level.cpp:57-81 (cv::resize of the
// previous level, INTER_LINEAR).  For an exact 2x reduction OpenCV takes its
// area fast path: the rounded mean of each 2x2 block.  Other ratios use the
// fixed-point bilinear rule of cv::resize (11-bit coefficients, vectorised
// vertical pass), pinned bit-exactly against cv2.resize by the test-suite.
static void resize_linear_generic(const uint8_t* src, int sw, int sh, uint8_t* dst, int dw, int dh)
{
    const double sx_scale = double(sw) / dw, sy_scale = double(sh) / dh;
    const int kScale = 2048;
    std::vector<int> xofs(dw), yofs(dh);
    std::vector<short> xa(2 * dw), ya(2 * dh);
    for (int d = 0; d < dw; ++d) {
        float f = float((d + 0.5) * sx_scale - 0.5);
        int s = int(std::floor(f));
        f -= s;
        if (s < 0) { f = 0; s = 0; }
        if (s >= sw - 1) { f = 0; s = sw - 1; }
        xofs[d] = s;
        short c0 = short(std::lrint((1.f - f) * kScale));
        xa[2 * d] = c0; xa[2 * d + 1] = short(kScale - c0);
    }
    for (int d = 0; d < dh; ++d) {
        float f = float((d + 0.5) * sy_scale - 0.5);
        int s = int(std::floor(f));
        f -= s;
        if (s < 0) { f = 0; s = 0; }
        if (s >= sh - 1) { f = 0; s = sh - 1; }
        yofs[d] = s;
        short c0 = short(std::lrint((1.f - f) * kScale));
        ya[2 * d] = c0; ya[2 * d + 1] = short(kScale - c0);
    }
    std::vector<int> r0(dw), r1(dw);
    for (int y = 0; y < dh; ++y) {
        const int sy0 = yofs[y], sy1 = std::min(sy0 + 1, sh - 1);
        for (int x = 0; x < dw; ++x) {
            const int s0 = xofs[x], s1 = std::min(s0 + 1, sw - 1);
            r0[x] = src[sy0 * sw + s0] * xa[2 * x] + src[sy0 * sw + s1] * xa[2 * x + 1];
            r1[x] = src[sy1 * sw + s0] * xa[2 * x] + src[sy1 * sw + s1] * xa[2 * x + 1];
        }
        for (int x = 0; x < dw; ++x) {
            // OpenCV's vectorised vertical pass: 16-bit high products of the
            // pre-shifted horizontal sums, then a rounding shift by 2.
            int v = ((((r0[x] >> 4) * ya[2 * y]) >> 16) + (((r1[x] >> 4) * ya[2 * y + 1]) >> 16) + 2) >> 2;
            dst[y * dw + x] = uint8_t(std::min(255, std::max(0, v)));
        }
    }
}

void pyramid_down(const uint8_t* src, int sw, int sh, uint8_t* dst, int dw, int dh)
{
    if (sw == 2 * dw && sh == 2 * dh) {
        for (int y = 0; y < dh; ++y)
            for (int x = 0; x < dw; ++x) {
                const uint8_t* p = src + (2 * y) * sw + 2 * x;
                dst[y * dw + x] = uint8_t((p[0] + p[1] + p[sw] + p[sw + 1] + 2) >> 2);
            }
    } else {
        resize_linear_generic(src, sw, sh, dst, dw, dh);
    }
}

// ------------------------------------------------------------ derivatives --
// filter/cvRecode.cpp:74-92.  kerneldX(i,j) = g(i) * d(j); kerneldY = kerneldX^T.
const float kDoG[9][9] = {
    {-0.000000143284235f, -0.000003558691641f, -0.000028902492951f, -0.000064765993382f, 0.f, 0.000064765993382f, 0.000028902492951f, 0.000003558691641f, 0.000000143284235f},
    {-0.000004744922188f, -0.000117847682078f, -0.000957119116802f, -0.002144755142391f, 0.f, 0.002144755142391f, 0.000957119116802f, 0.000117847682078f, 0.000004744922188f},
    {-0.000057804985902f, -0.001435678675203f, -0.011660097860113f, -0.026128466569370f, 0.f, 0.026128466569370f, 0.011660097860113f, 0.001435678675203f, 0.000057804985902f},
    {-0.000259063973527f, -0.006434265427174f, -0.052256933138740f, -0.117099663048638f, 0.f, 0.117099663048638f, 0.052256933138740f, 0.006434265427174f, 0.000259063973527f},
    {-0.000427124283626f, -0.010608310271112f, -0.086157117207395f, -0.193064705260108f, 0.f, 0.193064705260108f, 0.086157117207395f, 0.010608310271112f, 0.000427124283626f},
    {-0.000259063973527f, -0.006434265427174f, -0.052256933138740f, -0.117099663048638f, 0.f, 0.117099663048638f, 0.052256933138740f, 0.006434265427174f, 0.000259063973527f},
    {-0.000057804985902f, -0.001435678675203f, -0.011660097860113f, -0.026128466569370f, 0.f, 0.026128466569370f, 0.011660097860113f, 0.001435678675203f, 0.000057804985902f},
    {-0.000004744922188f, -0.000117847682078f, -0.000957119116802f, -0.002144755142391f, 0.f, 0.002144755142391f, 0.000957119116802f, 0.000117847682078f, 0.000004744922188f},
    {-0.000000143284235f, -0.000003558691641f, -0.000028902492951f, -0.000064765993382f, 0.f, 0.000064765993382f, 0.000028902492951f, 0.000003558691641f, 0.000000143284235f}};

static inline int16_t sat_round16(float s)
{
    float r = std::nearbyint(s);  // default rounding mode: half to even
    r = std::min(32767.f, std::max(-32768.f, r));
    return int16_t(r);
}

void derivatives(const uint8_t* src, int W, int H, int16_t* dx, int16_t* dy)
{
    // Replicated border of 4, converted to float once.  For each output row the
    // taps are applied in the reference's row-major order, vectorised over x
    // (the per-pixel accumulation order is unchanged).
    const int PW = W + 8;
    std::vector<float> pad(size_t(PW) * (H + 8));
    for (int y = 0; y < H + 8; ++y) {
        const int sy = std::min(H - 1, std::max(0, y - 4));
        for (int x = 0; x < PW; ++x) {
            const int sx = std::min(W - 1, std::max(0, x - 4));
            pad[size_t(y) * PW + x] = float(src[size_t(sy) * W + sx]);
        }
    }
    std::vector<float> ax(W), ay(W);
    for (int y = 0; y < H; ++y) {
        std::fill(ax.begin(), ax.end(), 0.f);
        std::fill(ay.begin(), ay.end(), 0.f);
        for (int i = 0; i < 9; ++i) {
            const float* row = &pad[size_t(y + i) * PW];
            for (int j = 0; j < 9; ++j) {
                const float kx = kDoG[i][j];  // kerneldX(i, j)
                const float ky = kDoG[j][i];  // kerneldY(i, j)
                const float* r = row + j;
                if (j != 4)
                    for (int x = 0; x < W; ++x) ax[x] = std::fma(kx, r[x], ax[x]);
                if (i != 4)
                    for (int x = 0; x < W; ++x) ay[x] = std::fma(ky, r[x], ay[x]);
            }
        }
        for (int x = 0; x < W; ++x) {
            dx[size_t(y) * W + x] = sat_round16(ax[x]);
            dy[size_t(y) * W + x] = sat_round16(ay[x]);
        }
    }
}

// ------------------------------------------------------------------ canny --
// filter/cvRecode.cpp:107-108 thresholds, :174-330 magnitude + NMS with the
// deferral rules (prev_flag, "pixel above already strong"), :362-394 stack
// hysteresis, :400-409 output.  Map values as in the reference:
// 1 = cannot be an edge, 0 = may be an edge (weak), 2 = edge (strong).
void canny(const int16_t* dx, const int16_t* dy, int W, int H, float thrLow, float thrHigh,
           uint8_t* edges, uint8_t* nms_out)
{
    if (thrLow > thrHigh) std::swap(thrLow, thrHigh);
    const int low = int(std::floor(thrLow)), high = int(std::floor(thrHigh));
    const int TG22 = int(0.4142135623730950488016887242097 * (1 << 15) + 0.5);
    const ptrdiff_t ms = W + 2;  // padded map stride
    std::vector<uint8_t> map(size_t(ms) * (H + 2), 1);
    std::vector<int> magrows(3 * size_t(ms), 0);
    auto magrow = [&](int r) -> int* {  // r in [-1, H]: image row r, padded by 1 each side
        return &magrows[size_t((r + 3) % 3) * ms + 1];
    };
    auto fill_mag = [&](int r) {
        int* m = magrow(r);
        m[-1] = m[W] = 0;
        if (r < 0 || r >= H) {
            for (int j = 0; j < W; ++j) m[j] = 0;
            return;
        }
        for (int j = 0; j < W; ++j) {
            const float x = float(dx[size_t(r) * W + j]), y = float(dy[size_t(r) * W + j]);
            m[j] = int(std::nearbyint(std::sqrt(x * x + y * y)));
        }
    };
    std::vector<uint8_t*> stack;
    stack.reserve(size_t(W) * H / 10 + 1024);
    auto push = [&](uint8_t* p) { *p = 2; stack.push_back(p); };

    fill_mag(-1);
    fill_mag(0);
    for (int i = 0; i < H; ++i) {
        fill_mag(i + 1);
        const int* mc = magrow(i);
        const int* mu = magrow(i - 1);
        const int* md = magrow(i + 1);
        uint8_t* mp = &map[size_t(i + 1) * ms + 1];
        int prev_flag = 0;
        for (int j = 0; j < W; ++j) {
            int x = dx[size_t(i) * W + j], y = dy[size_t(i) * W + j];
            const int s = x ^ y;
            const int m = mc[j];
            x = std::abs(x);
            y = std::abs(y);
            bool is_max = false;
            if (m > low) {
                const int tg22x = x * TG22;
                const int tg67x = tg22x + ((x + x) << 15);
                y <<= 15;
                if (y < tg22x) {
                    is_max = m > mc[j - 1] && m >= mc[j + 1];
                } else if (y > tg67x) {
                    is_max = m > mu[j] && m >= md[j];
                } else {
                    const int sg = s < 0 ? -1 : 1;
                    is_max = m > mu[j - sg] && m > md[j + sg];
                }
            }
            if (is_max) {
                if (m > high && !prev_flag && mp[j - ms] != 2) {
                    push(mp + j);
                    prev_flag = 1;
                } else {
                    mp[j] = 0;
                }
            } else {
                prev_flag = 0;
                mp[j] = 1;
            }
        }
    }
    if (nms_out) {
        for (int i = 0; i < H; ++i)
            for (int j = 0; j < W; ++j) nms_out[size_t(i) * W + j] = map[size_t(i + 1) * ms + 1 + j];
    }
    while (!stack.empty()) {
        uint8_t* m = stack.back();
        stack.pop_back();
        const ptrdiff_t nb[8] = {-1, 1, -ms - 1, -ms, -ms + 1, ms - 1, ms, ms + 1};
        for (ptrdiff_t o : nb)
            if (!m[o]) push(m + o);
    }
    for (int i = 0; i < H; ++i)
        for (int j = 0; j < W; ++j)
            edges[size_t(i) * W + j] = uint8_t(-(map[size_t(i + 1) * ms + 1 + j] >> 1));
}

// --------------------------------------------------------------- thinning --
// filter/thinning.cpp:12-51: two table-driven passes over the interior pixels,
// edges -> temp with the first table, temp -> edges with the second.  The
// tables are the two sub-iterations of the Lam-Lee-Suen parallel thinning
// (IEEE PAMI 14(9), 1992): a set pixel is deleted when G1 (crossing number
// X_H == 1), G2 (2 <= min(n1, n2) <= 3) and G3 (first pass) or G3' (second pass)
// hold.  The 9-bit index weights are (x-1,y-1)=1, (x-1,y)=2, (x-1,y+1)=4,
// (x,y-1)=8, (x,y)=16, (x,y+1)=32, (x+1,y-1)=64, (x+1,y)=128, (x+1,y+1)=256,
// with x the column and y the row.  The border of `temp` is never written by
// the reference (uninitialised); it is 0 here.
void thin_lut(int pass, uint8_t* lut)
{
    for (int idx = 0; idx < 512; ++idx) {
        auto bit = [&](int w) { return (idx & w) ? 1 : 0; };
        if (!bit(16)) { lut[idx] = 0; continue; }
        // x1..x8 counter-clockwise from east; x9 = x1
        const int x[10] = {0, bit(128), bit(64), bit(8), bit(1), bit(2), bit(4), bit(32), bit(256), bit(128)};
        int xh = 0, n1 = 0, n2 = 0;
        for (int i = 1; i <= 4; ++i) {
            xh += (x[2 * i - 1] == 0 && (x[2 * i] == 1 || x[2 * i + 1] == 1)) ? 1 : 0;
            n1 += x[2 * i - 1] | x[2 * i];
            n2 += x[2 * i] | x[2 * i + 1];
        }
        const bool g1 = xh == 1;
        const int mn = std::min(n1, n2);
        const bool g2 = mn >= 2 && mn <= 3;
        const bool g3 = pass == 1 ? (((x[2] | x[3] | (1 - x[8])) & x[1]) == 0)
                                  : (((x[6] | x[7] | (1 - x[4])) & x[5]) == 0);
        lut[idx] = (g1 && g2 && g3) ? 0 : 255;
    }
}

static void thin_pass(const uint8_t* in, uint8_t* out, int W, int H, const uint8_t* lut)
{
    for (int y = 1; y < H - 1; ++y)
        for (int x = 1; x < W - 1; ++x) {
            const uint8_t* c = in + size_t(y) * W + x;
            if (*c == 0) { out[size_t(y) * W + x] = 0; continue; }
            const int idx = (c[-W - 1] == 255) * 1 + (c[-1] == 255) * 2 + (c[W - 1] == 255) * 4 +
                            (c[-W] == 255) * 8 + (c[0] == 255) * 16 + (c[W] == 255) * 32 +
                            (c[-W + 1] == 255) * 64 + (c[1] == 255) * 128 + (c[W + 1] == 255) * 256;
            out[size_t(y) * W + x] = lut[idx];
        }
}

void thin(uint8_t* edges, int W, int H)
{
    uint8_t lut1[512], lut2[512];
    thin_lut(1, lut1);
    thin_lut(2, lut2);
    std::vector<uint8_t> temp(size_t(W) * H, 0);
    thin_pass(edges, temp.data(), W, H, lut1);
    thin_pass(temp.data(), edges, W, H, lut2);
}

// ---------------------------------------------------- edges, walk, vote --
// Canny.cpp:15-31 (raster collection), Types.cpp:40-61 (add_point),
// EdgePoint.hpp:24-91 (normGrad = sqrt(dx^2+dy^2) in float).
static inline int sgn_i(int v) { return (v > 0) - (v < 0); }

// Bresenham.cpp:18-31 updateXY, with the roles of x/y chosen by the caller.
static inline void update_xy(float d_major, float d_minor, int& major, int& minor, float& e, int& stp_major,
                             int& stp_minor)
{
    const float a = std::fabs(d_minor / d_major);
    stp_major = sgn_i(int(d_major));
    stp_minor = sgn_i(int(d_minor));
    e += a;
    major += stp_major;
    if (e >= 0.5f) {
        minor += stp_minor;
        e -= 1.f;
    }
}

// Bresenham.cpp:33-209 gradientDirectionDescent.  Returns the edge index or -1.
int gradient_walk(const int32_t* idxmap, int W, int H, int px, int py, int gdx, int gdy, int dir, int nmax,
                  int thrGradient)
{
    float e = 0.f;
    float dx = float(dir * gdx), dy = float(dir * gdy);
    const float dxRef = dx, dyRef = dy;
    const bool y_major = std::fabs(dy) > std::fabs(dx);
    int x = px, y = py, stpX = 0, stpY = 0;
    int n = 0;
    auto step = [&]() {
        if (y_major) update_xy(dy, dx, y, x, e, stpY, stpX);
        else         update_xy(dx, dy, x, y, e, stpX, stpY);
        ++n;
    };
    auto inside = [&](int xx, int yy) { return xx >= 0 && xx < W && yy >= 0 && yy < H; };
    step();
    if (dx * dx + dy * dy > float(thrGradient)) {
        // Re-orientation with the gradient at p itself (Bresenham.cpp:74-81).
        const float dx2 = float(gdx), dy2 = float(gdy);
        const float v = dx2 * dxRef + dy2 * dyRef;
        const int d = (v > 0.f) - (v < 0.f);
        dx = float(d) * dx2;
        dy = float(d) * dy2;
    }
    step();
    if (!inside(x, y)) return -1;
    if (idxmap[size_t(y) * W + x] >= 0) return idxmap[size_t(y) * W + x];
    while (n <= nmax) {
        step();
        if (!inside(x, y)) return -1;
        const int hit = idxmap[size_t(y) * W + x];
        if (hit >= 0) return hit;
        const int bx = y_major ? x : x - stpX;
        const int by = y_major ? y - stpY : y;
        if (!inside(bx, by)) return -1;
        const int hit2 = idxmap[size_t(by) * W + bx];
        if (hit2 >= 0) return hit2;
    }
    return -1;
}

// Vote.cpp:58-247.  `seeds_push` receives the seeds in the order the reference
// appends them (the voter that brings a point to minVotes); `seeds_sorted`
// applies Multiresolution.cpp:239-242 (std::sort by received votes, desc).
int vote(const uint8_t* edges, const int16_t* dxm, const int16_t* dym, int W, int H, const VoteParams& vp,
         int cap, int32_t* ex, int32_t* ey, int32_t* before, int32_t* after, int32_t* chosen_out, float* total_out,
         int32_t* nvotes, int32_t* is_max, float* flow_length, int32_t* voter_off, int32_t* voter_list,
         int32_t* seeds_push, int32_t* seeds_sorted, int32_t* n_seeds)
{
    std::vector<int32_t> idxmap(size_t(W) * H, -1);
    int E = 0;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
            if (edges[size_t(y) * W + x] == 255) {
                if (E >= cap) return -1;
                idxmap[size_t(y) * W + x] = E;
                ex[E] = x;
                ey[E] = y;
                ++E;
            }
    std::vector<float> gx(E), gy(E);
    for (int i = 0; i < E; ++i) {
        gx[i] = float(dxm[size_t(ey[i]) * W + ex[i]]);
        gy[i] = float(dym[size_t(ey[i]) * W + ex[i]]);
    }
    for (int i = 0; i < E; ++i) {
        const int gdx = dxm[size_t(ey[i]) * W + ex[i]], gdy = dym[size_t(ey[i]) * W + ex[i]];
        before[i] = gradient_walk(idxmap.data(), W, H, ex[i], ey[i], gdx, gdy, -1, vp.distSearch, vp.thrGradientMagInVote);
        after[i] = gradient_walk(idxmap.data(), W, H, ex[i], ey[i], gdx, gdy, +1, vp.distSearch, vp.thrGradientMagInVote);
    }
    auto dist = [&](int a, int b) {
        const int ddx = ex[b] - ex[a], ddy = ey[b] - ey[a];
        return std::sqrt(float(ddx * ddx) + float(ddy * ddy));
    };
    auto neg_dot = [&](int a, int b) { return -(gx[a] * gx[b] + gy[a] * gy[b]); };
    std::vector<std::vector<int32_t>> voters(E);
    std::vector<float> fl(E, 0.f);
    std::vector<int32_t> ismax(E, -1);
    std::vector<int32_t> seeds;
    const float ratio = vp.ratioVoting;
    auto ratio_ok = [&](const std::vector<float>& v) {
        int ok = 1;
        for (size_t i = 0; i < v.size(); ++i)
            for (size_t j = i + 1; j < v.size(); ++j)
                ok = (v[i] <= v[j] * ratio) && (v[j] <= v[i] * ratio) && ok;
        return ok;
    };
    for (int p = 0; p < E; ++p) {
        int current = before[p];
        int chosen = -1;
        std::vector<float> vDist;
        float total = 0.f;
        if (current >= 0 && neg_dot(p, current) >= vp.angleVoting) {
            float d = dist(p, current);
            vDist.push_back(d);
            total += d;
            for (int i = 1; i < vp.nCrowns; ++i) {
                chosen = -1;
                int target = after[current];
                if (target < 0) break;
                if (!(neg_dot(target, current) >= vp.angleVoting)) break;
                d = dist(target, current);
                vDist.push_back(d);
                total += d;
                int flag = 1;
                if (vDist.size() > 1) flag = ratio_ok(vDist);
                if (!flag) break;
                current = target;
                target = before[current];
                if (target < 0) break;
                if (!(neg_dot(target, current) >= vp.angleVoting)) break;
                d = dist(target, current);
                vDist.push_back(d);
                total += d;
                flag = flag && ratio_ok(vDist);
                if (!flag) break;
                current = target;
                chosen = current;
            }
        }
        if (chosen_out) chosen_out[p] = chosen;
        if (total_out) total_out[p] = chosen >= 0 ? total : 0.f;
        if (chosen >= 0) {
            voters[chosen].push_back(p);
            const float n = float(voters[chosen].size());
            fl[chosen] = (fl[chosen] * (n - 1.f) + total) / n;
            if (int(voters[chosen].size()) >= vp.minVotesToSelectCandidate) {
                if (ismax[chosen] == -1) seeds.push_back(chosen);
                ismax[chosen] = int(voters[chosen].size());
            }
        }
    }
    int off = 0;
    for (int i = 0; i < E; ++i) {
        nvotes[i] = int(voters[i].size());
        is_max[i] = ismax[i];
        flow_length[i] = fl[i];
        voter_off[i] = off;
        for (int v : voters[i]) voter_list[off++] = v;
    }
    voter_off[E] = off;
    for (size_t s = 0; s < seeds.size(); ++s) seeds_push[s] = seeds[s];
    std::vector<int32_t> sorted = seeds;
    if (sorted.size() > 1)
        std::sort(sorted.begin(), sorted.end(), [&](int a, int b) { return ismax[a] > ismax[b]; });
    for (size_t s = 0; s < sorted.size(); ++s) seeds_sorted[s] = sorted[s];
    *n_seeds = int(seeds.size());
    return E;
}

}  // namespace orc

// ------------------------------------------------------------- C entries --
extern "C" {

void orc_pyramid_down(const uint8_t* src, int sw, int sh, uint8_t* dst, int dw, int dh)
{
    orc::pyramid_down(src, sw, sh, dst, dw, dh);
}

void orc_derivatives(const uint8_t* src, int W, int H, int16_t* dx, int16_t* dy)
{
    orc::derivatives(src, W, H, dx, dy);
}

void orc_canny(const int16_t* dx, const int16_t* dy, int W, int H, float thrLow, float thrHigh, uint8_t* edges,
               uint8_t* nms_map)
{
    orc::canny(dx, dy, W, H, thrLow, thrHigh, edges, nms_map);
}

void orc_thin_lut(int pass, uint8_t* lut) { orc::thin_lut(pass, lut); }

void orc_thin(uint8_t* edges, int W, int H) { orc::thin(edges, W, H); }

int orc_vote(const uint8_t* edges, const int16_t* dx, const int16_t* dy, int W, int H, const orc_vote_params* p,
             int cap, int32_t* ex, int32_t* ey, int32_t* before, int32_t* after, int32_t* chosen, float* total,
             int32_t* nvotes, int32_t* is_max, float* flow_length, int32_t* voter_off, int32_t* voter_list,
             int32_t* seeds_push, int32_t* seeds_sorted, int32_t* n_seeds)
{
    orc::VoteParams vp{p->distSearch, p->thrGradientMagInVote, p->angleVoting, p->ratioVoting, p->nCrowns,
                       p->minVotesToSelectCandidate};
    return orc::vote(edges, dx, dy, W, H, vp, cap, ex, ey, before, after, chosen, total, nvotes, is_max, flow_length,
                     voter_off, voter_list, seeds_push, seeds_sorted, n_seeds);
}

// Whole image stage for one level: derivatives -> canny -> thin.
void orc_level(const uint8_t* src, int W, int H, float thrLow, float thrHigh, int16_t* dx, int16_t* dy,
               uint8_t* edges)
{
    orc::derivatives(src, W, H, dx, dy);
    orc::canny(dx, dy, W, H, thrLow, thrHigh, edges, nullptr);
    orc::thin(edges, W, H);
}

}  // extern "C"
