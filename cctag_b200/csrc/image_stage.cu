// Image stage of the CCTag hot path on sm_100a: pyramid, 9x9 DoG derivatives,
// Canny NMS + hysteresis, thinning, raster-order edge compaction, Bresenham
// gradient walk, vote, voter lists and seeds.  Every launch covers all pyramid
// levels at once (the block index is split into level and tile), no launch
// needs a host synchronisation, so a frame is one capturable launch sequence.
//
// Bit-exactness with the reference CPU path (file:line in the CCTag project):
//  * derivatives: same 72-tap FMA chain as cv::filter2D, cvRecode.cpp:74-92
//  * magnitude / NMS / hysteresis: cvRecode.cpp:174-409 (final edge set is the
//    8-connected components of NMS candidates that hold a strong pixel)
//  * thinning: thinning.cpp:12-51 (Lam-Lee-Suen tables, temp border = 0)
//  * edge order: raster order, Canny.cpp:15-31
//  * walk: Bresenham.cpp:18-209, vote: Vote.cpp:58-247 (no FMA contraction,
//    IEEE division and square root, same accumulation order)
#include <algorithm>
#include <cstdint>

#include "common.hpp"

namespace cctagb {

// kerneldX of cvRecode.cpp:74-83
__constant__ float cK[9][9] = {
    {-0.000000143284235f, -0.000003558691641f, -0.000028902492951f, -0.000064765993382f, 0.f, 0.000064765993382f, 0.000028902492951f, 0.000003558691641f, 0.000000143284235f},
    {-0.000004744922188f, -0.000117847682078f, -0.000957119116802f, -0.002144755142391f, 0.f, 0.002144755142391f, 0.000957119116802f, 0.000117847682078f, 0.000004744922188f},
    {-0.000057804985902f, -0.001435678675203f, -0.011660097860113f, -0.026128466569370f, 0.f, 0.026128466569370f, 0.011660097860113f, 0.001435678675203f, 0.000057804985902f},
    {-0.000259063973527f, -0.006434265427174f, -0.052256933138740f, -0.117099663048638f, 0.f, 0.117099663048638f, 0.052256933138740f, 0.006434265427174f, 0.000259063973527f},
    {-0.000427124283626f, -0.010608310271112f, -0.086157117207395f, -0.193064705260108f, 0.f, 0.193064705260108f, 0.086157117207395f, 0.010608310271112f, 0.000427124283626f},
    {-0.000259063973527f, -0.006434265427174f, -0.052256933138740f, -0.117099663048638f, 0.f, 0.117099663048638f, 0.052256933138740f, 0.006434265427174f, 0.000259063973527f},
    {-0.000057804985902f, -0.001435678675203f, -0.011660097860113f, -0.026128466569370f, 0.f, 0.026128466569370f, 0.011660097860113f, 0.001435678675203f, 0.000057804985902f},
    {-0.000004744922188f, -0.000117847682078f, -0.000957119116802f, -0.002144755142391f, 0.f, 0.002144755142391f, 0.000957119116802f, 0.000117847682078f, 0.000004744922188f},
    {-0.000000143284235f, -0.000003558691641f, -0.000028902492951f, -0.000064765993382f, 0.f, 0.000064765993382f, 0.000028902492951f, 0.000003558691641f, 0.000000143284235f}};

// Lam-Lee-Suen sub-iteration tables as bitsets (index = the 3x3 neighbourhood
// with the weights of thinning.cpp: (x-1,y-1)=1 ... (x+1,y+1)=256): bit set
// where the pixel stays.  Derived from the thinning conditions at compile time.
struct ThinTables {
    uint32_t bits[2][16];
};
constexpr ThinTables make_thin_tables()
{
    ThinTables t{};
    for (int pass = 1; pass <= 2; ++pass)
        for (int idx = 0; idx < 512; ++idx) {
            if (!(idx & 16)) continue;
            int x[10] = {0, (idx & 128) ? 1 : 0, (idx & 64) ? 1 : 0, (idx & 8) ? 1 : 0, (idx & 1) ? 1 : 0,
                         (idx & 2) ? 1 : 0, (idx & 4) ? 1 : 0, (idx & 32) ? 1 : 0, (idx & 256) ? 1 : 0, 0};
            x[9] = x[1];
            int xh = 0, n1 = 0, n2 = 0;
            for (int i = 1; i <= 4; ++i) {
                xh += (x[2 * i - 1] == 0 && (x[2 * i] == 1 || x[2 * i + 1] == 1)) ? 1 : 0;
                n1 += x[2 * i - 1] | x[2 * i];
                n2 += x[2 * i] | x[2 * i + 1];
            }
            const int mn = n1 < n2 ? n1 : n2;
            const bool g1 = xh == 1, g2 = mn >= 2 && mn <= 3;
            const bool g3 = pass == 1 ? (((x[2] | x[3] | (1 - x[8])) & x[1]) == 0)
                                      : (((x[6] | x[7] | (1 - x[4])) & x[5]) == 0);
            if (!(g1 && g2 && g3)) t.bits[pass - 1][idx >> 5] |= 1u << (idx & 31);
        }
    return t;
}
__constant__ ThinTables cThinTab = make_thin_tables();

// ------------------------------------------------------------------ utils --
__device__ __forceinline__ int level_of_block(const Levels& lv, int b, int LevelView::*tiles, int& local)
{
    int l = 0;
    while (l < lv.n - 1 && b >= lv.l[l].*tiles) {
        b -= lv.l[l].*tiles;
        ++l;
    }
    local = b;
    return l;
}

__device__ __forceinline__ int16_t sat_round16(float s)
{
    float r = rintf(s);
    r = fminf(32767.f, fmaxf(-32768.f, r));
    return int16_t(r);
}

// Gradient magnitude, rintf(sqrtf(dx^2 + dy^2)) as cvRecode.cpp:200-211.
__device__ __forceinline__ int magnitude(int16_t gx, int16_t gy)
{
    const float fx = float(gx), fy = float(gy);
    return int(rintf(__fsqrt_rn(__fadd_rn(__fmul_rn(fx, fx), __fmul_rn(fy, fy)))));
}

__device__ __forceinline__ bool edge_bit(const LevelView& L, int x, int y)
{
    return (L.bitmap[size_t(y) * L.WW + (x >> 5)] >> (x & 31)) & 1u;
}

// ---------------------------------------------------------------- pyramid --
// ImagePyramid.cpp:23-52, Level.cpp:57-81.  Exact 2x reductions (every level
// of a frame whose sides are multiples of 8) are the rounded 2x2 mean, as
// cv::resize's area fast path; one thread builds an 8x8 block of level 0 into
// levels 1..3.
__global__ void k_pyramid3(Levels lv)
{
    const int base = blockIdx.z * (lv.n / lv.frames);  // this frame's level 0
    const LevelView& L0 = lv.l[base];
    const int W3 = L0.W >> 3, H3 = L0.H >> 3;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W3 || y >= H3) return;
    uint32_t p[8][8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const uint2 v = *reinterpret_cast<const uint2*>(L0.src + size_t(8 * y + r) * L0.W + 8 * x);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            p[r][c] = (v.x >> (8 * c)) & 0xff;
            p[r][c + 4] = (v.y >> (8 * c)) & 0xff;
        }
    }
    uint32_t q1[4][4], q2[2][2];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c)
            q1[r][c] = (p[2 * r][2 * c] + p[2 * r][2 * c + 1] + p[2 * r + 1][2 * c] + p[2 * r + 1][2 * c + 1] + 2) >> 2;
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int c = 0; c < 2; ++c)
            q2[r][c] = (q1[2 * r][2 * c] + q1[2 * r][2 * c + 1] + q1[2 * r + 1][2 * c] + q1[2 * r + 1][2 * c + 1] + 2) >> 2;
    const uint32_t q3 = (q2[0][0] + q2[0][1] + q2[1][0] + q2[1][1] + 2) >> 2;
    const LevelView& L1 = lv.l[base + 1];
    const LevelView& L2 = lv.l[base + 2];
    const LevelView& L3 = lv.l[base + 3];
#pragma unroll
    for (int r = 0; r < 4; ++r)
        *reinterpret_cast<uint32_t*>(L1.src + size_t(4 * y + r) * L1.W + 4 * x) =
            q1[r][0] | (q1[r][1] << 8) | (q1[r][2] << 16) | (q1[r][3] << 24);
#pragma unroll
    for (int r = 0; r < 2; ++r)
        *reinterpret_cast<uint16_t*>(L2.src + size_t(2 * y + r) * L2.W + 2 * x) = uint16_t(q2[r][0] | (q2[r][1] << 8));
    L3.src[size_t(y) * L3.W + x] = uint8_t(q3);
}

// One level from the previous one, any size: exact 2x -> 2x2 rounded mean,
// otherwise cv::resize INTER_LINEAR fixed point (11-bit coefficients and the
// vectorised vertical pass of OpenCV: 16-bit high products, rounding shift 2).
__device__ __forceinline__ void resize_coef(int d, int dn, int sn, int& s, int& c0)
{
    const double scale = double(sn) / dn;
    float f = float((d + 0.5) * scale - 0.5);
    s = int(floorf(f));
    f -= float(s);
    if (s < 0) { f = 0.f; s = 0; }
    if (s >= sn - 1) { f = 0.f; s = sn - 1; }
    c0 = int(rintf(__fmul_rn(1.f - f, 2048.f)));
}

__global__ void k_resize_level(const uint8_t* __restrict__ src, int sw, int sh, uint8_t* __restrict__ dst, int dw, int dh)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= dw || y >= dh) return;
    if (sw == 2 * dw && sh == 2 * dh) {
        const uint8_t* p = src + size_t(2 * y) * sw + 2 * x;
        dst[size_t(y) * dw + x] = uint8_t((p[0] + p[1] + p[sw] + p[sw + 1] + 2) >> 2);
        return;
    }
    int sx, cx0, sy, cy0;
    resize_coef(x, dw, sw, sx, cx0);
    resize_coef(y, dh, sh, sy, cy0);
    const int cx1 = 2048 - cx0, cy1 = 2048 - cy0;
    const int sx1 = min(sx + 1, sw - 1), sy1 = min(sy + 1, sh - 1);
    const int r0 = src[size_t(sy) * sw + sx] * cx0 + src[size_t(sy) * sw + sx1] * cx1;
    const int r1 = src[size_t(sy1) * sw + sx] * cx0 + src[size_t(sy1) * sw + sx1] * cx1;
    int v = ((((r0 >> 4) * cy0) >> 16) + (((r1 >> 4) * cy1) >> 16) + 2) >> 2;
    dst[size_t(y) * dw + x] = uint8_t(min(255, max(0, v)));
}

// --------------------------------------------- derivatives + magnitude + NMS --
// Output tile 30x30.  Derivatives are computed on the 32x32 region around it
// (NMS needs the magnitude of the 8 neighbours) from a 40x40 source region.
// Thread t owns derivative column t&31 and the 8-row strip t>>5: it walks the
// 16 source rows of its strip once and feeds each loaded row to every output
// row whose 9x9 window covers it, which keeps each pixel's taps in the
// reference's row-major order.
constexpr int kNmsT = 30;      // output tile side
constexpr int kNmsD = 32;      // derivative region side
constexpr int kNmsS = 40;      // source region side

__global__ void __launch_bounds__(128) k_deriv_nms(Levels lv, VoteParamsDev vp, int write_derivs)
{
    __shared__ float s_src[kNmsS][kNmsS];
    __shared__ int16_t s_dx[kNmsD][kNmsD];
    __shared__ int16_t s_dy[kNmsD][kNmsD];
    __shared__ int s_mag[kNmsD][kNmsD + 1];

    int tile;
    const int l = level_of_block(lv, blockIdx.x, &LevelView::nms_tiles, tile);
    const LevelView& L = lv.l[l];
    const int W = L.W, H = L.H;
    const int x0 = (tile % L.nms_tx) * kNmsT;
    const int y0 = (tile / L.nms_tx) * kNmsT;
    const int t = threadIdx.x;

    if (write_derivs) {
        for (int i = t; i < kNmsS * kNmsS; i += 128) {
            const int sr = i / kNmsS, sc = i % kNmsS;
            const int yy = min(H - 1, max(0, y0 - 5 + sr));
            const int xx = min(W - 1, max(0, x0 - 5 + sc));
            s_src[sr][sc] = float(L.src[size_t(yy) * W + xx]);
        }
        __syncthreads();
        const int c = t & 31;
        const int r0 = (t >> 5) * 8;
        float ax[8], ay[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) { ax[r] = 0.f; ay[r] = 0.f; }
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            float v[9];
#pragma unroll
            for (int j = 0; j < 9; ++j) v[j] = s_src[r0 + q][c + j];
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const int i = q - r;
                if (i < 0 || i > 8) continue;
#pragma unroll
                for (int j = 0; j < 9; ++j) {
                    if (j != 4) ax[r] = __fmaf_rn(cK[i][j], v[j], ax[r]);
                    if (i != 4) ay[r] = __fmaf_rn(cK[j][i], v[j], ay[r]);
                }
            }
        }
        // derivatives and magnitude of this thread's 8 pixels
        const int xx = x0 - 1 + c;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int16_t gx = sat_round16(ax[r]), gy = sat_round16(ay[r]);
            s_dx[r0 + r][c] = gx;
            s_dy[r0 + r][c] = gy;
            const int yy = y0 - 1 + r0 + r;
            s_mag[r0 + r][c] = xx >= 0 && xx < W && yy >= 0 && yy < H ? magnitude(gx, gy) : 0;
        }
    } else {
        // Derivatives supplied by the caller: load them with the same halo.
        for (int i = t; i < kNmsD * kNmsD; i += 128) {
            const int r = i / kNmsD, c = i % kNmsD;
            const int yy = y0 - 1 + r, xx = x0 - 1 + c;
            int16_t gx = 0, gy = 0;
            if (xx >= 0 && xx < W && yy >= 0 && yy < H) {
                gx = L.dx[size_t(yy) * W + xx];
                gy = L.dy[size_t(yy) * W + xx];
            }
            s_dx[r][c] = gx;
            s_dy[r][c] = gy;
            s_mag[r][c] = xx >= 0 && xx < W && yy >= 0 && yy < H ? magnitude(gx, gy) : 0;
        }
    }
    __syncthreads();
    // NMS, cvRecode.cpp:258-323: lane ox of warp w takes column ox of rows
    // w, w + 4, ...
    const int TG22 = int(0.4142135623730950488016887242097 * (1 << 15) + 0.5);
    const int ox = t & 31;
    for (int oy = t >> 5; oy < kNmsT; oy += 4) {
        const int x = x0 + ox, y = y0 + oy;
        if (ox >= kNmsT || x >= W || y >= H) continue;
        const int r = oy + 1, c = ox + 1;
        int gx = s_dx[r][c], gy = s_dy[r][c];
        const int s = gx ^ gy;
        const int m = s_mag[r][c];
        gx = abs(gx);
        gy = abs(gy);
        bool is_max = false;
        if (m > vp.low) {
            const int tg22x = gx * TG22;
            const int tg67x = tg22x + ((gx + gx) << 15);
            const int gy15 = gy << 15;
            if (gy15 < tg22x) {
                is_max = m > s_mag[r][c - 1] && m >= s_mag[r][c + 1];
            } else if (gy15 > tg67x) {
                is_max = m > s_mag[r - 1][c] && m >= s_mag[r + 1][c];
            } else {
                const int sg = s < 0 ? -1 : 1;
                is_max = m > s_mag[r - 1][c - sg] && m > s_mag[r + 1][c + sg];
            }
        }
        const size_t p = size_t(y) * W + x;
        const uint8_t cls = is_max ? (m > vp.high ? 2 : 1) : 0;
        L.map[p] = cls;
        if (write_derivs) {
            L.dx[p] = s_dx[r][c];
            L.dy[p] = s_dy[r][c];
        }
    }
}

// ------------------------------------------------------------- hysteresis --
// The reference's stack hysteresis (cvRecode.cpp:362-394) keeps exactly the
// 8-connected components of NMS candidates that contain a strong pixel.  Here
// the image is cut into 32x32 tiles, one warp each, lane r holding row r of
// the tile as 32-bit masks (candidates C, strong S):
//  1. k_hyst_tiles: the closure of S within C inside the tile (R, bit-parallel
//     dilation: rows shifted by one bit, neighbour rows by shuffles), and the
//     components that touch the tile border, one flood fill each, labelled
//     per border position, with whether they hold a strong pixel;
//  2. k_hyst_unions / k_hyst_roots: those border components joined across
//     tile borders by a lock-free union-find over (tile, component) ids
//     (parent <= self, roots linked by atomicMin, so any schedule gives the
//     same sets), and each set marked strong at its root if a member is;
//  3. k_hyst_final: per tile, R plus the border pixels of strong sets, closed
//     within C again: the hysteresis result H, one bit per pixel.
// A pixel is in H exactly when its component holds a strong pixel: a path to
// one either stays in the tile (step 1) or leaves it through a border pixel
// of its tile component, whose set is then strong (steps 2-3).
constexpr int kUfCap = 1 << 22;
constexpr int kTile = 32;          // hysteresis tile side
constexpr int kBorderPos = 128;    // border positions of a tile (4 x 32, some unused)
constexpr int kTileComps = 64;     // border components per tile (at most 62: runs on a 124-pixel cycle)

__device__ __forceinline__ int uf_find(const int32_t* L, int p)
{
    int q = *(volatile const int32_t*)&L[p];
    int guard = 0;
    while (q != p && guard++ < kUfCap) {
        p = q;
        q = *(volatile const int32_t*)&L[p];
    }
    return p;
}

__device__ __forceinline__ void uf_union(int32_t* L, int a, int b, int32_t* err)
{
    for (int it = 0; it < kUfCap; ++it) {
        a = uf_find(L, a);
        b = uf_find(L, b);
        if (a == b) return;
        if (a > b) { const int tmp = a; a = b; b = tmp; }
        const int old = atomicMin(&L[b], a);
        if (old == b) return;
        b = old;
    }
    atomicOr(err, kErrUnionFind);
}

// The closure of `seed` (a subset of c) within c, 8-connected, over the
// warp's tile (lane = row).  Each round adds a pixel or ends the loop, so it
// ends within the tile's 1024 pixels.
__device__ __forceinline__ uint32_t tile_closure(uint32_t seed, uint32_t c, int lane)
{
    uint32_t r = seed & c;
    for (int it = 0; it <= kTile * kTile; ++it) {
        uint32_t up = __shfl_up_sync(0xffffffffu, r, 1);
        uint32_t dn = __shfl_down_sync(0xffffffffu, r, 1);
        if (lane == 0) up = 0u;
        if (lane == kTile - 1) dn = 0u;
        const uint32_t v = r | up | dn;
        const uint32_t nb = (v | (v << 1) | (v >> 1)) & c;
        if (!__any_sync(0xffffffffu, nb != r)) break;
        r = nb;
    }
    return r;
}

// Border position of tile pixel (x, y) (tile coordinates), -1 inside:
// row 0 -> x, row 31 -> 32 + x, column 0 -> 64 + y, column 31 -> 96 + y.
__device__ __forceinline__ int border_pos(int x, int y)
{
    if (y == 0) return x;
    if (y == kTile - 1) return kTile + x;
    if (x == 0) return 2 * kTile + y;
    if (x == kTile - 1) return 3 * kTile + y;
    return -1;
}

// Warp w of the launch: its level and tile (tiles of all levels back to back).
__device__ __forceinline__ int level_of_tile(const Levels& lv, int g, int& tile)
{
    int l = 0;
    while (l < lv.n - 1 && g >= lv.l[l].uf_tiles) {
        g -= lv.l[l].uf_tiles;
        ++l;
    }
    tile = g;
    return l;
}

__device__ __forceinline__ uint32_t* plane_c(const LevelView& L) { return L.hbits; }
__device__ __forceinline__ uint32_t* plane_r(const LevelView& L) { return L.hbits + size_t(L.WW) * L.H; }
__device__ __forceinline__ uint32_t* plane_h(const LevelView& L) { return L.hbits + 2 * size_t(L.WW) * L.H; }

constexpr int kHystWarps = 4;

__global__ void __launch_bounds__(32 * kHystWarps) k_hyst_tiles(Levels lv, int total_tiles)
{
    __shared__ uint8_t s_lab[kHystWarps][kBorderPos];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = blockIdx.x * kHystWarps + warp;
    if (g >= total_tiles) return;
    int tile;
    const int l = level_of_tile(lv, g, tile);
    const LevelView& L = lv.l[l];
    const int tx = tile % L.uf_tx, ty = tile / L.uf_tx;
    const int x0 = tx * kTile, y0 = ty * kTile;
    const int rows = min(kTile, L.H - y0), cols = min(kTile, L.W - x0);
    // row masks of the tile: lane r keeps row r
    uint32_t c = 0u, st = 0u;
#pragma unroll 4
    for (int r = 0; r < kTile; ++r) {
        uint8_t v = 0;
        if (r < rows && lane < cols) v = L.map[size_t(y0 + r) * L.W + x0 + lane];
        const uint32_t cm = __ballot_sync(0xffffffffu, v != 0), sm = __ballot_sync(0xffffffffu, v == 2);
        if (lane == r) {
            c = cm;
            st = sm;
        }
    }
    const uint32_t R = tile_closure(st, c, lane);
    if (lane < rows) {
        const size_t w = size_t(y0 + lane) * L.WW + tx;
        plane_c(L)[w] = c;
        plane_r(L)[w] = R;
    }
    for (int i = lane; i < kBorderPos; i += 32) s_lab[warp][i] = 0xff;
    __syncwarp();
    // border components, one flood fill each from an unlabelled border pixel
    const uint32_t bmask = (lane == 0 || lane == kTile - 1) ? c : (c & (1u | (1u << (kTile - 1))));
    uint32_t unl = bmask;
    uint64_t strong = 0ull;
    int ncomp = 0;
    while (__any_sync(0xffffffffu, unl != 0u)) {
        const uint32_t have = __ballot_sync(0xffffffffu, unl != 0u);
        const int sl = __ffs(have) - 1;
        const uint32_t sb = __shfl_sync(0xffffffffu, unl & (0u - unl), sl);
        const uint32_t m = tile_closure(lane == sl ? sb : 0u, c, lane);
        if (ncomp >= kTileComps) {  // cannot happen (<= 62 components); flagged, not silent
            if (lane == 0) atomicOr(&lv.cnt[l].err, kErrUnionFind);
            break;
        }
        if (__any_sync(0xffffffffu, (m & R) != 0u)) strong |= 1ull << ncomp;
        uint32_t bm = m & bmask;
        while (bm) {
            const int b = __ffs(bm) - 1;
            bm &= bm - 1;
            s_lab[warp][border_pos(b, lane)] = uint8_t(ncomp);
        }
        unl &= ~m;
        ++ncomp;
    }
    __syncwarp();
    const size_t base = size_t(tile) * kTileComps;
    for (int k = lane; k < kTileComps; k += 32) {
        L.tcomp[base + k] = int32_t(base + k);
        L.tflag[base + k] = (k < ncomp && ((strong >> k) & 1ull)) ? 1 : 0;
    }
    for (int i = lane; i < kBorderPos; i += 32) L.blab[size_t(tile) * kBorderPos + i] = s_lab[warp][i];
}

// The (tile, component) id of border pixel (x, y) of the level.
__device__ __forceinline__ int border_comp(const LevelView& L, int x, int y)
{
    const int tile = (y / kTile) * L.uf_tx + x / kTile;
    const int lab = L.blab[size_t(tile) * kBorderPos + border_pos(x % kTile, y % kTile)];
    return tile * kTileComps + lab;
}

__device__ __forceinline__ bool cand_bit(const LevelView& L, int x, int y)
{
    return (plane_c(L)[size_t(y) * L.WW + (x >> 5)] >> (x & 31)) & 1u;
}

// Unions across tile borders: the first row of a tile with the row above
// (three neighbours each), the first column with the column to the left.
// Every 8-neighbour pair that straddles a tile border meets here.
__global__ void __launch_bounds__(64) k_hyst_unions(Levels lv)
{
    int tile;
    const int l = level_of_block(lv, blockIdx.x, &LevelView::uf_tiles, tile);
    const LevelView& L = lv.l[l];
    const int x0 = (tile % L.uf_tx) * kTile, y0 = (tile / L.uf_tx) * kTile;
    const int t = threadIdx.x;
    const bool row = t < 32;
    const int x = row ? x0 + t : x0, y = row ? y0 : y0 + (t - 32);
    if (x >= L.W || y >= L.H) return;
    if (row ? y == 0 : x == 0) return;
    if (!cand_bit(L, x, y)) return;
    int32_t* err = &lv.cnt[l].err;
    const int a = border_comp(L, x, y);
    for (int d = -1; d <= 1; ++d) {
        const int qx = row ? x + d : x - 1, qy = row ? y - 1 : y + d;
        if (qx < 0 || qx >= L.W || qy < 0 || qy >= L.H) continue;
        if (qx / kTile == x / kTile && qy / kTile == y / kTile) continue;  // same tile: joined in step 1
        if (cand_bit(L, qx, qy)) uf_union(L.tcomp, a, border_comp(L, qx, qy), err);
    }
}

// Each set with a strong member is marked strong at its root.
__global__ void __launch_bounds__(kTileComps) k_hyst_roots(Levels lv)
{
    int tile;
    const int l = level_of_block(lv, blockIdx.x, &LevelView::uf_tiles, tile);
    const LevelView& L = lv.l[l];
    const int id = tile * kTileComps + threadIdx.x;
    if (L.tflag[id] & 1) atomicOr(&L.tflag[uf_find(L.tcomp, id)], 2);
}

__global__ void __launch_bounds__(32 * kHystWarps) k_hyst_final(Levels lv, int total_tiles)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = blockIdx.x * kHystWarps + warp;
    if (g >= total_tiles) return;
    int tile;
    const int l = level_of_tile(lv, g, tile);
    const LevelView& L = lv.l[l];
    const int tx = tile % L.uf_tx, ty = tile / L.uf_tx;
    const int y0 = ty * kTile;
    const int rows = min(kTile, L.H - y0);
    uint32_t c = 0u, R = 0u;
    if (lane < rows) {
        const size_t w = size_t(y0 + lane) * L.WW + tx;
        c = plane_c(L)[w];
        R = plane_r(L)[w];
    }
    // which of the tile's components belong to a strong set (two per lane,
    // the finds side by side; unused components are their own roots, flag 0)
    const int base = tile * kTileComps;
    const bool s0 = L.tflag[uf_find(L.tcomp, base + lane)] & 2;
    const bool s1 = L.tflag[uf_find(L.tcomp, base + 32 + lane)] & 2;
    const uint64_t strongSets =
        uint64_t(__ballot_sync(0xffffffffu, s0)) | (uint64_t(__ballot_sync(0xffffffffu, s1)) << 32);
    // border pixels of those components seed the closure
    __shared__ uint32_t s_lab[kHystWarps][kBorderPos / 4];
    s_lab[warp][lane] = reinterpret_cast<const uint32_t*>(L.blab + size_t(tile) * kBorderPos)[lane];
    __syncwarp();
    const uint8_t* lab = reinterpret_cast<const uint8_t*>(s_lab[warp]);
    const uint32_t bmask = (lane == 0 || lane == kTile - 1) ? c : (c & (1u | (1u << (kTile - 1))));
    uint32_t seed = 0u, bm = strongSets ? (bmask & ~R) : 0u;
    while (bm) {
        const int b = __ffs(bm) - 1;
        bm &= bm - 1;
        if ((strongSets >> lab[border_pos(b, lane)]) & 1ull) seed |= 1u << b;
    }
    const uint32_t H = __any_sync(0xffffffffu, seed != 0u) ? tile_closure(R | seed, c, lane) : R;
    if (lane < rows) plane_h(L)[size_t(y0 + lane) * L.WW + tx] = H;
}

// ------------------------------------------------ final edges + thinning --
// thin() (thinning.cpp:12-51): two Lam-Lee-Suen sub-iterations over the
// hysteresis result, interior pixels only, the image border keeping its
// Canny value.  Evaluated bit-parallel: a warp takes one 32-pixel word column
// and 28 output rows, lane r holding row y0 - 2 + r as a 64-bit window
// (x0 - 16 .. x0 + 47) built from three words of the H plane.  The neighbour
// masks are the window shifted by one bit and the rows above and below
// (shuffles); each sub-iteration's "delete" condition is the conjunction of
// G1 (exactly one of four 0 -> 1 transitions), G2 (2 <= min(n1, n2) <= 3) and
// the sub-iteration's G3, in bitwise form -- the same function as the
// reference's 512-entry tables (checked entry by entry in the tests).  Rows
// and columns two away from the output are enough for the two passes.
constexpr int kThinRows = 28;
constexpr int kThinWarps = 4;

__device__ __forceinline__ uint64_t atl2(uint64_t a, uint64_t b, uint64_t c, uint64_t d)
{
    return ((a | b) & (c | d)) | (a & b) | (c & d);
}

// Pixels of plane P that one sub-iteration keeps (pass 1 or 2), as a mask;
// up / dn are the rows above and below.
__device__ __forceinline__ uint64_t thin_keep(uint64_t P, uint64_t up, uint64_t dn, int pass)
{
    const uint64_t x1 = P >> 1, x2 = up >> 1, x3 = up, x4 = up << 1;  // E, NE, N, NW
    const uint64_t x5 = P << 1, x6 = dn << 1, x7 = dn, x8 = dn >> 1;  // W, SW, S, SE
    const uint64_t b1 = ~x1 & (x2 | x3), b2 = ~x3 & (x4 | x5), b3 = ~x5 & (x6 | x7), b4 = ~x7 & (x8 | x1);
    const uint64_t g1 = (b1 | b2 | b3 | b4) & ~atl2(b1, b2, b3, b4);
    const uint64_t a1 = x1 | x2, a2 = x3 | x4, a3 = x5 | x6, a4 = x7 | x8;
    const uint64_t c1 = x2 | x3, c2 = x4 | x5, c3 = x6 | x7, c4 = x8 | x1;
    const uint64_t g2 = atl2(a1, a2, a3, a4) & atl2(c1, c2, c3, c4) & ~((a1 & a2 & a3 & a4) & (c1 & c2 & c3 & c4));
    const uint64_t g3 = pass == 1 ? ~((x2 | x3 | ~x8) & x1) : ~((x6 | x7 | ~x4) & x5);
    return P & ~(g1 & g2 & g3);
}

// Bits of the window (bit i = column x0 - 16 + i) whose column lies in [lo, hi].
__device__ __forceinline__ uint64_t col_range(int x0, int lo, int hi)
{
    const int a = max(lo - (x0 - 16), 0), b = min(hi - (x0 - 16), 63);
    if (b < a) return 0ull;
    const uint64_t upto = b == 63 ? ~0ull : ((1ull << (b + 1)) - 1ull);
    return upto & ~((1ull << a) - 1ull);
}

__global__ void __launch_bounds__(32 * kThinWarps) k_final_thin(Levels lv, int total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int g = blockIdx.x * kThinWarps + warp;
    if (g >= total) return;
    int l = 0;
    while (l < lv.n - 1 && g >= lv.l[l].thin_tiles) {
        g -= lv.l[l].thin_tiles;
        ++l;
    }
    const LevelView& L = lv.l[l];
    const int W = L.W, H = L.H, WW = L.WW;
    const int wx = g % WW, y0 = (g / WW) * kThinRows;
    const int x0 = wx * 32;
    const int y = y0 - 2 + lane;
    uint64_t P = 0ull;
    if (y >= 0 && y < H) {
        const uint32_t* row = plane_h(L) + size_t(y) * WW;
        const uint32_t wl = wx > 0 ? row[wx - 1] : 0u, wc = row[wx], wr = wx + 1 < WW ? row[wx + 1] : 0u;
        P = uint64_t((wl >> 16) | (wc << 16)) | (uint64_t((wc >> 16) | (wr << 16)) << 32);
    }
    const bool rowInterior = y >= 1 && y <= H - 2;
    const uint64_t interior = rowInterior ? col_range(x0, 1, W - 2) : 0ull;
    uint64_t up = __shfl_up_sync(0xffffffffu, P, 1), dn = __shfl_down_sync(0xffffffffu, P, 1);
    const uint64_t T = thin_keep(P, up, dn, 1) & interior;
    up = __shfl_up_sync(0xffffffffu, T, 1);
    dn = __shfl_down_sync(0xffffffffu, T, 1);
    const uint64_t inImage = (y >= 0 && y < H) ? col_range(x0, 0, W - 1) : 0ull;
    const uint64_t out = (thin_keep(T, up, dn, 2) & interior) | (P & inImage & ~interior);
    if (lane >= 2 && lane < 2 + kThinRows && y < H) {
        const uint32_t word = uint32_t(out >> 16);
        L.bitmap[size_t(y) * WW + wx] = word;
        if (word) atomicAdd(&L.row_count[y], __popc(word));
    }
}

// ------------------------------------------------------------------ scans --
__device__ __forceinline__ int warp_incl_scan(int v)
{
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int n = __shfl_up_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) >= o) v += n;
    }
    return v;
}

// Exclusive block scan (blockDim.x multiple of 32, <= 1024); returns the block total in *total.
__device__ __forceinline__ int block_excl_scan(int v, int* s_warp, int* total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int inc = warp_incl_scan(v);
    if (lane == 31) s_warp[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        const int w = lane < nw ? s_warp[lane] : 0;
        const int wi = warp_incl_scan(w);
        if (lane < nw) s_warp[lane] = wi - w;
        if (lane == nw - 1) s_warp[32] = wi;
    }
    __syncthreads();
    const int res = inc - v + s_warp[wid];
    *total = s_warp[32];
    __syncthreads();
    return res;
}

// One block per level: row_off = exclusive scan of row_count; E clamped to the
// capacity (overflow flagged); row_count is cleared for the next frame.
__global__ void __launch_bounds__(1024) k_row_scan(Levels lv)
{
    __shared__ int s_warp[33];
    const int l = blockIdx.x;
    const LevelView& L = lv.l[l];
    int carry = 0;
    for (int base = 0; base < L.H; base += 1024) {
        const int i = base + threadIdx.x;
        const int v = i < L.H ? L.row_count[i] : 0;
        int total;
        const int ex = block_excl_scan(v, s_warp, &total);
        if (i < L.H) {
            L.row_off[i] = carry + ex;
            L.row_count[i] = 0;
        }
        carry += total;
    }
    if (threadIdx.x == 0) {
        L.row_off[L.H] = carry;
        int E = carry;
        if (E > L.cap) {
            atomicOr(&lv.cnt[l].err, kErrEdgeOverflow);
            E = L.cap;
        }
        lv.cnt[l].E = E;
    }
}

// One block (4 warps) per image row: raster-order edge list, per-point state
// reset, and per bitmap word the word with the index of its first edge point
// (an edge pixel's index is that plus the word's set bits below it).
// EdgePointCollection::add_point, Types.cpp:40-61.
__global__ void __launch_bounds__(128) k_emit(Levels lv, int rows_total)
{
    __shared__ int s_warp[4];
    int y = blockIdx.x, l = 0;
    while (l < lv.n - 1 && y >= lv.l[l].H) { y -= lv.l[l].H; ++l; }
    const LevelView& L = lv.l[l];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int per = (L.WW + 3) / 4;
    const int w0 = wid * per, w1 = min(L.WW, w0 + per);
    const uint32_t* row = L.bitmap + size_t(y) * L.WW;
    int cnt = 0;
    for (int w = w0 + lane; w < w1; w += 32) cnt += __popc(row[w]);
#pragma unroll
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0) s_warp[wid] = cnt;
    __syncthreads();
    int base = L.row_off[y];
    for (int k = 0; k < wid; ++k) base += s_warp[k];
    uint2* bi = L.bitidx + size_t(y) * L.WW;
    for (int w = w0; w < w1; ++w) {
        const uint32_t m = row[w];
        if (lane == 0) bi[w] = make_uint2(m, uint32_t(base));
        if (!m) continue;
        if ((m >> lane) & 1u) {
            const int idx = base + __popc(m & ((1u << lane) - 1u));
            if (idx < L.cap) {
                const int x = (w << 5) + lane;
                const size_t p = size_t(y) * L.W + x;
                L.exy[idx] = x | (y << 16);
                L.grad[idx] = int32_t(uint16_t(L.dx[p])) | (int32_t(L.dy[p]) << 16);
                L.nvotes[idx] = 0;
                L.fill[idx] = 0;
            }
        }
        base += __popc(m);
    }
}

// ------------------------------------------------------ gradient walk --
// Bresenham.cpp:18-209: from an edge point, follow the gradient (dir = -1
// backward, +1 forward) for up to distSearch steps and return the index of the
// first edge point met, or -1.  Walk lengths spread widely (most stop within
// two or three steps, a few run the full distance), so a warp does not run
// one walk per lane to the end of its longest: each lane takes the next walk
// of the warp's chunk as soon as its current one stops.  One iteration of the
// loop below is kWalkAhead steps of a lane's walk, with the probes the
// reference makes after each step, all loaded before the first is tested; the
// steps and probes of every walk are those of the reference in the same order
// (steps past the walk's end are computed and dropped), so the results do not
// depend on the schedule.
constexpr int kWalkWarps = 8;
constexpr int kWalkChunk = 512;  // walks (two per point) a warp takes at once, at most
// steps a lane takes per iteration (16-frame C2 launch: 2 steps 0.50 ms, 3 steps
// 0.52 ms; with the steps re-derived per step, 1 step 0.71 ms, 4 steps 0.69 ms,
// 8 steps 0.92 ms: more lookahead costs occupancy)
constexpr int kWalkAhead = 2;

__device__ __forceinline__ int sgn_i(int v) { return (v > 0) - (v < 0); }

__global__ void __launch_bounds__(32 * kWalkWarps) k_walk(Levels lv, VoteParamsDev vp)
{
    __shared__ int s_xy[kWalkWarps][kWalkChunk / 2];
    __shared__ int s_g[kWalkWarps][kWalkChunk / 2];
    __shared__ float s_a[kWalkWarps][kWalkChunk / 2];
    __shared__ int s_res[kWalkWarps][kWalkChunk];
    const unsigned kAll = 0xffffffffu;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1u;
    const int gw = blockIdx.x * kWalkWarps + wid, NW = gridDim.x * kWalkWarps;
    const int nmax = vp.distSearch;
    // chunk size: the launch's walks spread over its warps (a multiple of 32,
    // 32 .. kWalkChunk), the same in every block
    long long walks = 0;
    for (int l = 0; l < lv.n; ++l) walks += 2LL * lv.cnt[l].E;
    long long per = (walks / NW + 31) / 32 * 32;
    const int chunk = per < 32 ? 32 : per > kWalkChunk ? kWalkChunk : int(per);
    int first = 0;  // global number of the level's first chunk
    for (int l = 0; l < lv.n; ++l) {
        const LevelView& L = lv.l[l];
        const int E = lv.cnt[l].E;
        const int W = L.W, H = L.H, WW = L.WW;
        const int nch = (2 * E + chunk - 1) / chunk;
        int c = (gw - first % NW + NW) % NW;
        first += nch;
        for (; c < nch; c += NW) {
            const int t0 = c * chunk, t1 = min(2 * E, t0 + chunk);
            const int p0 = t0 >> 1, np = (t1 - t0) >> 1;
            // the chunk's points, |dmin / dmaj| per point (the same for both
            // directions) and the major and minor steps of the +1 direction,
            // (x, y) components packed as value + 1 in 2 bits each (the -1
            // direction's are their negatives)
            for (int i = lane; i < np; i += 32) {
                const int xy = L.exy[p0 + i], g = L.grad[p0 + i];
                const int gxi = int16_t(g & 0xffff), gyi = g >> 16;
                const float gx = float(gxi), gy = float(gyi);
                const bool ym = fabsf(gy) > fabsf(gx);
                const int smaj = sgn_i(ym ? gyi : gxi), smin = sgn_i(ym ? gxi : gyi);
                s_xy[wid][i] = xy;
                s_g[wid][i] = ((ym ? 0 : smaj) + 1) | ((ym ? smaj : 0) + 1) << 2 | ((ym ? smin : 0) + 1) << 4 |
                              ((ym ? 0 : smin) + 1) << 6;
                s_a[wid][i] = fabsf(__fdiv_rn(ym ? gx : gy, ym ? gy : gx));
            }
            __syncwarp();
            int q = t0, t = 0, x = 0, y = 0, n = 0;
            int mx = 0, my = 0, nx = 0, ny = 0;  // major and minor step (the side probe is one major step back)
            float e = 0.f, a = 0.f;
            bool act = false;
            while (true) {
                const unsigned idle = __ballot_sync(kAll, !act);
                if (!act) {
                    const int k = q + __popc(idle & below);
                    if (k < t1) {
                        t = k;
                        act = true;
                        const int i = (k - t0) >> 1;
                        const int xy = s_xy[wid][i], st = s_g[wid][i];
                        const int dir = (k & 1) ? 1 : -1;
                        x = xy & 0xffff;
                        y = xy >> 16;
                        mx = dir * ((st & 3) - 1);
                        my = dir * ((st >> 2 & 3) - 1);
                        nx = dir * ((st >> 4 & 3) - 1);
                        ny = dir * ((st >> 6 & 3) - 1);
                        a = s_a[wid][i];
                        e = 0.f;
                        n = 0;
                    }
                }
                q += __popc(idle);
                if (!__any_sync(kAll, act)) break;
                if (!act) continue;
                // The next kWalkAhead steps of the walk: its positions do not
                // depend on what the probes find, so all their probes are
                // issued before the first is looked at.  kind: 0 a step without
                // a probe, 1 one probe, 2 a probe and the side probe, 3 the
                // walk ends here (distSearch), 4 past the end.
                int kind[kWalkAhead], px[kWalkAhead], py[kWalkAhead], sx[kWalkAhead], sy[kWalkAhead];
                bool over = false;
#pragma unroll
                for (int j = 0; j < kWalkAhead; ++j) {
                    kind[j] = 4;
                    px[j] = py[j] = sx[j] = sy[j] = -1;
                    if (over) continue;
                    if (n >= 2 && n > nmax) {
                        kind[j] = 3;
                        over = true;
                        continue;
                    }
                    e = __fadd_rn(e, a);
                    x += mx;
                    y += my;
                    if (e >= 0.5f) {
                        x += nx;
                        y += ny;
                        e = __fadd_rn(e, -1.f);
                    }
                    ++n;
                    // After the first step the reference re-orients the walk
                    // along the gradient at its start point (Bresenham.cpp:
                    // 74-81): the direction already is dir * g, its product
                    // with g is dir * |g|^2, so the direction stays dir * g
                    // (0 when g is 0) and the steps are unchanged.
                    if (n == 1) {
                        kind[j] = 0;
                    } else {
                        kind[j] = n > 2 ? 2 : 1;
                        px[j] = x;
                        py[j] = y;
                        sx[j] = x - mx;
                        sy[j] = y - my;
                    }
                }
                uint2 w[kWalkAhead], ws[kWalkAhead];
#pragma unroll
                for (int j = 0; j < kWalkAhead; ++j) {
                    w[j] = ws[j] = make_uint2(0u, 0u);
                    if (kind[j] == 1 || kind[j] == 2) {
                        if (unsigned(px[j]) < unsigned(W) && unsigned(py[j]) < unsigned(H))
                            w[j] = __ldg(&L.bitidx[size_t(py[j]) * WW + (px[j] >> 5)]);
                        if (kind[j] == 2 && unsigned(sx[j]) < unsigned(W) && unsigned(sy[j]) < unsigned(H))
                            ws[j] = __ldg(&L.bitidx[size_t(sy[j]) * WW + (sx[j] >> 5)]);
                    }
                }
                // the first step, in walk order, that ends the walk: -1
                // outside the level or at distSearch, else the index of the
                // edge pixel met (-1 past a clamped edge count)
                auto found = [&](uint2 v, int qx, int qy) -> int {
                    if (unsigned(qx) >= unsigned(W) || unsigned(qy) >= unsigned(H)) return -1;
                    const uint32_t bit = 1u << (qx & 31);
                    if (!(v.x & bit)) return -2;
                    const int idx = int(v.y) + __popc(v.x & (bit - 1u));
                    return idx < E ? idx : -1;
                };
                int res = -2;  // -2: the walk goes on
#pragma unroll
                for (int j = 0; j < kWalkAhead; ++j) {
                    if (res != -2) continue;
                    if (kind[j] == 3) {
                        res = -1;
                    } else if (kind[j] == 1 || kind[j] == 2) {
                        res = found(w[j], px[j], py[j]);
                        if (res == -2 && kind[j] == 2) res = found(ws[j], sx[j], sy[j]);
                    }
                }
                if (res != -2) {
                    s_res[wid][t - t0] = res;
                    act = false;
                }
            }
            __syncwarp();
            for (int i = lane; i < np; i += 32) {
                L.before[p0 + i] = s_res[wid][2 * i];
                L.after[p0 + i] = s_res[wid][2 * i + 1];
            }
            __syncwarp();
        }
    }
}

// ------------------------------------------------------------------ vote --
// Vote.cpp:101-243: follow before/after links across the 2*nCrowns-1 ring
// edges with the gradient-angle and distance-ratio tests.
__device__ __forceinline__ float pt_dist(int xya, int xyb)
{
    const int ddx = (xyb & 0xffff) - (xya & 0xffff), ddy = (xyb >> 16) - (xya >> 16);
    return __fsqrt_rn(__fadd_rn(float(ddx * ddx), float(ddy * ddy)));
}

__device__ __forceinline__ float neg_dot(int ga, int gb)
{
    const int d = int(int16_t(ga & 0xffff)) * int(int16_t(gb & 0xffff)) + (ga >> 16) * (gb >> 16);
    return -float(d);
}

__global__ void k_vote(Levels lv, VoteParamsDev vp)
{
    const int stride = gridDim.x * blockDim.x;
    constexpr int kMaxSeg = 16;
    for (int l = 0; l < lv.n; ++l) {
        const LevelView& L = lv.l[l];
        const int E = lv.cnt[l].E;
        for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < E; p += stride) {
            float vd[kMaxSeg];
            int nd = 0;
            float total = 0.f;
            int chosen = -1;
            int current = L.before[p];
            const int gp = L.grad[p];
            const int xyp = L.exy[p];
            auto ratio_ok = [&]() {
                bool ok = true;
                for (int i = 0; i < nd; ++i)
                    for (int j = i + 1; j < nd; ++j)
                        ok = ok && (vd[i] <= __fmul_rn(vd[j], vp.ratioVoting)) && (vd[j] <= __fmul_rn(vd[i], vp.ratioVoting));
                return ok;
            };
            if (current >= 0 && neg_dot(gp, L.grad[current]) >= vp.angleVoting && 2 * vp.nCrowns - 1 <= kMaxSeg) {
                float d = pt_dist(xyp, L.exy[current]);
                vd[nd++] = d;
                total = __fadd_rn(total, d);
                for (int i = 1; i < vp.nCrowns; ++i) {
                    chosen = -1;
                    int target = L.after[current];
                    if (target < 0) break;
                    if (!(neg_dot(L.grad[target], L.grad[current]) >= vp.angleVoting)) break;
                    d = pt_dist(L.exy[target], L.exy[current]);
                    vd[nd++] = d;
                    total = __fadd_rn(total, d);
                    if (nd > 1 && !ratio_ok()) break;
                    current = target;
                    target = L.before[current];
                    if (target < 0) break;
                    if (!(neg_dot(L.grad[target], L.grad[current]) >= vp.angleVoting)) break;
                    d = pt_dist(L.exy[target], L.exy[current]);
                    vd[nd++] = d;
                    total = __fadd_rn(total, d);
                    if (!ratio_ok()) break;
                    current = target;
                    chosen = current;
                }
            }
            L.chosen[p] = chosen;
            L.total[p] = chosen >= 0 ? total : 0.f;
            if (chosen >= 0) atomicAdd(&L.nvotes[chosen], 1);
        }
    }
}

// ----------------------------------------------------- voter lists (CSR) --
// Chunked exclusive scan of nvotes[0, E) into voff, all levels, fixed grid.
constexpr int kScanBlocks = kScanBlocksPerLevel;
constexpr int kScanThreads = 256;
constexpr int kScanChunks = 32;  // chunks per level (partial sums at stride kScanBlocks)

// Voter-count scan: level blockIdx.y, chunk blockIdx.x of kScanChunks.
__global__ void __launch_bounds__(kScanThreads) k_vscan_partial(Levels lv, int32_t* partial)
{
    __shared__ int s_red[kScanThreads / 32];
    const int l = blockIdx.y;
    const LevelView& L = lv.l[l];
    const int E = lv.cnt[l].E;
    const int chunk = (E + kScanChunks - 1) / kScanChunks;
    const int b0 = blockIdx.x * chunk, b1 = min(E, b0 + chunk);
    int s = 0;
    for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) s += L.nvotes[i];
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        int v = threadIdx.x < kScanThreads / 32 ? s_red[threadIdx.x] : 0;
#pragma unroll
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) partial[l * kScanBlocks + blockIdx.x] = v;
    }
}

__global__ void __launch_bounds__(kScanThreads) k_vscan_final(Levels lv, const int32_t* partial)
{
    __shared__ int s_warp[33];
    __shared__ int s_base;
    const int l = blockIdx.y;
    const LevelView& L = lv.l[l];
    const int E = lv.cnt[l].E;
    const int chunk = (E + kScanChunks - 1) / kScanChunks;
    const int b0 = blockIdx.x * chunk, b1 = min(E, b0 + chunk);
    if (threadIdx.x == 0) {
        int b = 0;
        for (int k = 0; k < int(blockIdx.x); ++k) b += partial[l * kScanBlocks + k];
        s_base = b;
    }
    __syncthreads();
    int carry = s_base;
    for (int base = b0; base < b1; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int v = i < b1 ? L.nvotes[i] : 0;
        int total;
        const int ex = block_excl_scan(v, s_warp, &total);
        if (i < b1) L.voff[i] = carry + ex;
        carry += total;
    }
    if (blockIdx.x == kScanChunks - 1 && threadIdx.x == 0) {
        int V = 0;
        for (int k = 0; k < kScanChunks; ++k) V += partial[l * kScanBlocks + k];
        L.voff[E] = V;
        lv.cnt[l].V = V;
    }
}

__global__ void k_vfill(Levels lv)
{
    const int stride = gridDim.x * blockDim.x;
    for (int l = 0; l < lv.n; ++l) {
        const LevelView& L = lv.l[l];
        const int E = lv.cnt[l].E;
        for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < E; p += stride) {
            const int c = L.chosen[p];
            if (c < 0) continue;
            const int slot = atomicAdd(&L.fill[c], 1);
            L.vlist[L.voff[c] + slot] = p;
        }
    }
}

// Running mean of the field-line lengths in ascending voter order
// (Vote.cpp:232) and seed registration (Vote.cpp:236-241).
__device__ __forceinline__ void finish_point(const LevelView& L, LevelCounters& cnt, const VoteParamsDev& vp, int c,
                                             const int32_t* list, int n)
{
    float fl = 0.f;
    for (int k = 0; k < n; ++k) {
        const float nk = float(k + 1);
        fl = __fdiv_rn(__fadd_rn(__fmul_rn(fl, float(k)), L.total[list[k]]), nk);
    }
    L.flow[c] = fl;
    if (n >= vp.minVotes) {
        const int s = atomicAdd(&cnt.S, 1);
        if (s < L.seedcap) {
            L.seed_idx[s] = c;
            L.seed_key[s] = list[vp.minVotes - 1];
            L.seed_votes[s] = n;
        } else {
            atomicOr(&cnt.err, kErrSeedOverflow);
        }
    }
}

constexpr int kSmallList = 32;

__global__ void k_vlists_small(Levels lv, VoteParamsDev vp)
{
    const int stride = gridDim.x * blockDim.x;
    for (int l = 0; l < lv.n; ++l) {
        const LevelView& L = lv.l[l];
        const int E = lv.cnt[l].E;
        for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < E; c += stride) {
            const int n = L.voff[c + 1] - L.voff[c];
            if (n == 0) {
                L.flow[c] = 0.f;
                continue;
            }
            if (n > kSmallList) {
                const int q = atomicAdd(&lv.cnt[l].bigq, 1);
                L.bigq[q] = c;
                continue;
            }
            int32_t* list = L.vlist + L.voff[c];
            int v[kSmallList];
            for (int k = 0; k < n; ++k) v[k] = list[k];
            for (int k = 1; k < n; ++k) {
                const int key = v[k];
                int j = k - 1;
                while (j >= 0 && v[j] > key) { v[j + 1] = v[j]; --j; }
                v[j + 1] = key;
            }
            for (int k = 0; k < n; ++k) list[k] = v[k];
            finish_point(L, lv.cnt[l], vp, c, list, n);
        }
    }
}

// Long voter lists: one block per list, rank sort (voter indices are distinct).
constexpr int kBigSmem = 4096;

__global__ void __launch_bounds__(256) k_vlists_big(Levels lv, VoteParamsDev vp)
{
    __shared__ int32_t s_in[kBigSmem];
    __shared__ int32_t s_out[kBigSmem];
    for (int l = 0; l < lv.n; ++l) {
        const LevelView& L = lv.l[l];
        const int nq = lv.cnt[l].bigq;
        for (int qi = blockIdx.x; qi < nq; qi += gridDim.x) {
            const int c = L.bigq[qi];
            int32_t* list = L.vlist + L.voff[c];
            const int n = L.voff[c + 1] - L.voff[c];
            if (n <= kBigSmem) {
                for (int k = threadIdx.x; k < n; k += blockDim.x) s_in[k] = list[k];
                __syncthreads();
                for (int k = threadIdx.x; k < n; k += blockDim.x) {
                    const int v = s_in[k];
                    int rank = 0;
                    for (int j = 0; j < n; ++j) rank += s_in[j] < v;
                    s_out[rank] = v;
                }
                __syncthreads();
                for (int k = threadIdx.x; k < n; k += blockDim.x) list[k] = s_out[k];
            } else {
                // Very long list: rank from global memory into the upper half of
                // the chosen list's own slots is impossible in place, so stage
                // the ranks through the fill array (free after k_vfill).
                for (int k = threadIdx.x; k < n; k += blockDim.x) {
                    const int v = list[k];
                    int rank = 0;
                    for (int j = 0; j < n; ++j) rank += list[j] < v;
                    L.fill[L.voff[c] + rank] = v;
                }
                __syncthreads();
                for (int k = threadIdx.x; k < n; k += blockDim.x) list[k] = L.fill[L.voff[c] + k];
            }
            __syncthreads();
            if (threadIdx.x == 0) finish_point(L, lv.cnt[l], vp, c, list, n);
            __syncthreads();
        }
    }
}

// ------------------------------------------------------------- launchers --
static int total_of(const Levels& lv, int LevelView::*f)
{
    int s = 0;
    for (int l = 0; l < lv.n; ++l) s += lv.l[l].*f;
    return s;
}

void upload_constants(const float*, int, int)
{
    // The tables are initialised statically with the module (cK, cThinTab);
    // nothing is uploaded, so a context that reloads the module after a
    // device reset sees them too.
}

// fused: every frame has 4 levels and sides that are multiples of 8 (one
// k_pyramid3 launch, blockIdx.z = frame); else one resize launch per level.
static void launch_pyramid(const Levels& lv, cudaStream_t s, bool fused)
{
    const int lpf = lv.n / lv.frames;
    if (lpf < 2) return;
    if (fused && lpf == 4) {
        int w8 = 0, h8 = 0;
        for (int f = 0; f < lv.frames; ++f) {
            w8 = std::max(w8, lv.l[f * lpf].W / 8);
            h8 = std::max(h8, lv.l[f * lpf].H / 8);
        }
        const dim3 blk(32, 8);
        const dim3 grd((w8 + 31) / 32, (h8 + 7) / 8, lv.frames);
        k_pyramid3<<<grd, blk, 0, s>>>(lv);
        return;
    }
    for (int f = 0; f < lv.frames; ++f)
        for (int k = 1; k < lpf; ++k) {
            const LevelView& a = lv.l[f * lpf + k - 1];
            const LevelView& b = lv.l[f * lpf + k];
            const dim3 blk(32, 8);
            const dim3 grd((b.W + 31) / 32, (b.H + 7) / 8);
            k_resize_level<<<grd, blk, 0, s>>>(a.src, a.W, a.H, b.src, b.W, b.H);
        }
}

const char* stage_name(int k)
{
    static const char* names[kStageCount] = {"pyramid", "deriv_nms", "hyst_merge", "hyst_compress", "final_thin",
                                             "row_scan", "emit", "walk", "vote", "voter_scan", "voter_fill",
                                             "voter_sort"};
    return (k >= 0 && k < kStageCount) ? names[k] : "?";
}

static void mark(cudaEvent_t* ev, int k, cudaStream_t s)
{
    if (ev) CCTAGB_CUDA(cudaEventRecord(ev[k], s));
}

// Holds the stream for about `us` microseconds (bounded loop) so that the
// host can queue every stage behind it; used only by the per-stage timing
// mode, which launches without a graph.
__global__ void k_gate(int us)
{
    for (int i = 0; i < us; ++i) __nanosleep(1000);
}

void launch_gate(cudaStream_t s, int us) { k_gate<<<1, 1, 0, s>>>(us); }

// The segments of p back to back into dst: a flat grid-stride loop over the
// total, each thread advancing its segment cursor as its index grows.
__global__ void __launch_bounds__(256) k_pack_words(PackSegs p, int32_t* __restrict__ dst)
{
    const long long total = p.off[p.n];
    const long long stride = (long long)gridDim.x * blockDim.x;
    int g = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        while (i >= p.off[g + 1]) ++g;  // i < off[n], so g < n
        dst[i] = __ldg(p.src[g] + (i - p.off[g]));
    }
}

int launch_pack(const PackSegs& p, int32_t* dst, cudaStream_t s)
{
    if (p.n <= 0 || p.n > kMaxPackSegs) return 0;
    const long long total = p.off[p.n];
    if (total <= 0) return 0;
    const int blocks = int(std::min<long long>((total + 255) / 256, 148 * 4));
    k_pack_words<<<blocks, 256, 0, s>>>(p, dst);
    CCTAGB_CUDA(cudaGetLastError());
    return 1;
}

static void launch_edges(const Levels& lv, const VoteParamsDev& vp, cudaStream_t s, int write_derivs,
                         cudaEvent_t* ev)
{
    k_deriv_nms<<<total_of(lv, &LevelView::nms_tiles), 128, 0, s>>>(lv, vp, write_derivs);
    mark(ev, kStDerivNms + 1, s);
    const int tiles = total_of(lv, &LevelView::uf_tiles);
    const int hb = (tiles + kHystWarps - 1) / kHystWarps;
    k_hyst_tiles<<<hb, 32 * kHystWarps, 0, s>>>(lv, tiles);
    k_hyst_unions<<<tiles, 64, 0, s>>>(lv);
    mark(ev, kStHystMerge + 1, s);
    k_hyst_roots<<<tiles, kTileComps, 0, s>>>(lv);
    k_hyst_final<<<hb, 32 * kHystWarps, 0, s>>>(lv, tiles);
    mark(ev, kStHystCompress + 1, s);
    const int tt = total_of(lv, &LevelView::thin_tiles);
    k_final_thin<<<(tt + kThinWarps - 1) / kThinWarps, 32 * kThinWarps, 0, s>>>(lv, tt);
    mark(ev, kStFinalThin + 1, s);
    k_row_scan<<<lv.n, 1024, 0, s>>>(lv);
    mark(ev, kStRowScan + 1, s);
    int rows = 0;
    for (int l = 0; l < lv.n; ++l) rows += lv.l[l].H;
    k_emit<<<rows, 128, 0, s>>>(lv, rows);
    mark(ev, kStEmit + 1, s);
}

void launch_image_stage(const Levels& lv, const VoteParamsDev& vp, cudaStream_t s, bool fused_pyramid,
                        cudaEvent_t* ev)
{
    CCTAGB_CUDA(cudaMemsetAsync(lv.cnt, 0, sizeof(LevelCounters) * lv.n, s));
    mark(ev, 0, s);
    launch_pyramid(lv, s, fused_pyramid);
    mark(ev, kStPyramid + 1, s);
    launch_edges(lv, vp, s, 1, ev);
    const int G = 148 * 8;
    static const int walkBlocks = [] {
        int per = 0;
        CCTAGB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_walk, 32 * kWalkWarps, 0));
        return 148 * (per > 0 ? per : 1);
    }();
    k_walk<<<walkBlocks, 32 * kWalkWarps, 0, s>>>(lv, vp);  // the blocks resident at once
    mark(ev, kStWalk + 1, s);
    k_vote<<<G, 256, 0, s>>>(lv, vp);
    mark(ev, kStVote + 1, s);
    k_vscan_partial<<<dim3(kScanChunks, lv.n), kScanThreads, 0, s>>>(lv, lv.partial);
    k_vscan_final<<<dim3(kScanChunks, lv.n), kScanThreads, 0, s>>>(lv, lv.partial);
    mark(ev, kStVoterScan + 1, s);
    k_vfill<<<G, 256, 0, s>>>(lv);
    mark(ev, kStVoterFill + 1, s);
    k_vlists_small<<<G, 256, 0, s>>>(lv, vp);
    k_vlists_big<<<148, 256, 0, s>>>(lv, vp);
    mark(ev, kStVoterSort + 1, s);
    CCTAGB_CUDA(cudaGetLastError());
}

void launch_canny_only(const Levels& lv, const VoteParamsDev& vp, cudaStream_t s)
{
    CCTAGB_CUDA(cudaMemsetAsync(lv.cnt, 0, sizeof(LevelCounters) * lv.n, s));
    launch_edges(lv, vp, s, 0, nullptr);
    CCTAGB_CUDA(cudaGetLastError());
}

// Edge stage of one level from its gray image (derivatives, NMS, hysteresis,
// thinning, edge bitmap) without the compaction.  The caller clears
// lv.cnt[0] and lv.l[0].row_count beforehand.
__global__ void k_bitmap_to_bytes(Levels lv, uint8_t* out)
{
    const LevelView& L = lv.l[0];
    const size_t n = size_t(L.W) * L.H;
    for (size_t p = size_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n; p += size_t(gridDim.x) * blockDim.x) {
        const int x = int(p % L.W), y = int(p / L.W);
        out[p] = edge_bit(L, x, y) ? 255 : 0;
    }
}

__global__ void k_scatter_counters(const LevelCounters* __restrict__ src, CounterTargets t)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < t.n) *t.dst[i] = src[i];
}

void launch_scatter_counters(const LevelCounters* src, const CounterTargets& t, cudaStream_t s)
{
    k_scatter_counters<<<1, kMaxLaunchLevels, 0, s>>>(src, t);
    CCTAGB_CUDA(cudaGetLastError());
}

__global__ void k_copy_status(const LevelCounters* cnt, int32_t* status)
{
    *status = cnt->err;
}

void launch_edge_level(const Levels& lv, const VoteParamsDev& vp, cudaStream_t s, uint8_t* edges_out,
                       int32_t* status_out)
{
    const LevelView& L = lv.l[0];
    k_deriv_nms<<<L.nms_tiles, 128, 0, s>>>(lv, vp, 1);
    const int hb = (L.uf_tiles + kHystWarps - 1) / kHystWarps;
    k_hyst_tiles<<<hb, 32 * kHystWarps, 0, s>>>(lv, L.uf_tiles);
    k_hyst_unions<<<L.uf_tiles, 64, 0, s>>>(lv);
    k_hyst_roots<<<L.uf_tiles, kTileComps, 0, s>>>(lv);
    k_hyst_final<<<hb, 32 * kHystWarps, 0, s>>>(lv, L.uf_tiles);
    k_final_thin<<<(L.thin_tiles + kThinWarps - 1) / kThinWarps, 32 * kThinWarps, 0, s>>>(lv, L.thin_tiles);
    k_bitmap_to_bytes<<<148 * 4, 256, 0, s>>>(lv, edges_out);
    if (status_out) k_copy_status<<<1, 1, 0, s>>>(lv.cnt, status_out);
    CCTAGB_CUDA(cudaGetLastError());
}

}  // namespace cctagb
