// Allocation-free edge stage: cctagb_edges_noalloc.
//
// Some callers cannot allocate device memory at the time they want edges: an
// application that hands every byte of the GPU to its own memory pool at start
// up, a real-time loop whose rules forbid cudaMalloc/cudaFree after
// initialisation (they can block and synchronise the device), or a caller that
// has no handle and only owns the frame and output buffers.  This entry point
// runs the edge stage of one frame (9x9 derivatives, Canny NMS, hysteresis,
// thinning) with the caller's input and output buffers and keeps its own
// scratch (class map, hysteresis bit planes and tile components, edge bitmap,
// row counts, counters) in the file-scope device array below.  It calls no
// cudaMalloc, cudaFree or allocating library routine.
//
// Limits and rules:
//  * at most kNoAllocMaxPixels pixels and kNoAllocMaxSide per side, frame rows
//    contiguous (pitch == width); larger frames are rejected with
//    CCTAGB_TOO_LARGE;
//  * the array (about 2.5 MB) is held by every GPU that loads the library,
//    until the process exits;
//  * the first call on a device (in each CUDA context: after a
//    cudaDeviceReset the next call does it again) resolves the array's device
//    address with cudaGetSymbolAddress, with that device current; make that
//    first call before any stream capture.  The filter tables are
//    initialised statically with the module, so nothing is uploaded;
//  * all calls share the one array and it keeps the last call's contents:
//    calls whose GPU work overlaps (different streams, or host threads) race
//    and give wrong results; serialise them on one stream.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>

#include "common.hpp"

namespace cctagb {

namespace {

constexpr int kNoAllocMaxPixels = 1 << 20;
constexpr int kNoAllocMaxSide = 4096;
constexpr size_t kAlign = 256;

constexpr size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

// Layout of the scratch array.
constexpr size_t kOffCounters = 0;
constexpr size_t kOffRowCount = align_up(kOffCounters + sizeof(LevelCounters));
// bitmap words of one plane: ceil(w / 32) * h <= w h / 32 + h
constexpr size_t kBitmapWords = size_t(kNoAllocMaxPixels) / 32 + kNoAllocMaxSide;
// 32x32 tiles: ceil(w / 32) ceil(h / 32) <= w h / 1024 + (w + h) / 32 + 1
constexpr size_t kMaxTiles = size_t(kNoAllocMaxPixels) / 1024 + 2 * kNoAllocMaxSide / 32 + 1;
constexpr size_t kOffMap = align_up(kOffRowCount + sizeof(int32_t) * kNoAllocMaxSide);
constexpr size_t kOffHyst = align_up(kOffMap + size_t(kNoAllocMaxPixels));           // 3 bitmap planes
constexpr size_t kOffBlab = align_up(kOffHyst + 3 * sizeof(uint32_t) * kBitmapWords);  // 128 B per tile
constexpr size_t kOffTcomp = align_up(kOffBlab + 128 * kMaxTiles);                     // 64 ints per tile
constexpr size_t kOffTflag = align_up(kOffTcomp + 64 * sizeof(int32_t) * kMaxTiles);  // 64 ints per tile
constexpr size_t kOffBitmap = align_up(kOffTflag + 64 * sizeof(int32_t) * kMaxTiles);
constexpr size_t kScratchBytes = align_up(kOffBitmap + sizeof(uint32_t) * kBitmapWords);

constexpr int kMaxDevices = 64;

struct DeviceSlot {
    void* ctx = nullptr;  // the context the address was resolved in
    uint8_t* base = nullptr;
};

// cuCtxGetCurrent through the runtime's driver entry point (no link to the
// driver library): the current context, or nullptr when it cannot be read.
void* current_context()
{
    using GetCtx = int (*)(void**);
    static GetCtx fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            f = nullptr;
        }
        return reinterpret_cast<GetCtx>(f);
    }();
    void* ctx = nullptr;
    if (!fn || fn(&ctx) != 0) return nullptr;
    return ctx;
}

std::mutex g_mu;
DeviceSlot g_slots[kMaxDevices];

}  // namespace

static __device__ __align__(256) uint8_t g_edge_scratch[kScratchBytes];

// Resolves the device address of the scratch array on the current device,
// once per device and context (a new context after a device reset resolves it
// again; where the context cannot be read, every call resolves it).
static uint8_t* scratch_for_current_device(cctagb_status& st)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        st = CCTAGB_NO_DEVICE;
        return nullptr;
    }
    void* ctx = current_context();
    std::lock_guard<std::mutex> lock(g_mu);
    DeviceSlot& s = g_slots[dev];
    if (!s.base || !ctx || s.ctx != ctx) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_edge_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            st = CCTAGB_CUDA_ERROR;
            return nullptr;
        }
        // the first call may have created the context: read it again
        s.ctx = ctx ? ctx : current_context();
        s.base = static_cast<uint8_t*>(p);
    }
    st = CCTAGB_OK;
    return s.base;
}

}  // namespace cctagb

extern "C" cctagb_status cctagb_edges_noalloc(const uint8_t* d_gray, int w, int h, size_t pitch, float cannyThrLow,
                                              float cannyThrHigh, int16_t* d_dx, int16_t* d_dy, uint8_t* d_edges,
                                              int32_t* d_status, void* stream)
{
    using namespace cctagb;
    if (!d_gray || !d_dx || !d_dy || !d_edges || w < 1 || h < 1 || pitch != size_t(w)) return CCTAGB_BAD_ARG;
    if (size_t(w) * size_t(h) > size_t(kNoAllocMaxPixels) || w > kNoAllocMaxSide || h > kNoAllocMaxSide)
        return CCTAGB_TOO_LARGE;
    cctagb_status st;
    uint8_t* base = scratch_for_current_device(st);
    if (!base) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // What must start at zero: the counters (error bits) and the per-row edge
    // counts the thinning kernel accumulates into.
    if (cudaMemsetAsync(base + kOffCounters, 0, sizeof(LevelCounters), s) != cudaSuccess ||
        cudaMemsetAsync(base + kOffRowCount, 0, sizeof(int32_t) * size_t(h), s) != cudaSuccess) {
        cudaGetLastError();
        return CCTAGB_CUDA_ERROR;
    }
    Levels lv{};
    lv.n = 1;
    lv.frames = 1;
    lv.cnt = reinterpret_cast<LevelCounters*>(base + kOffCounters);
    LevelView& L = lv.l[0];
    L.W = w;
    L.H = h;
    L.WW = (w + 31) / 32;
    L.src = const_cast<uint8_t*>(d_gray);
    L.dx = d_dx;
    L.dy = d_dy;
    L.map = base + kOffMap;
    L.hbits = reinterpret_cast<uint32_t*>(base + kOffHyst);
    L.blab = base + kOffBlab;
    L.tcomp = reinterpret_cast<int32_t*>(base + kOffTcomp);
    L.tflag = reinterpret_cast<int32_t*>(base + kOffTflag);
    L.bitmap = reinterpret_cast<uint32_t*>(base + kOffBitmap);
    L.row_count = reinterpret_cast<int32_t*>(base + kOffRowCount);
    L.nms_tx = (w + 29) / 30;
    L.nms_tiles = L.nms_tx * ((h + 29) / 30);
    L.thin_tx = (w + 31) / 32;
    L.thin_tiles = L.thin_tx * ((h + 27) / 28);  // word columns x 28-row strips
    L.pix_blocks = int((size_t(w) * h + 255) / 256);
    L.uf_tx = (w + 31) / 32;
    L.uf_tiles = L.uf_tx * ((h + 31) / 32);
    VoteParamsDev vp{};
    float lo = cannyThrLow * 256.f, hi = cannyThrHigh * 256.f;
    if (lo > hi) std::swap(lo, hi);
    vp.low = int(std::floor(lo));
    vp.high = int(std::floor(hi));
    try {
        launch_edge_level(lv, vp, s, d_edges, d_status);
    } catch (const Error& err) {
        return err.status;
    }
    return CCTAGB_OK;
}
