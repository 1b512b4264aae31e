// Ellipse growing of the candidate stage on the GPU (completeFlowComponent's
// growing half, Detection.cpp:190-267, with ellipseGrowing2,
// EllipseGrowing.cpp:459-551): one block per candidate, the candidates of all
// levels of a frame in one launch.
#pragma once

#include <cstdint>
#include <vector>

#include "common.hpp"

namespace cctagb {

constexpr int kGrowMaxOuter = 2048;   // outer points one block holds (shared memory)

// One candidate: its level and its filtered points pts[first, first + count).
struct GrowTask {
    int level;
    int first, count;
};

enum GrowStatus : int32_t {
    kGrowDrop = 0,   // the candidate leaves the list (a fit failed or a check rejected it)
    kGrowKeep = 1,   // it goes on to loop 3 with its outer points and ellipse
    kGrowHost = 2,   // more outer points than kGrowMaxOuter: grown by the host code instead
};

struct GrowResult {
    int32_t status;
    int32_t nOuter;
    float cx, cy, a, b, angle;
    float Q[9];
};

class GrowGpu {
public:
    GrowGpu(int spin_us, int max_points);
    ~GrowGpu();
    GrowGpu(const GrowGpu&) = delete;
    GrowGpu& operator=(const GrowGpu&) = delete;

    // Grows the tasks on the frame's levels (lv.l[0 .. lv.n), E[l] edge
    // points each) on stream s and waits; res[t] and the outer point indices
    // outer[t * stride, + res[t].nOuter) come back on the host.
    void run(const Levels& lv, const int* E, const std::vector<GrowTask>& tasks, const std::vector<int32_t>& pts,
             float hullWidth, float thrMedian, cudaStream_t s, std::vector<GrowResult>& res,
             std::vector<int32_t>& outer, int& stride);

    long long h2d_bytes() const { return h2d_; }
    long long d2h_bytes() const { return d2h_; }
    int launches() const { return launches_; }

private:
    void ensure(int tasks, int pts);
    HostWaiter waiter_;
    GrowTask* d_tasks_ = nullptr;
    int32_t* d_pts_ = nullptr;
    GrowResult* d_res_ = nullptr;
    int32_t* d_outer_ = nullptr;
    GrowTask* h_tasks_ = nullptr;
    int32_t* h_pts_ = nullptr;
    GrowResult* h_res_ = nullptr;
    int32_t* h_outer_ = nullptr;
    int cap_ = kGrowMaxOuter;
    int taskCap_ = 0, ptsCap_ = 0;
    long long h2d_ = 0, d2h_ = 0;
    int launches_ = 0;
};

}  // namespace cctagb
