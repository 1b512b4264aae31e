// Arithmetic of the candidate stage that runs both on the host
// (candidates.cpp) and on the GPU (loop_one.cu).  Each helper is one source
// for both compilers; with no contraction into fused multiply-adds (host
// -ffp-contract=off, device --fmad=false) they give the same bits.
#pragma once

#include <cmath>
#include <cstdint>

#include "geometry.hpp"
#include "cctag_b200/portable/pmath.hpp"

#if defined(__CUDACC__)
#define CCTAGB_UNROLL _Pragma("unroll")
#else
#define CCTAGB_UNROLL
#endif

namespace cctagb {
namespace cand {

constexpr float kPiF = 3.14159265358979323846f;
constexpr int kEdgeNotFound = -1;
constexpr int kConvexityLost = -2;
constexpr int kLinkMaxLength = 100;  // Vote.cpp:294 maxLength
constexpr int kLinkMaxWindow = 64;   // bound on windowSizeOnInnerEllipticSegment

// Vote.cpp:300-301: gradient angle in [0, 2 pi).
CCTAGB_HD inline float link_angle(float dx, float dy)
{
    return ::fmodf(pm::atan2f_(dy, dx) + 2.0f * kPiF, 2.0f * kPiF);
}

// Vote.cpp:307: first neighbour direction to try.
CCTAGB_HD inline int link_shift(float angle)
{
    return int(::roundf(((angle + kPiF / 4.0f) / (2.0f * kPiF)) * 8.0f)) - 1;
}

// Vote.cpp:329-344: convexity test between the oldest and the newest angle of
// the window (full: the window holds windowSize angles).
CCTAGB_HD inline bool link_convexity_lost(float front, float back, bool full, int dir)
{
    const float d = back - front;
    if (full) return float(dir) * pm::sinf_(d) < 0.0f;
    const float s = float(dir) * pm::sinf_(d);
    const float c = pm::cosf_(d);
    return (s < -0.707f && c > 0.f) || (s < 0.f && c < 0.f);
}

// Vote.cpp:352: running mean of the votes received along the segment.
CCTAGB_HD inline float link_average_vote(float average, int segSize, int voters)
{
    return (average * float(segSize) + float(voters)) / (float(segSize) + 1.f);
}

// Vote.cpp:101-106: averageReceivedVote of a segment.
CCTAGB_HD inline float received_vote_key(int nReceived, int nVoted)
{
    return float(nReceived * nReceived) / float(nVoted);
}

// 5x5 linear solve with partial pivoting (FP64); false if singular.  Loops
// with constant bounds and constant-index row swaps, so that the GPU keeps
// the system in registers; the operations are those of the textbook
// elimination in the same order on both sides.
CCTAGB_HD inline bool solve5(double A[5][5], double b[5], double x[5])
{
CCTAGB_UNROLL
    for (int c = 0; c < 5; ++c) {
        int piv = c;
        double best = ::fabs(A[c][c]);
CCTAGB_UNROLL
        for (int r = c + 1; r < 5; ++r) {
            const double v = ::fabs(A[r][c]);
            if (v > best) {
                best = v;
                piv = r;
            }
        }
        if (best == 0.0) return false;
CCTAGB_UNROLL
        for (int r = c + 1; r < 5; ++r)
            if (r == piv) {
CCTAGB_UNROLL
                for (int k = 0; k < 5; ++k) {
                    const double t = A[r][k];
                    A[r][k] = A[c][k];
                    A[c][k] = t;
                }
                const double t = b[r];
                b[r] = b[c];
                b[c] = t;
            }
CCTAGB_UNROLL
        for (int r = c + 1; r < 5; ++r) {
            const double f = A[r][c] / A[c][c];
CCTAGB_UNROLL
            for (int k = c; k < 5; ++k) A[r][k] -= f * A[c][k];
            b[r] -= f * b[c];
        }
    }
CCTAGB_UNROLL
    for (int r = 4; r >= 0; --r) {
        double s = b[r];
CCTAGB_UNROLL
        for (int k = r + 1; k < 5; ++k) s -= A[r][k] * x[k];
        x[r] = s / A[r][r];
    }
    return true;
}

// One LMedS draw of outlierRemoval (Vote.cpp:478-512): the conic through five
// points, normalised with Q22 = 1.  Returns 0 when the draw counts as a
// failure (singular system, not an ellipse, axis ratio out of range), 2 when
// the conic's parameters are not real (the reference's exception: the draw
// is neither counted nor used), 1 when Q is a usable ellipse.
CCTAGB_HD inline int lmeds_conic(const geo::Pt* pts, const int perm[5], geo::Mat3& Q)
{
    double A[5][5], b[5], t[5];
    for (int i = 0; i < 5; ++i) {
        const double x = pts[perm[i]].x, y = pts[perm[i]].y;
        A[i][0] = x * x;
        A[i][1] = 2.0 * x * y;
        A[i][2] = y * y;
        A[i][3] = 2.0 * x;
        A[i][4] = 2.0 * y;
        b[i] = -1.0;
    }
    if (!solve5(A, b, t)) return 0;
    if (!(float(t[0]) * float(t[2]) - float(t[1]) * float(t[1]) > 0)) return 0;
    Q.m[0][0] = float(t[0]);
    Q.m[0][1] = Q.m[1][0] = float(t[1]);
    Q.m[0][2] = Q.m[2][0] = float(t[3]);
    Q.m[1][1] = float(t[2]);
    Q.m[1][2] = Q.m[2][1] = float(t[4]);
    Q.m[2][2] = 1.f;
    float cx, cy, a, bb, angle;
    if (!geo::params_of_conic(Q, cx, cy, a, bb, angle)) return 2;
    const float ratio = a / bb;
    if (ratio < 0.04f || ratio > 25) return 0;
    return 1;
}

// PCG32 stream of one candidate in one loop: results do not depend on how
// candidates are spread over threads.
CCTAGB_HD inline geo::Pcg32 candidate_rng(int level, uint64_t index, int phase)
{
    return geo::Pcg32(271828, (uint64_t(level) << 32) | (index << 1) | uint64_t(phase));
}

}  // namespace cand
}  // namespace cctagb
