/*
 * cctag_b200 -- C ABI of the B200 CCTag detection hot path.
 *
 * Every entry point returns a cctagb_status, never exits and never throws
 * across the ABI.  Device memory, streams and captured CUDA graphs are owned by
 * the handle.  A handle is not thread-safe: use one handle per host thread.
 *
 * Reference interfaces replaced (paths inside the CCTag project):
 *   cctagb_detect          <- cctag::cctagDetection(ptr_list<ICCTag>&, pipeId, frame,
 *                             const cv::Mat&, const Parameters&, logtime::Mgmt*,
 *                             const CCTagMarkersBank*)           src/cctag/ICCTag.hpp:125-131
 *                             (file-path overload                 src/cctag/ICCTag.hpp:103-110)
 *   cctagb_params          <- cctag::Parameters                   src/cctag/Params.hpp:108-255
 *   cctagb_params_default  <- Parameters::Parameters(nCrowns)     src/cctag/Params.cpp:38-82
 *   cctagb_set_bank        <- CCTagMarkersBank(nCrowns / file)    src/cctag/CCTagMarkersBank.cpp:22-78
 *   cctagb_marker          <- ICCTag / CCTag accessors            src/cctag/ICCTag.hpp:28-82, CCTag.hpp
 *   status codes           <- cctag::status                       src/cctag/CCTag.hpp:416-426
 *   cctagb_create          <- initCuda / TagPipe::initialize      src/cctag/Detection.cpp:732-760,
 *                                                                  src/cctag/cuda/tag.cu:76-127
 *   cctagb_level_*         <- ImagePyramid::getLevel(i)->getSrc/getDx/getDy/getEdges
 *                                                                  src/cctag/Level.hpp:38-42
 *   cctagb_level_edge_points / _links / _votes
 *                          <- EdgePointCollection + vote()        src/cctag/Types.hpp:19-158,
 *                                                                  src/cctag/Vote.cpp:58-247
 *   cctagb_canny_from_derivatives
 *                          <- cvRecodedCanny after filter2D        src/cctag/filter/cvRecode.cpp:94-421
 *                             followed by thin()                  src/cctag/filter/thinning.cpp:15-19
 *   cctagb_detect_batch    <- one cctagDetection call per camera  src/cctag/ICCTag.hpp:125-131
 *   cctagb_identify_tasks  <- identify_step_2 / refineConicFamilyGlob + orazioDistanceRobust
 *                                                                  src/cctag/Identification.cpp:813-965,1318-1480
 *   cctagb_last_tasks      <- the cuts identify_step_1 selects     src/cctag/Identification.cpp:1172-1301
 *   cctagb_level_loop_two  <- loop 1 + outlier removal of cctagDetectionFromEdges
 *                                                                  src/cctag/Detection.cpp:69-156,609-627
 *   cctagb_cut_cost        <- costFunctionGlob (forward only in the reference; here with its
 *                             gradient in the center and in H)   src/cctag/Identification.cpp:1122-1158
 *   cctagb_cut_cost_f64    <- the same in double precision (a check form; no reference counterpart)
 *   cctagb_edges_noalloc   <- no reference counterpart (the edge stage on caller buffers,
 *                             allocating nothing)
 *   cctagb_autotune / cctagb_tune_*
 *                          <- no reference counterpart (the reference fixes its batch layout,
 *                             one host thread and stream per pyramid level, at build time:
 *                                                                  src/cctag/cuda/tag_threads.cu:19-91)
 *   cctagb_host_frames / cctagb_submit / cctagb_wait
 *                          <- page-locked frames + async upload    src/cctag/cuda/frame.cu:110-148
 */
#ifndef CCTAG_B200_H
#define CCTAG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum cctagb_status {
    CCTAGB_OK = 0,
    CCTAGB_BAD_ARG = 1,            /* null pointer, bad size, bad parameter value      */
    CCTAGB_CUDA_ERROR = 2,         /* a CUDA runtime call failed (see last_error)       */
    CCTAGB_NO_DEVICE = 3,          /* no CUDA device, or not an sm_100 device           */
    CCTAGB_OVERFLOW_EDGES = 4,     /* more edge points than the handle's capacity       */
    CCTAGB_OVERFLOW_SEEDS = 5,     /* more seeds than the handle's capacity             */
    CCTAGB_OVERFLOW_VOTERS = 6,    /* a candidate gathers more voters than its capacity */
    CCTAGB_HYST_NO_CONVERGE = 7,   /* hysteresis union-find exceeded its iteration cap  */
    CCTAGB_TOO_LARGE = 8,          /* frame larger than the handle was created for      */
    CCTAGB_BANK_ERROR = 9,         /* marker bank missing, empty or malformed           */
    CCTAGB_INTERNAL = 10
} cctagb_status;

/* Marker status values, as cctag::status (CCTag.hpp:416-426). */
#define CCTAGB_ID_RELIABLE 1
#define CCTAGB_TOO_FEW_OUTER_POINTS (-1)
#define CCTAGB_NO_COLLECTED_CUTS (-1)
#define CCTAGB_NO_SELECTED_CUTS (-2)
#define CCTAGB_OPTI_HAS_DIVERGED (-3)
#define CCTAGB_ID_NOT_RELIABLE (-4)
#define CCTAGB_DEGENERATE (-5)

/* Center refinement used by identification. */
#define CCTAGB_REFINE_GRID 0          /* the reference's 5x5 shrinking grid search       */
#define CCTAGB_REFINE_GAUSS_NEWTON 1  /* adjoint-driven Gauss-Newton, FP64 normal solve  */

/* Field names and defaults follow cctag::Parameters (Params.hpp:27-66). */
typedef struct cctagb_params {
    float cannyThrLow;                          /* 0.01  */
    float cannyThrHigh;                         /* 0.04  */
    int distSearch;                             /* 30    */
    int thrGradientMagInVote;                   /* 2500  */
    float angleVoting;                          /* 0     */
    float ratioVoting;                          /* 4     */
    float averageVoteMin;                       /* 0     */
    float thrMedianDistanceEllipse;             /* 3     */
    int maximumNbSeeds;                         /* 500   */
    int maximumNbCandidatesLoopTwo;             /* 40    */
    int nCrowns;                                /* 3     */
    int nCircles;                               /* 2*nCrowns */
    int minPointsSegmentCandidate;              /* 10    */
    int minVotesToSelectCandidate;              /* 3     */
    float threshRobustEstimationOfOuterEllipse; /* 30    */
    float ellipseGrowingEllipticHullWidth;      /* 2.3   */
    int windowSizeOnInnerEllipticSegment;       /* 20    */
    int numberOfMultiresLayers;                 /* 4     */
    int numberOfProcessedMultiresLayers;        /* 4     */
    int nSamplesOuterEllipse;                   /* 150   */
    int numCutsInIdentStep;                     /* 22    */
    int numSamplesOuterEdgePointsRefinement;    /* 20    */
    int cutsSelectionTrials;                    /* 500   */
    int sampleCutLength;                        /* 100   */
    int imagedCenterNGridSample;                /* 5     */
    float imagedCenterNeighbourSize;            /* 0.2   */
    float minIdentProba;                        /* 1e-6  */
    int useLMDif;                               /* 1 (unused by the reference path) */
    int searchForAnotherSegment;                /* 1     */
    int writeOutput;                            /* 0     */
    int doIdentification;                       /* 1     */
    uint32_t maxEdges;                          /* 20000 (unused by the reference path) */
    /* B200-specific */
    int refineMode;                             /* CCTAGB_REFINE_GRID */
    int gnIterations;                           /* 12: cost evaluations at most in REFINE_GAUSS_NEWTON */
    int gnCoarseRounds;                         /* 1: grid rounds before Gauss-Newton */
    int edgeCapacityDivisor;                    /* 4: edge capacity per level = W*H/divisor */
    int hostThreads;                            /* 0: host threads of the candidate stage; 0 = one per physical core, less one per detection slot beyond the first */
    int gnCoarseGrid;                           /* 3: trial grid (3 or 5 per side) of the coarse rounds of REFINE_GAUSS_NEWTON */
    float gnCoarseNeighbourSize;                /* 0.1: their neighbourhood, as imagedCenterNeighbourSize */
    int batchWaveFrames;                        /* 4: frames whose image stages share one launch in cctagb_detect_batch (1..16) */
    int identLayout;                            /* CCTAGB_IDENT_AUTO: block layout of the identification kernel */
    int hostSpinMicros;                         /* -1: a host thread waiting on the GPU spins this long (microseconds), then sleeps until the GPU is done; < 0 spins throughout (least latency; sleeping frees the core for other work) */
    int gpuEllipseGrowing;                      /* 0: the candidates' ellipse growing runs on the host; 1: on the GPU, one block per candidate (the same results bit for bit, but slower on B200: its fits are serial FP64 sums in point order) */
    int gpuGrowMaxPoints;                       /* 2048: outer points a candidate may reach on the GPU (16..2048); a larger one grows on the host */
} cctagb_params;

/* Block layouts of the identification kernel (the results are the same bits). */
#define CCTAGB_IDENT_AUTO 0     /* a cluster of 4 blocks per marker when a call's markers fit the SMs (least latency for one frame), else one block each */
#define CCTAGB_IDENT_BLOCK 1    /* one block per marker (least SM time: for several frames in flight) */

typedef struct cctagb_ellipse {
    float cx, cy, a, b, angle; /* parameters (Ellipse.hpp)            */
    float m[9];                /* row-major conic matrix               */
} cctagb_ellipse;

typedef struct cctagb_marker {
    int id;                    /* 0-based bank row, -1 if none         */
    int status;                /* CCTAGB_ID_RELIABLE or a failure code */
    float x, y;                /* refined imaged center (centerImg)    */
    cctagb_ellipse outer;      /* rescaledOuterEllipse (level-0 frame) */
    float homography[9];       /* row-major, marker plane -> image     */
    float quality;             /* 1 / normalised residual              */
    int pyramidLevel;
    float scale;
} cctagb_marker;

typedef struct cctagb_stats {
    int edge_points[8];        /* per level                            */
    int seeds[8];              /* per level                            */
    int candidates;            /* markers before identification        */
    int markers;               /* markers returned                     */
    float ms_image_stage;      /* device time: pyramid .. seeds        */
    float ms_host_candidates;  /* host wall time of the candidate stage */
    float ms_identify;         /* device time of identification        */
    float ms_total;            /* host wall time of the whole call     */
    long long h2d_bytes;       /* host->device bytes copied by the call */
    long long d2h_bytes;       /* device->host bytes copied by the call */
    int kernel_launches;       /* kernels launched by the call         */
    float ms_download;         /* host wall time of the edge-point downloads */
    float ms_cut_selection;    /* host wall time of the cut-selection set-up (outer points and tasks staged); the angular sort, subsampling and cut selection then run on the GPU, just before identification */
    int grown_gpu;             /* candidates whose ellipse growing ran on the GPU */
    int grown_host;            /* ... on the host (gpuEllipseGrowing 0, or too many outer points for the kernel) */
} cctagb_stats;

typedef struct cctagb_handle cctagb_handle;

void cctagb_params_default(cctagb_params* p, int nCrowns);
const char* cctagb_status_string(cctagb_status s);

cctagb_status cctagb_create(const cctagb_params* p, int max_w, int max_h, int max_batch, cctagb_handle** out);
cctagb_status cctagb_destroy(cctagb_handle* h);
const char* cctagb_last_error_string(const cctagb_handle* h);

/* Replace the marker bank: n_ids rows of n_ratios radius ratios (outer/ring). */
cctagb_status cctagb_set_bank(cctagb_handle* h, const float* ratios, int n_ids, int n_ratios);

/* Full detection of one 8-bit gray frame held in host memory. */
cctagb_status cctagb_detect(cctagb_handle* h, const uint8_t* gray, int w, int hgt, size_t pitch, int frame_id,
                            cctagb_marker* out, int cap, int* n_out, cctagb_stats* stats);

/* Same, with the frame already in device memory (pitch in bytes). */
cctagb_status cctagb_detect_device(cctagb_handle* h, const uint8_t* d_gray, int w, int hgt, size_t pitch,
                                   int frame_id, cctagb_marker* out, int cap, int* n_out, cctagb_stats* stats);

/* One frame of a batch: input view, caller-owned output array, and what the
 * call wrote back for this frame. */
typedef struct cctagb_frame {
    const uint8_t* gray;       /* host or device pointer (is_device)   */
    int w, h;
    size_t pitch;              /* bytes between rows                   */
    int frame_id;
    int is_device;
    cctagb_marker* out;        /* cap entries                          */
    int cap;
    int n_out;                 /* written: markers returned            */
    cctagb_status status;      /* written: this frame's status         */
    cctagb_stats stats;        /* written: this frame's statistics     */
} cctagb_frame;

/* Detection of n independent frames (cameras), of any sizes up to the
 * handle's max_w x max_h.  Frames go in waves of params.batchWaveFrames: the
 * image stages (pyramid .. seeds) of a wave's frames run as one launch per
 * kernel over all their levels, then each frame continues on its own
 * detection slot (device buffers and stream); min(max_batch, 32) slots keep
 * several waves in flight, so later waves' image stages overlap earlier
 * frames' GPU and host stages.  Every frame's result equals that of
 * cctagb_detect on the same frame.  Returns CCTAGB_OK when every frame
 * succeeded, else the status of the first failing frame (last_error_string
 * names it); per-frame statuses are in frames[i].status.  The reference runs
 * one frame per cctagDetection call (ICCTag.hpp:125-131); this is the
 * multi-camera form of that call. */
cctagb_status cctagb_detect_batch(cctagb_handle* h, cctagb_frame* frames, int n);

/* ---- Streaming ingest ----------------------------------------------------
 * For cameras that deliver a frame at a time.  The reference keeps page-locked
 * frame buffers and uploads them asynchronously (cuda/frame.cu:110-148); here
 * the handle owns pinned buffers the caller may fill, and cctagb_submit queues
 * a frame on the detection slots (min(max_batch, 32) of them) and returns at
 * once, so that one frame's upload and GPU stages overlap another frame's
 * host stage.  cctagb_wait(ticket) returns that frame's markers, exactly what
 * cctagb_detect returns for it.  The frame memory must stay valid until its
 * ticket has been waited for.  When `cap` is smaller than the frame's marker
 * count, cctagb_wait returns CCTAGB_BAD_ARG with *n_out set to that count and
 * keeps the ticket, so the caller can wait on it again with a larger buffer.  While tickets are outstanding, every other
 * call that uses the handle's detection slots returns CCTAGB_BAD_ARG. */

/* n (<= 64) pinned host buffers of max_w * max_h bytes owned by the handle
 * (kept across calls; freed by cctagb_destroy); out[i] receives buffer i. */
cctagb_status cctagb_host_frames(cctagb_handle* h, int n, uint8_t** out);

cctagb_status cctagb_submit(cctagb_handle* h, const uint8_t* gray, int w, int hgt, size_t pitch, int is_device,
                            int frame_id, int* ticket);

/* Blocks until the ticket's detection is done; the ticket is then released.
 * A frame's failure is returned here (and named by last_error_string). */
cctagb_status cctagb_wait(cctagb_handle* h, int ticket, cctagb_marker* out, int cap, int* n_out,
                          cctagb_stats* stats);

/* Image stage only (pyramid, derivatives, Canny, thinning, edge points, vote,
 * seeds) on the handle's stream; results stay on the device and are read with
 * the cctagb_level_* calls.  d_gray may be a device or a host pointer
 * (is_device says which). */
cctagb_status cctagb_image_stage(cctagb_handle* h, const uint8_t* gray, int w, int hgt, size_t pitch, int is_device);

/* Per-level results of the last image stage (host copies). */
cctagb_status cctagb_level_size(cctagb_handle* h, int level, int* w, int* hgt);
cctagb_status cctagb_level_planes(cctagb_handle* h, int level, uint8_t* src, int16_t* dx, int16_t* dy,
                                  uint8_t* edges);
cctagb_status cctagb_level_edge_points(cctagb_handle* h, int level, int cap, int* n, int32_t* x, int32_t* y);
cctagb_status cctagb_level_links(cctagb_handle* h, int level, int cap, int32_t* before, int32_t* after);
cctagb_status cctagb_level_votes(cctagb_handle* h, int level, int cap, int32_t* chosen, int32_t* nvotes,
                                 float* flow_length, int32_t* voter_off, int32_t* voter_list, int voter_cap,
                                 int32_t* n_voters);
/* Seeds in the reference's processing order (push order, then std::sort by votes). */
cctagb_status cctagb_level_seeds(cctagb_handle* h, int level, int cap, int32_t* seeds, int* n);

/* Loop-one candidates of level `level` in the last cctagb_detect /
 * cctagb_detect_device call: the first maximumNbCandidatesLoopTwo of them in
 * loop-one order (Detection.cpp:609-627), after the children collection and
 * the LMedS outlier removal of loop two (Detection.cpp:115-156, Vote.cpp:
 * 396-576), as the GPU computed them.  Per candidate: seed (edge-point index),
 * score (number of children, 0 when too few), keep (1 when it goes on to the
 * ellipse growing) and, for kept candidates, the number of filtered children;
 * `filtered` receives the kept candidates' filtered children one after the
 * other.  These lists are locals of cctagDetectionFromEdges in the reference;
 * the call exposes them for parity checks. */
cctagb_status cctagb_level_loop_two(cctagb_handle* h, int level, int cap, int32_t* seed, int32_t* score,
                                    int32_t* keep, int32_t* n_filtered, int* n, int filtered_cap,
                                    int32_t* filtered, int* n_filtered_total);

/* The CUDA stream (cudaStream_t) on which the handle launches its work, so a
 * caller can order its own work or CUDA events against it. */
cctagb_status cctagb_get_stream(cctagb_handle* h, void** stream);

/* Per-stage device timing of the image stage: when enabled, CUDA events are
 * captured between the stages and cctagb_stage_times returns the last frame's
 * milliseconds per stage (names from cctagb_stage_name). */
cctagb_status cctagb_set_stage_timing(cctagb_handle* h, int enable);
cctagb_status cctagb_stage_times(cctagb_handle* h, int cap, float* ms, int* n);
const char* cctagb_stage_name(int stage);

/* Canny NMS + hysteresis + thinning from caller-given derivatives (host
 * arrays, w*hgt int16 each); edges out as 0/255 bytes. */
cctagb_status cctagb_canny_from_derivatives(cctagb_handle* h, const int16_t* dx, const int16_t* dy, int w, int hgt,
                                            uint8_t* edges);

/* Edge stage of one frame without any device allocation.  No counterpart in
 * the reference: it is for callers that cannot allocate device memory when
 * they need edges (all memory handed to their own pool, or a real-time loop
 * that forbids cudaMalloc/cudaFree after start-up), and it needs no handle.
 * d_gray (w*hgt bytes, pitch == w), d_dx, d_dy (w*hgt int16 each) and d_edges
 * (w*hgt bytes, 0/255) are device buffers owned by the caller; d_status (one
 * int, may be null) receives 0 or an internal error bit.  Runs asynchronously
 * on `stream` (a cudaStream_t; null = legacy default stream).  Its scratch is a
 * fixed device array inside the library (about 2.5 MB on every GPU that loads
 * it): frames are limited to 1,048,576 pixels and 4096 per side
 * (CCTAGB_TOO_LARGE beyond).  The first call on a device (in each CUDA
 * context) sets the array up (resolves its device address) with that device
 * current: make it before any stream capture.  Calls share the array: calls whose GPU
 * work overlaps race; serialise them on one stream. */
cctagb_status cctagb_edges_noalloc(const uint8_t* d_gray, int w, int hgt, size_t pitch, float cannyThrLow,
                                   float cannyThrHigh, int16_t* d_dx, int16_t* d_dy, uint8_t* d_edges,
                                   int32_t* d_status, void* stream);

/* ---- Identification of candidate markers (batched form) -----------------
 * The reference identifies each candidate inside cctagDetection
 * (Identification.cpp:1172-1480 identify: cut collection and selection, then
 * refineConicFamilyGlob :813-965 and the ID vote).  These calls expose the
 * second half on caller-given candidates, many per call, on one device image
 * (one frame, or an atlas of crops with one rectangle per candidate). */

#define CCTAGB_MAX_CUTS 32

/* One candidate: what identify_step_1 (cut selection) hands to the
 * refinement.  Coordinates are image pixels of the whole device image. */
typedef struct cctagb_cut_task {
    float Q[9];                     /* outer ellipse conic, row-major              */
    float cx, cy, a, b, angle;      /* its parameters                              */
    float x0, y0;                   /* initial imaged center (centerImg)           */
    int ncuts;                      /* selected cuts, <= CCTAGB_MAX_CUTS           */
    float stop[CCTAGB_MAX_CUTS][2]; /* cut end points on the outer edge            */
    int roi[4];                     /* x, y, w, h: the candidate's image rectangle;
                                       a sample outside it drops its cut, as the
                                       image border does in the reference        */
    int local;                      /* 0: Q, cx, cy, x0, y0 and stop are image
                                       coordinates; nonzero: they are relative to
                                       the rectangle's corner (roi[0], roi[1]),
                                       and so are the results.  Candidates from
                                       a large atlas keep their FP32 positions
                                       as precise as in a frame that way.         */
} cctagb_cut_task;

typedef struct cctagb_ident_result {
    int status;                     /* CCTAGB_ID_RELIABLE, _ID_NOT_RELIABLE, _OPTI_HAS_DIVERGED */
    int id;                         /* bank row, -1 if none                        */
    float x, y;                     /* refined imaged center                       */
    float H[9];                     /* marker plane -> image at (x, y), row-major  */
    float residual;                 /* sqrt(cost) / barcode range                  */
    float score;                    /* mean probability of the winning id          */
    int nvalid;                     /* cuts inside the rectangle at the end        */
    int iterations;                 /* grid rounds + Gauss-Newton evaluations      */
} cctagb_ident_result;

/* The identification tasks of the last cctagb_detect / cctagb_detect_device
 * call on this handle (the candidates whose cut selection succeeded, in the
 * order they were identified); *n receives their number. */
cctagb_status cctagb_last_tasks(cctagb_handle* h, cctagb_cut_task* out, int cap, int* n);

/* Center refinement and ID reading of n candidates on the device image d_img
 * (w x hgt, pitch bytes per row).  refine_mode CCTAGB_REFINE_GRID is the
 * reference's shrinking 5x5 grid; CCTAGB_REFINE_GAUSS_NEWTON runs the first
 * params.gnCoarseRounds grid rounds, then Levenberg-Marquardt steps on the cut-consistency
 * cost with the center Jacobian from forward derivatives of the homography
 * (params.gnIterations evaluations at most).  tasks and out are host arrays. */
cctagb_status cctagb_identify_tasks(cctagb_handle* h, const uint8_t* d_img, int w, int hgt, size_t pitch,
                                    const cctagb_cut_task* tasks, int n, int refine_mode,
                                    cctagb_ident_result* out);

/* The cut-consistency cost (costFunctionGlob, Identification.cpp:1122-1158)
 * of each task at the imaged center centers[2i], centers[2i+1], with its
 * gradient with respect to the center (d_center, 2 per task) and to the nine
 * entries of the homography H (d_h, 9 per task, row-major; the cut end points
 * are back-projected through H, so both uses of H are differentiated).  Any
 * of cost, d_center, d_h may be null.  A cut with a sample outside its task's
 * rectangle is left out; with fewer than two cuts the cost is FLT_MAX and the
 * gradients are zero.  All arrays are host arrays. */
cctagb_status cctagb_cut_cost(cctagb_handle* h, const uint8_t* d_img, int w, int hgt, size_t pitch,
                              const cctagb_cut_task* tasks, int n, const float* centers, float* cost,
                              float* d_center, float* d_h);

/* cctagb_cut_cost with every step in double precision on the GPU (canonic
 * form, homography and its center derivatives, cut ends, sample positions,
 * bilinear reads, sums).  It has no counterpart in the reference: it exists
 * to check the adjoint against central differences below the ~1e-4 relative
 * noise that FP32 sample positions put on the cost.  Same arguments. */
cctagb_status cctagb_cut_cost_f64(cctagb_handle* h, const uint8_t* d_img, int w, int hgt, size_t pitch,
                                  const cctagb_cut_task* tasks, int n, const float* centers, float* cost,
                                  float* d_center, float* d_h);

/* ---- batch autotuning ---------------------------------------------------- */

#define CCTAGB_TUNE_MAX_TRIED 16

/* A batch configuration and how it was chosen. */
typedef struct cctagb_tune_choice {
    int batchWaveFrames;       /* frames per batched image-stage launch   */
    int identLayout;           /* CCTAGB_IDENT_AUTO / CCTAGB_IDENT_BLOCK   */
    float ms_per_frame;        /* median batch time / frames, when measured */
    int from_cache;            /* 1: read from the cache file; 0: measured by this call */
    int n_tried;               /* configurations measured by this call    */
    int tried_wave[CCTAGB_TUNE_MAX_TRIED];
    int tried_layout[CCTAGB_TUNE_MAX_TRIED];
    float tried_ms_per_frame[CCTAGB_TUNE_MAX_TRIED];
    int hostThreads;           /* host worker pool size (params.hostThreads) */
    int tried_threads[CCTAGB_TUNE_MAX_TRIED];
} cctagb_tune_choice;

/* Picks the configuration of cctagb_detect_batch (params.batchWaveFrames,
 * params.identLayout, then the host pool size params.hostThreads) for this
 * handle's GPU, the frames' size and count and the number of crowns, and sets
 * it on the handle.  With a cache file that
 * holds an entry for that key (cctagb_tune_key), the entry is used; otherwise
 * every candidate configuration detects the given frames `reps` times (after
 * one untimed call) and the one with the least median time wins, and is
 * written to the cache file when cache_path is not NULL.  Frames of several
 * sizes are keyed by their total pixel count.  When measuring, the frames'
 * markers and statistics are written as by cctagb_detect_batch. */
cctagb_status cctagb_autotune(cctagb_handle* h, cctagb_frame* frames, int n, const char* cache_path, int reps,
                              cctagb_tune_choice* out);

/* Cache key of a configuration: the GPU's name and SM count, the frame size,
 * frames per call, crowns and the cache format version.  Host only. */
cctagb_status cctagb_tune_key(const char* gpu_name, int sm_count, int w, int hgt, int frames, int nCrowns, char* out,
                              int cap);
/* The cache is a JSON object {"version": V, "entries": {key: {...}}}.
 * cctagb_tune_cache_get returns CCTAGB_OK and fills *out (from_cache = 1) when
 * the file holds the key; CCTAGB_BAD_ARG when the file or key is absent, of
 * another version or malformed.  cctagb_tune_cache_put adds or replaces the
 * key's entry (other entries are kept) by writing a temporary file and
 * renaming it over the cache file.  Host only. */
cctagb_status cctagb_tune_cache_get(const char* cache_path, const char* key, cctagb_tune_choice* out);
cctagb_status cctagb_tune_cache_put(const char* cache_path, const char* key, const cctagb_tune_choice* c);

#ifdef __cplusplus
}
#endif

#endif /* CCTAG_B200_H */
