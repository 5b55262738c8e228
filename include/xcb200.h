/*
 * xcb200.h -- C ABI of the B200-native xclean hot path (libxcb200.so, sm_100a).
 *
 * The reference has no native library: its boundary is Python (src/xclean/front/gpu_front.py for the frontend,
 * src/xclean/backend/{kernels,ba}.py for the bundle adjustment).  These entry points sit UNDER those Python
 * signatures; the ctypes bindings in xclean_b200/front/gpu_front.py and xclean_b200/backend/*.py call them.  Each
 * declaration names the reference interface it replaces.  Plain pointers and sizes only; "host" entry points take host
 * memory, "dev" entry points take device memory and a cudaStream_t (as void*, NULL = the handle's own stream).
 *
 * Every function returns an xcb status (0 = ok).  A failure never aborts the process: the message is kept in the
 * handle (xcb_front_last_error / xcb_ba_last_error) or, for handle-free calls, in a thread-local (xcb_last_error).
 */
#ifndef XCB200_H
#define XCB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define XCB_OK 0
#define XCB_ERR_ARG (-1)          /* bad argument (size, null pointer, unsupported option) */
#define XCB_ERR_CUDA (-2)         /* a CUDA runtime call failed */
#define XCB_ERR_CAPACITY (-3)     /* more data than the buffers allocated at creation hold (gpu_front.py:1398, :1403) */
#define XCB_ERR_NOT_CALIBRATED (-4)
#define XCB_ERR_DEVICE (-5)       /* a kernel reported an error word (bounded loop ran out, overflow) */

/* device error word bits (set by kernels, read back by the host after each call) */
#define XCB_DEVERR_GREEDY_ROUNDS 1u
#define XCB_DEVERR_STEREO_SMEM 2u
#define XCB_DEVERR_CHOL_NOT_PD 4u

const char* xcb_last_error(void);
int xcb_version(void);

/* ===================================================== frontend ===================================================== */
typedef struct xcb_front xcb_front;

/* Device buffers of a front, frame-major with per-frame capacity `cap` (the pipeline's outputs). */
typedef struct {
    int32_t* counts;   /* [F] keypoints per frame */
    float* kp;         /* [F][cap][2] sub-pixel keypoints */
    uint8_t* desc;     /* [F][cap][32] ORB descriptors */
    double* d;         /* [F][cap] disparity (0 unless ok) */
    double* sig;       /* [F][cap] disparity sigma (inf unless ok) */
    uint8_t* ok;       /* [F][cap] */
    double* zn;        /* [F][cap] peak ZNCC */
    double* dy;        /* [F][cap] column-scan vertical offset (NaN unless set) */
    int64_t* m0;       /* [F][cap] matches of frame f-1 (query) ... */
    int64_t* m1;       /* [F][cap] ... to frame f (train) */
    int32_t* nmatch;   /* [F] */
    double* floor;     /* [F] noise floor (float64) */
    int32_t* anypos;   /* [F] any response > 0 */
} xcb_front_bufs;

/* GpuFront.__init__ (gpu_front.py:1076-1198): all device and pinned buffers for W x H frames, `cap` keypoints per
   frame, up to `max_frames` frames per batched call; one stream. */
int xcb_front_create(int width, int height, int cap, int max_frames, xcb_front** out);
/* GpuFront teardown / release_device (gpu_front.py:1653-1686): frees every buffer; the CUDA context is kept. */
void xcb_front_destroy(xcb_front* f);
const char* xcb_front_last_error(const xcb_front* f);
/* GpuFront.pool_bytes (gpu_front.py:1570): device bytes held by the front */
size_t xcb_front_device_bytes(const xcb_front* f);
/* GpuFront.calibrate results (gpu_front.py:1423-1513): SIMD split points of cv2's Sobel and ORB blur, the float32
   Gaussian taps, the 256 ORB test pairs (x1, y1, x2, y2 as int8) and the noise quantile features._NOISE_Q99. */
int xcb_front_set_calibration(xcb_front* f, int dy_vend, int dx_vend, int blur_vr, int blur_vc, const float* kf7,
                              const int8_t* pattern, double noise_q99);
/* GpuFront._response (gpu_front.py:1227-1238; k_sobel/k_boxrows/k_boxcols/k_eig): the calibration probe form,
   with explicit split points.  gray [H][W] -> R [H][W] float32. */
int xcb_front_response_host(xcb_front* f, const uint8_t* gray, int dy_vend, int dx_vend, float* R);
/* GpuFront._noise_floor (gpu_front.py:1240-1247): -> floor (float64) */
int xcb_front_noise_floor_host(xcb_front* f, const uint8_t* gray, double* floor_out);
/* GpuFront._describe_dev blur stage (gpu_front.py:1319-1325) as the calibration probe: -> [H+64][W+64] u8 */
int xcb_front_blur_host(xcb_front* f, const uint8_t* gray, int blur_vr, int blur_vc, uint8_t* out);
/* GpuFront.detect (gpu_front.py:1250-1317) for `nframes` frames of one budget: gray [F][H][W] -> counts [F],
   kp [F][cap][2], desc [F][cap][32], floor [F], anypos [F] */
int xcb_front_detect_host(xcb_front* f, const uint8_t* gray, int nframes, int budget, int32_t* counts, float* kp,
                          uint8_t* desc, double* floor_out, int32_t* anypos);
/* GpuFront.describe_points (gpu_front.py:1556-1568): ORB of given keypoints */
int xcb_front_describe_host(xcb_front* f, const uint8_t* gray, const float* kp, int n, uint8_t* desc);
/* GpuFront.stereo (gpu_front.py:1342-1383; k_shift/k_tof + k_stereo), patch half-size `half` in {3, 4, 5}
   (5 = the reference).  kp [n][2] float64, dlo/dhi [n] int64 -> d, sig, ok, zn, ody [n] */
int xcb_front_stereo_host(xcb_front* f, const uint8_t* left, const uint8_t* right, const double* kp,
                          const int64_t* dlo, const int64_t* dhi, int n, double dy, int band, int half, double* d,
                          double* sig, uint8_t* ok, double* zn, double* ody);
/* GpuFront.hamming (gpu_front.py:1386-1420; k_ham_rows/k_ham_cols): A [L][32], B [N][32] -> row best, second,
   index (first minimum) and column best index */
int xcb_front_hamming_host(xcb_front* f, const uint8_t* A, int L, const uint8_t* B, int N, int32_t* b1, int32_t* b2,
                           int32_t* bi, int32_t* ci);
/* match_desc_gpu (gpu_front.py:1871-1893) with the epilogue on the device: mutual NN, b1 <= ham_max,
   b1 < ratio * b2 -> i0, i1 in query order */
int xcb_front_match_host(xcb_front* f, const uint8_t* A, int L, const uint8_t* B, int N, int ham_max, double ratio,
                         int64_t* i0, int64_t* i1, int32_t* nmatch);
/* GpuFront.check_lk_solver's k_lkcheck (gpu_front.py:1515-1554, :707-719): device 3x3 solve + inverse */
int xcb_front_lk_check_host(xcb_front* f, const double* As, const double* gs, int n, double* X, double* Inv);

/* The per-frame hot path for a batch, on device memory (no reference counterpart as one call: it is
   Detector.__call__ + disparities + match_desc_gpu of engine_live.P1Engine._step, engine_live.py:993-999, :837-845,
   :1599-1609, for `nframes` frames in one launch sequence, replayed from a CUDA graph).  left/right [F][H][W].
   Frame f's descriptors are matched against frame f-1's; frame 0 against the previous call's last frame when
   match_prev != 0.  Results stay in the front's device buffers (xcb_front_buffers). */
int xcb_front_pipeline_dev(xcb_front* f, const uint8_t* left, const uint8_t* right, int nframes, int budget, int half,
                           int dlo, int dhi, int match_prev, void* stream);
int xcb_front_buffers(xcb_front* f, xcb_front_bufs* out);
/* the same from host memory (H2D, pipeline, D2H of every non-NULL result array into the host arrays of `out`, then a
   wait on `stream`); host buffers in page-locked memory make the copies asynchronous */
int xcb_front_pipeline_host(xcb_front* f, const uint8_t* left, const uint8_t* right, int nframes, int budget,
                            int half, int dlo, int dhi, int match_prev, const xcb_front_bufs* out, void* stream);
/* number of kernel launches the last pipeline call issued */
int xcb_front_last_launches(const xcb_front* f);
/* wait for `stream` (NULL = the front's own) and read the device error word -> XCB_OK or XCB_ERR_DEVICE */
int xcb_front_sync_check(xcb_front* f, void* stream);
/* Stage timing of the batched pipeline (no reference counterpart; the reference times stages on the host with
   obs/latency.Ledger, latency.py:177-212): when on, every captured pipeline graph records an event at each stage
   boundary.  xcb_front_stage_times sums, over the graphs replayed since the last read, the device time of each stage:
   0 response, 1 noise floor, 2 thresholds + candidate lists, 3 greedy + rank + sub-pixel, 4 blur + ORB,
   5 stereo, 6 Hamming + match.  Call after the stream has been synchronised. */
#define XCB_FRONT_STAGES 7
int xcb_front_set_stage_timing(xcb_front* f, int on);
int xcb_front_stage_times(xcb_front* f, float* ms, int* ngraphs);

/* ============================================== sliding-window bundle adjustment ============================================== */
/* A batch of windows of the reference's stereo window solve (src/xclean/vio/window.py: Problem :768-792, solve
   :889-982), concatenated: window w owns slots [slot_off[w], slot_off[w] + P[w]) and landmarks [lm_off[w],
   lm_off[w] + L[w]); landmark l's observation rows are [lm_ob[l], lm_ob[l + 1]) (at most 32), its host and the
   rows' poses are window-local slot indices.  All pointers are device memory. */
typedef struct {
    int nw;                     /* windows */
    const int32_t* P;           /* [nw] slots (<= 20) */
    const int32_t* L;           /* [nw] landmarks */
    const int32_t* slot_off;    /* [nw] */
    const int32_t* lm_off;      /* [nw] */
    const int32_t* hold;        /* [nw] slot held fixed (-1 none), or NULL */
    const int32_t* order;       /* [nw] processing order (largest first), or NULL */
    const double* cam;          /* [nw][6] fx fy cx cy B huber_k */
    const double* ext;          /* [nw][12] Rbc (row-major) pbc */
    double* Rwb;                /* [S][9] in / out */
    double* pwb;                /* [S][3] in / out */
    double* lmp;                /* [Lt][3] (a, b, rho) in / out */
    const int32_t* lm_host;     /* [Lt] */
    const uint8_t* lm_mask;     /* [Lt] */
    const double* rho_meas;     /* [Lt] */
    const double* rho_isig;     /* [Lt] */
    const int32_t* lm_ob;       /* [Lt + 1] */
    const int32_t* ob_pose;     /* [Mt] */
    const uint8_t* ob_cam;      /* [Mt] 0 = left (u, v), 1 = right u_R */
    const double* ob_z;         /* [Mt][2] */
    const double* ob_isig;      /* [Mt] */
    const uint8_t* ob_valid;    /* [Mt] */
} xcb_ba_windows;

#define XCB_BA_FP64 0           /* everything in float64: the plain form */
#define XCB_BA_MIXED 1          /* FP32 linearisation + Schur, FP64 Cholesky, one FP64 refinement step */

/* Device scratch the batched solve needs for `Lt` landmarks (trial landmark states and the work counter). */
size_t xcb_ba_scratch_bytes(int nw, int Lt);
/* window.solve (window.py:889-982, purely visual, fixed `iters` LM iterations from lam0) for every window of the batch
   in ONE persistent launch (no reference counterpart as one call; the reference solves one window per call on the
   CPU).  stats [nw][8] = cost0, cost, accepted, lam, status (0 ok, -1 window too large), iters, -, -;
   dx0 [nw][dx0_stride] (optional) = the first iteration's pose step.  grid = 0: one CTA per SM. */
int xcb_ba_solve_windows_dev(const xcb_ba_windows* w, int max_slots, int iters, double lam0, int mode, double* stats,
                             double* dx0, int dx0_stride, void* scratch, size_t scratch_bytes, int grid, void* stream);

/* Allocation-free form of xcb_ba_solve_windows_dev.  No counterpart in the reference.  It is for callers that cannot
   call cudaMalloc while running: a real-time loop whose latency budget rules out an allocation (which may synchronise
   the device), or a plugin whose host owns the device memory through its own allocator.  The caller passes inputs and
   outputs as for xcb_ba_solve_windows_dev but no scratch: the scratch is a static device array of
   XCB_BA_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until exit, which limits one call to
   xcb_ba_noalloc_max_landmarks() landmarks in total (`Lt`, the batch's landmark count; more -> XCB_ERR_CAPACITY).
   The first call on a device looks up the array's device address (call it before any stream capture).  Calls share
   the array: calls that overlap on the GPU race.  No cudaMalloc, cudaFree or allocating library call is made. */
#define XCB_BA_NOALLOC_SCRATCH_BYTES ((size_t)4 << 20)
#define XCB_NOALLOC_MAX_DEVICES 64
int xcb_ba_noalloc_max_landmarks(void);
int xcb_ba_solve_windows_noalloc(const xcb_ba_windows* w, int Lt, int max_slots, int iters, double lam0, int mode,
                                 double* stats, double* dx0, int dx0_stride, int grid, void* stream);

#ifdef __cplusplus
}
#endif
#endif
