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

/* Launch-shape knobs chosen per (device, workload shape) by the package's autotuner (xclean_b200/tune.py); no
   reference counterpart (the reference's launch shapes are constants).  0 = the built-in default. */
#define XCB_TUNE_MM_LANES 1       /* map matcher gate: lanes per landmark, 1, 2, 4 or 8 (default 2) */
#define XCB_TUNE_STEREO_WARPS 2   /* stereo: warps (point groups) per block, 1..8 (default 8; 6 for the 11x11 window) */
#define XCB_TUNE_STEREO_GROUP 3   /* stereo: points per warp, searched one after another, LKs one per lane, 1..32 */
#define XCB_TUNE_KNOBS 4

/* device error word bits (set by kernels, read back by the host after each call) */
#define XCB_DEVERR_GREEDY_ROUNDS 1u
#define XCB_DEVERR_STEREO_SMEM 2u
#define XCB_DEVERR_CHOL_NOT_PD 4u
#define XCB_DEVERR_TC_WAIT 8u          /* a tensor-core completion wait ran out (the kernel gave up, results invalid) */

const char* xcb_last_error(void);
int xcb_version(void);
/* The FP64 (fp64 = 1) or FP32 FMA peak of this device at its current clocks: one timed launch of 8 independent FMA
   chains per thread, 8 blocks of 256 threads per SM, `iters` steps per chain (65536 takes ~10 ms in FP64).  No
   reference counterpart: the compute rooflines of the window BA and of the stereo's LK are quoted against it.
   tflops: FLOP/s / 1e12 (an FMA counts 2); ms (may be NULL): the launch's duration.  Synchronises the device. */
int xcb_peak_fma(int fp64, int iters, double* tflops, float* ms);

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
   frame, up to `max_frames` frames per batched call; one stream.  48 <= width <= 8192, 48 <= height <= 65535. */
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
/* xcb_front_pipeline_host over `nframes` frames in batches of `batch` (<= max_frames), the results of every batch
   going to its frames' rows of `out` (arrays for all `nframes` frames); batch b's frames are matched as by
   consecutive xcb_front_pipeline_host calls (batch 0 against the previous call's last frame when match_prev != 0).
   No reference counterpart as one call: the reference uploads and processes frame by frame.  The next batch's
   frames are copied in on a second stream into a second input buffer pair while the current batch computes, and
   each batch's results are copied on the device into one of two staging blocks and read back on a third stream
   while the next batch computes (page-locked `left` / `right` / `out` make the copies overlap); the first call
   allocates the buffers, the streams and the events. */
int xcb_front_pipeline_host_batches(xcb_front* f, const uint8_t* left, const uint8_t* right, int nframes, int batch,
                                    int budget, int half, int dlo, int dhi, int match_prev, const xcb_front_bufs* out,
                                    void* stream);
/* number of kernel launches the last pipeline call issued */
int xcb_front_last_launches(const xcb_front* f);
/* Set a launch-shape knob of this front (XCB_TUNE_STEREO_*; no reference counterpart): later calls launch with it;
   the captured pipeline graphs are dropped and re-captured on their next use.  Results do not depend on it. */
int xcb_front_set_tuning(xcb_front* f, int knob, int value);
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

/* ================================================ gated map matching ================================================ */
/* Landmarks of the window, projected with the predicted pose, matched to the frame's keypoints inside the chi2 ellipse
   of their innovation covariance: minimum Hamming distance over the landmark's descriptors, chance bound 104, Lowe
   ratio 0.8 against the second-best in-gate distance, then one landmark per keypoint (smaller distance, then smaller
   Mahalanobis d2, then lower landmark index).  Outputs per landmark: keypoint index or -1, Hamming distance (9999 when
   rejected at the gate), Mahalanobis d2 (inf when rejected at the gate); a landmark that loses the one-per-keypoint
   step keeps its distance and d2 and gets index -1, as in the reference. */
/* ============================================== dense 32-direction SGM ============================================== */
/* The reference's dense stereo (src/xclean/stereo/sgm32.py SGM32, CuPy kernels :105-266, launches :333-360):
   census 9x9 -> Hamming cost volume -> one 32-direction aggregation into a uint16 volume -> left winner with
   uniqueness and parabola -> right winner off the same volume -> left-right check; disp 0 = invalid.  Bit for bit
   the reference's outputs.  A handle serves one image size (width <= 2048) and owns its volumes (W x H x 384 B). */
typedef struct xcb_sgm xcb_sgm;
int xcb_sgm_create(int width, int height, int p1, int p2, float uniqueness, float lr_threshold, float min_disp,
                   xcb_sgm** out);                              /* SGM32.__init__ (sgm32.py:278-320) */
void xcb_sgm_destroy(xcb_sgm* s);
const char* xcb_sgm_last_error(const xcb_sgm* s);
/* SGM32.compute_gpu (sgm32.py:333-360): left / right (H x W u8) and disp / conf (H x W float32) in device memory;
   launches on `stream` (NULL = the handle's stream), no synchronisation */
int xcb_sgm_compute_dev(xcb_sgm* s, const uint8_t* left, const uint8_t* right, float* disp, float* conf, void* stream);
/* SGM32.compute (sgm32.py:362-368): host arrays in and out, synchronous */
int xcb_sgm_compute_host(xcb_sgm* s, const uint8_t* left, const uint8_t* right, float* disp, float* conf);
/* the handle's device volumes after the last call (SGM32.cost_volume / aggregated_volume, sgm32.py:370-376): cost
   [H][W][128] u8, sum [H][W][128] u16; npaths: the aggregation's paths over the 32 directions */
int xcb_sgm_buffers(xcb_sgm* s, void** cost, void** sum, int* npaths);
/* the same volumes copied to host memory (either may be NULL); waits for the handle's stream and the device */
int xcb_sgm_read_volumes(xcb_sgm* s, uint8_t* cost, uint16_t* sum);
/* in-stream stage timing (no reference counterpart; the bench's per-kernel roofline): when on, each compute records
   events around the cost kernel, the aggregation (with the zeroing of the sum volume) and the selection;
   xcb_sgm_stage_times returns ms[3] summed over the calls since its last call (at most the last 256) and waits for them */
int xcb_sgm_set_stage_timing(xcb_sgm* s, int on);
int xcb_sgm_stage_times(xcb_sgm* s, float* ms, int* ncalls);

/* ============================ multi-scale oriented ORB: pyramid, FAST, orientation, steered rBRIEF ============================
   Beyond the reference, whose frontend is single-scale Shi-Tomasi with unoriented ORB (src/xclean/stages/features.py:27-28,
   :102-103; src/xclean/front/gpu_front.py:1712-1717, where ORB is created with nlevels=1 and KeyPoint.angle 0).  No
   reference entry point is replaced; the per-level descriptor is the reference's Frontend.describe (features.py:405-421:
   cv2 ORB on the reflect-101 pad-32 image) with the pattern rotated, and level 0 at bin 0 is that descriptor bit for bit.
   Every device pointer below is device memory; `stream` NULL = the legacy default stream (primitives) or the handle's. */
/* FAST 9-of-16 with the score cv2.FastFeatureDetector gives (TYPE_9_16): keypoints (x, y) in row-major order and
   their scores; with nonmax, only corners whose score beats all 8 neighbours'.  count (device int): the number found,
   of which the first `cap` are written.  scratch: device bytes, at least xcb_fast_scratch_bytes(width, height). */
size_t xcb_fast_scratch_bytes(int width, int height);
int xcb_fast_dev(const uint8_t* img, int width, int height, int threshold, int nonmax, int cap, float* kp, float* resp,
                 int32_t* count, void* scratch, size_t scratch_bytes, void* stream);
/* of the first min(*n_in, cap_in) keypoints, those at least `edge` px inside width x height: the `quota` best by score,
   ties in input order, written in input order; *count = how many */
int xcb_fast_select_dev(const float* kp_in, const float* resp_in, const int32_t* n_in, int cap_in, int width, int height,
                        int edge, int quota, float* kp, float* resp, int32_t* count, void* stream);
/* bilinear downsampling of n_src samples to n_dst = cv2.resize(INTER_LINEAR_EXACT): per destination sample the source
   index and an 8-bit weight (host arrays of n_dst) */
int xcb_pyr_tables(int n_src, int n_dst, int32_t* idx, int32_t* w);
int xcb_pyr_down_dev(const uint8_t* src, int ws, int hs, uint8_t* dst, int wd, int hd, const int32_t* x0,
                     const int32_t* wx, const int32_t* y0, const int32_t* wy, void* stream);
/* orientation: the intensity centroid over the disc u^2 + v^2 <= 240 (radius 15) -> bin k of 30 (centre 12 k degrees,
   image axes); host tables umax[16], boundary directions bdir[30][2] and centres cdir[30][2] */
int xcb_orient_tables(int32_t* umax, double* bdir, double* cdir);
int xcb_ic_bins_dev(const uint8_t* img, int width, int height, const float* kp, int n, const int32_t* count,
                    const int32_t* umax, const double* bdir, const double* cdir, int32_t* bins, int64_t* moments,
                    void* stream);              /* count: optional device count (min(*count, n) keypoints) */
/* steered rBRIEF on a blurred image padded by `pad`: patterns [30][256][4] int8 (x1, y1, x2, y2) rotated per bin */
int xcb_orb_steered_dev(const uint8_t* blur, int wp, int hp, int pad, const float* kp, int n, const int32_t* count,
                        const int32_t* bins, const int8_t* patterns, uint8_t* desc, void* stream);
/* the ORB blur of the reference's describe stage (reflect-101 pad 32, 7x7 Gaussian sigma 2 in OpenCV's float
   arithmetic with the SIMD split points vr / vc of this width): width x height -> (height + 64) x (width + 64); kf7
   device taps */
int xcb_blur_dev(const uint8_t* img, int width, int height, const float* kf7, int vr, int vc, uint8_t* out,
                 void* stream);
/* the per-frame handle: `levels` levels at `scale` (sizes rint(n / scale^l)), FAST at fast_threshold on each, per
   level a geometric share of nfeatures (the best by score at least `edge` >= 16 px inside), orientation bins, the level's
   blur and steered descriptors.  Outputs in nfeatures slots, level l's from its offset (xcb_orbx_level). */
typedef struct xcb_orbx xcb_orbx;
int xcb_orbx_create(int width, int height, int levels, double scale, int nfeatures, int fast_threshold, int edge,
                    int nonmax, xcb_orbx** out);
void xcb_orbx_destroy(xcb_orbx* h);
const char* xcb_orbx_last_error(const xcb_orbx* h);
int xcb_orbx_level(const xcb_orbx* h, int level, int* width, int* height, float* scale, int* quota, int* offset);
int xcb_orbx_set_blur(xcb_orbx* h, int level, int vr, int vc, const float* kf7);      /* host taps */
int xcb_orbx_set_patterns(xcb_orbx* h, const int8_t* patterns);                       /* host [30][256][4] */
int xcb_orbx_detect_dev(xcb_orbx* h, const uint8_t* img, void* stream);              /* asynchronous */
int xcb_orbx_launches(const xcb_orbx* h);                                              /* kernels per detect */
int xcb_orbx_outputs(xcb_orbx* h, float** kp, float** kp_level, float** resp, int32_t** level, int32_t** bins,
                     uint8_t** desc, int32_t** counts);                               /* device pointers */
int xcb_orbx_detect_host(xcb_orbx* h, const uint8_t* img, float* kp, float* kp_level, float* resp, int32_t* level,
                         int32_t* bins, uint8_t* desc, int32_t* counts);               /* synchronous */
/* the slot arrays of the last detect (either entry) copied to the host after a device-wide wait; any may be NULL */
int xcb_orbx_read(xcb_orbx* h, float* kp, float* kp_level, float* resp, int32_t* level, int32_t* bins, uint8_t* desc,
                  int32_t* counts);
/* a pyramid level of the last xcb_orbx_detect_host frame (level 0 = the frame) to the host */
int xcb_orbx_read_level(xcb_orbx* h, int level, uint8_t* out);

typedef struct xcb_mm xcb_mm;

/* MapMatcher.__init__ (src/xclean/front/mapmatch.py:134-139, mapmatch_fast.py:164-170): a 16-px grid over a
   width x height image (at most 49152 cells), device scratch for batches of up to max_frames frames of max_kp keypoints
   and max_lm landmarks (xcb_mm_match_dev), one stream. */
int xcb_mm_create(int width, int height, int max_frames, int max_kp, int max_lm, xcb_mm** out);
int xcb_mm_destroy(xcb_mm* m);
const char* xcb_mm_last_error(xcb_mm* m);
int xcb_mm_grid_dims(xcb_mm* m, int* gw, int* gh);
/* Set a launch-shape knob of this matcher (XCB_TUNE_MM_LANES; no reference counterpart).  Results do not depend on
   it. */
int xcb_mm_set_tuning(xcb_mm* m, int knob, int value);
/* MapMatcher.match (mapmatch.py:148-169 + _gated :49-131; mapmatch_fast.py:172-184 + _match_fused :113-161) from host
   arrays: kp (N x 2 float64), desc (N x 32), uv (L x 2 float64), S (L x 2 x 2 float64), lm_desc (L x D x 32),
   lm_ndesc (L, int64, each <= D, else XCB_ERR_ARG: the reference would read past the landmark's slots), chi2 (the
   reference's default is 13.815510557964274).  Outputs out_kp / out_d (int64) and out_d2 (float64), L each.  Grows
   the device scratch when N or L exceed the handle's capacities; returns when the results are in the output arrays. */
int xcb_mm_match_host(xcb_mm* m, const double* kp, int N, const uint8_t* desc, const double* uv, const double* S,
                      const uint8_t* lm_desc, int D, const int64_t* lm_ndesc, int L, double chi2, int64_t* out_kp,
                      int64_t* out_d, double* out_d2, void* stream);
/* The same for F frames resident in device memory (no reference counterpart as one call: the reference matches one
   frame per call on the CPU).  Frame f: nkp[f] keypoints of kp_stride in kp (float32, the frontend's layout) and desc,
   nlm[f] landmarks of lm_stride in uv / S / lm_desc / lm_ndesc / outputs (counts read on the device, clamped to the
   strides; lm_ndesc values above D read as D; output rows past nlm[f] are not written).  Three launches on `stream`
   (NULL = the handle's own), nothing allocated, no synchronisation. */
int xcb_mm_match_dev(xcb_mm* m, int F, const float* kp, const int32_t* nkp, int kp_stride, const uint8_t* desc,
                     const double* uv, const double* S, const uint8_t* lm_desc, int D, const int64_t* lm_ndesc,
                     const int32_t* nlm, int lm_stride, double chi2, int64_t* out_kp, int64_t* out_d, double* out_d2,
                     void* stream);
int xcb_mm_sync(xcb_mm* m, void* stream);
/* window.predict_projection (src/xclean/vio/window.py:1032-1144): every landmark (host camera Rwc_h (L x 3 x 3) /
   pwc_h (L x 3), inverse-depth state lmp (L x 3) = a, b, rho) projected into the predicted body pose Rwb_t (3 x 3) /
   pwb_t (3) through the body-to-camera extrinsic Rbc / pbc, with the innovation covariance
   S = Jp Spose Jp^T + Jl Sl Jl^T + sig_px^2 I (Spose 6 x 6 in [dphi, dp], Sl (L x 3 x 3)); all row-major float64.
   Writes ok (L) for every landmark and, as the reference does, uv (L x 2) and depth (L) only where the point is in
   front (q2 > 1e-9, rho > 0) and S (L x 2 x 2) only where it also projects inside W x H; other entries keep the
   caller's values.  Bit-identical to the reference's float64 arithmetic. */
int xcb_mm_predict_host(xcb_mm* m, const double* Rwb_t, const double* pwb_t, const double* Rbc, const double* pbc,
                        const double* Rwc_h, const double* pwc_h, const double* lmp, const double* Spose,
                        const double* Sl, double sig_px, double fx, double fy, double cx, double cy, double W, double H,
                        int L, double* uv, double* S, uint8_t* ok, double* depth, void* stream);
/* The engine's tracking step in one call (vio/engine_live.py:1580-1582 and :1618-1632: _project, then
   MapMatcher.match on the landmarks predicted in view): xcb_mm_predict_host over the handle's W x H, then the gated
   map matching of the in-view landmarks against kp (N x 2 float64) / desc (N x 32), one upload and one read-back.
   out_kp / out_d / out_d2 have one entry per landmark (L); at the in-view landmarks sel = nonzero(ok) they equal
   MapMatcher.match(kp, desc, uv[sel], S[sel], lm_desc[sel], lm_ndesc[sel]), elsewhere they hold the defaults
   (-1, 9999, inf).  lm_ndesc is checked against D for every landmark. */
int xcb_mm_predict_match_host(xcb_mm* m, const double* Rwb_t, const double* pwb_t, const double* Rbc, const double* pbc,
                              const double* Rwc_h, const double* pwc_h, const double* lmp, const double* Spose,
                              const double* Sl, double sig_px, double fx, double fy, double cx, double cy, int L,
                              const double* kp, int N, const uint8_t* desc, const uint8_t* lm_desc, int D,
                              const int64_t* lm_ndesc, double chi2, double* uv, double* S, uint8_t* ok, double* depth,
                              int64_t* out_kp, int64_t* out_d, double* out_d2, void* stream);

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
    /* Marginal priors over pose blocks (src/xclean/vio/marg.py Prior, added to the system, the gradient and the cost
       as window.py _full_system / solve do, :865-887, :963-964), or pr_m == NULL for none.  Window w's prior is
       1/2 |S d + r|^2 with pr_m[w] rows (0 = no prior, at most 6 pr_nb[w]) over pr_nb[w] blocks: block k of the
       window is entry pr_boff[w] + k of pr_blk (its window-local slot) and of pr_x0 (its first-estimate pose: R0
       row-major, p0); d = per block [Log(R0^T R), p - p0]; S is pr_m[w] x 6 pr_nb[w] row-major at pr_S + pr_soff[w],
       r at pr_r + pr_roff[w]. */
    const int32_t* pr_m;        /* [nw] */
    const int32_t* pr_nb;       /* [nw] */
    const int32_t* pr_boff;     /* [nw] */
    const int32_t* pr_soff;     /* [nw] */
    const int32_t* pr_roff;     /* [nw] */
    const int32_t* pr_blk;      /* [blocks] */
    const double* pr_x0;        /* [blocks][12] */
    const double* pr_S;
    const double* pr_r;
} xcb_ba_windows;

#define XCB_BA_FP64 0           /* everything in float64: the plain form */
#define XCB_BA_MIXED 1          /* FP32 linearisation + Schur, FP64 Cholesky, FP64 refinement (to 1e-9, <= 3 steps) */
#define XCB_BA_LINEARISE 2      /* internal: one float64 linearisation, the reduced system exported (no step) */
#define XCB_BA_MIXED_NOTC 3     /* large-window path only: XCB_BA_MIXED with the Schur term scattered on the CUDA
                                   cores instead of accumulated on the tensor cores (for comparison) */
/* per-window status (stats [w][4] of the window solves, stats [w][3] of the Newton calls) when the scratch cannot
   hold the batch's per-landmark records; the kernel counts the landmarks from the windows themselves (lm_off + L),
   writes nothing else and leaves the state unchanged */
#define XCB_BA_STATUS_SCRATCH (-3)
/* per-window status of the Newton / adjoint calls for a window with a marginal prior (not supported there) */
#define XCB_BA_STATUS_PRIOR (-4)
/* per-window status of the large-window path when a tensor-core completion wait ran out (the window is not solved) */
#define XCB_BA_STATUS_TC (-5)

/* Device scratch the batched solve needs for `Lt` landmarks: the work counter, the trial landmark states and, for the
   float64 mode, each landmark's back-substitution record (118 doubles: ~0.95 kB per landmark).  A smaller scratch
   that still holds the trial states (3 doubles per landmark) works too: the float64 mode then re-linearises the
   landmarks for the back-substitution. */
size_t xcb_ba_scratch_bytes(int nw, int Lt);
/* window.solve (window.py:889-982, purely visual, fixed `iters` LM iterations from lam0) for every window of the batch
   in ONE persistent launch (no reference counterpart as one call; the reference solves one window per call on the
   CPU).  stats [nw][8] = cost0, cost, accepted, lam, status (0 ok, -1 window too large, -2 a landmark touches more
   than 16 keyframes, XCB_BA_STATUS_SCRATCH the scratch holds fewer than 3 doubles per landmark), iters, -, -;
   dx0 [nw][dx0_stride] (optional) = the first iteration's pose step.  grid = 0: one CTA per SM. */
int xcb_ba_solve_windows_dev(const xcb_ba_windows* w, int max_slots, int iters, double lam0, int mode, double* stats,
                             double* dx0, int dx0_stride, void* scratch, size_t scratch_bytes, int grid, void* stream);

/* The same LM iterations as xcb_ba_solve_windows_dev (no reference counterpart as one call: window.solve,
   window.py:889-982, for every window of the batch), for batches of few, large windows: each iteration is a sequence
   of launches whose landmark passes run over chunks of every window at once on all SMs (chunks: [nchunks][3] int32 in
   device memory = window, first landmark, end (window-local); together they cover each window's landmarks once), and
   whose Cholesky, solves and LM control run one CTA per window.  slots / Lt: the batch's slot and landmark totals.
   Windows with a marginal prior are refused (XCB_ERR_ARG).  stats / dx0 as xcb_ba_solve_windows_dev. */
size_t xcb_ba_large_scratch_bytes(int nw, int slots, int Lt);
int xcb_ba_solve_windows_large_dev(const xcb_ba_windows* w, int slots, int Lt, const int32_t* chunks, int nchunks,
                                   int max_slots, int iters, double lam0, int mode, double* stats, double* dx0,
                                   int dx0_stride, void* scratch, size_t scratch_bytes, void* stream);
/* xcb_ba_solve_windows_free_dev (float64, the landmarks that the Newton calls on `newton_scratch` flagged held
   constant) on the large-window path (no reference counterpart: the differentiable BA's forward on few large
   windows).  Arguments as xcb_ba_solve_windows_large_dev; newton_scratch / newton_scratch_bytes: the scratch of those
   Newton calls (its flags: 19 doubles per landmark after its first 256 bytes). */
int xcb_ba_solve_windows_large_free_dev(const xcb_ba_windows* w, int slots, int Lt, const int32_t* chunks, int nchunks,
                                        int max_slots, int iters, double lam0, double* stats, void* scratch,
                                        size_t scratch_bytes, const void* newton_scratch, size_t newton_scratch_bytes,
                                        void* stream);

/* The engine's state from which a window Problem is assembled (P1Engine._problem, src/xclean/vio/engine_live.py
   :407-530, visual part).  All pointers are device memory.  The slots' observation lists are concatenated in slot
   order (slot_n[i] observations for slot i). */
typedef struct {
    int P;                      /* slots (<= 64) */
    const int64_t* sids;        /* [P] slot ids */
    const int64_t* slot_n;      /* [P] observations of each slot */
    long long M;                /* total observations */
    const int64_t* lid;         /* [M] observed landmark id */
    const double* uv;           /* [M][2] pixel */
    const int64_t* cam;         /* [M] 0 left, 1 right */
    const uint8_t* valid;       /* [M] */
    const double* sig;          /* [M] the row's LK sigma */
    int n_lm;                   /* landmark ids 0 .. n_lm - 1 */
    const uint8_t* lm_alive;    /* [n_lm] */
    const uint8_t* select;      /* [n_lm] the selection of alive landmarks (lm_select), or NULL for all */
    const int64_t* lm_host;     /* [n_lm] host slot id */
    const double* lm_p;         /* [n_lm][3] (a, b, rho) */
    const double* lm_rho_meas;  /* [n_lm] */
    const double* lm_sig_lk;    /* [n_lm] */
    const double* lm_span;      /* [n_lm] */
    int prior_mode;             /* 1: the "prior" stereo mode (inverse-depth priors); 0: "ur" */
    double kappa_d, fB, sig_px;
} xcb_ba_engine;
/* The assembled window in the layout of one window of xcb_ba_windows (device memory, capacity n_lm landmarks and M
   rows): counts [3] = L, the rows kept, and 1 when a landmark's host slot is not in the window (the reference raises
   there); alive [n_lm] landmark ids in the window order; src [M][2] (slot, index in the slot) of every row. */
typedef struct {
    int32_t* counts;
    int64_t* alive;
    int32_t* src;
    double* lmp;                /* [n_lm][3] */
    int32_t* lm_host;           /* [n_lm] window slot */
    uint8_t* lm_mask;           /* [n_lm] */
    double* rho_meas;           /* [n_lm] */
    double* rho_isig;           /* [n_lm] */
    int32_t* lm_ob;             /* [n_lm + 1] */
    int32_t* ob_pose;           /* [M] */
    uint8_t* ob_cam;            /* [M] */
    double* ob_z;               /* [M][2] */
    double* ob_isig;            /* [M] */
    uint8_t* ob_valid;          /* [M] */
} xcb_ba_assembled;
/* Assemble the window on the device (replaces P1Engine._problem's host work, engine_live.py:407-530: the alive and
   selected landmarks in id order, their observations sorted stably by landmark, host slots, the inverse-depth
   priors of the "prior" stereo mode, the rows' whitening; no marginal prior, no IMU, the pose-free landmarks kept as
   ordinary ones).  Launches only (no synchronisation); the outputs feed xcb_ba_solve_windows_dev directly. */
size_t xcb_ba_assemble_scratch_bytes(int n_lm, int M, int P);
int xcb_ba_assemble_dev(const xcb_ba_engine* e, xcb_ba_assembled* out, void* scratch, size_t scratch_bytes,
                        void* stream);

/* The dense Gram product D = U U^T on the tensor cores (no reference counterpart: the contraction of the Schur term
   S -= W V^-1 W^T = U U^T, U = W chol(V^-1), that the large-window path's mixed-precision build runs per chunk):
   U (n x K, row-major float32, device), n <= 128; D (n x n, row-major, device) written.  tcgen05 kind::tf32 MMAs with
   every operand split into its TF32 rounding and remainder (hi hi^T + hi lo^T + lo hi^T: float32 accuracy), FP32
   accumulation in tensor memory.  err (device word, may be NULL): XCB_DEVERR_TC_WAIT if a completion wait ran out. */
int xcb_ba_gram_tc(const float* U, int n, int K, float* D, unsigned int* err, void* stream);

/* Allocation-free form of xcb_ba_solve_windows_dev.  No counterpart in the reference.  It is for callers that cannot
   call cudaMalloc while running: a real-time loop whose latency budget rules out an allocation (which may synchronise
   the device), or a plugin whose host owns the device memory through its own allocator.  The caller passes inputs and
   outputs as for xcb_ba_solve_windows_dev but no scratch: the scratch is a static device array of
   XCB_BA_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until exit, which limits one call to
   xcb_ba_noalloc_max_landmarks() landmarks in total (`Lt`, the batch's landmark count; more -> XCB_ERR_CAPACITY).
   The kernel also counts the landmarks from the windows (lm_off + L) and answers XCB_BA_STATUS_SCRATCH for every
   window, writing nothing else, when they exceed the array whatever `Lt` said.  Up to 4,332 landmarks the array also
   holds the float64 back-substitution records; above that the solve re-linearises the landmarks for the
   back-substitution instead (the same results, slower).  The first call on a device looks up the array's device
   address (call it before any stream capture); the address is kept for the life of the process, so it does not
   survive cudaDeviceReset or a re-created primary context on that device.  Calls share the array: calls that
   overlap on the GPU race.  No cudaMalloc, cudaFree or allocating library call is made. */
#define XCB_BA_NOALLOC_SCRATCH_BYTES ((size_t)4 << 20)
#define XCB_NOALLOC_MAX_DEVICES 64
int xcb_ba_noalloc_max_landmarks(void);
int xcb_ba_solve_windows_noalloc(const xcb_ba_windows* w, int Lt, int max_slots, int iters, double lam0, int mode,
                                 double* stats, double* dx0, int dx0_stride, int grid, void* stream);

/* Exact second-order steps on the window cost (no reference counterpart: the differentiable-BA API behind BAAdjoint).
   XCB_BA_NEWTON_POLISH: at most `steps` Newton steps with the exact Hessian (window.solve's LM converges only
   linearly when Huber weights are active), the state updated in place.  Each step moves every landmark to the
   minimum of its own cost with the poses fixed (Newton on its exact 3x3 block), then takes a Newton step on the poses
   with the exact reduced Hessian Hpp - Hpl Hll^-1 Hlp (Cholesky; Levenberg-Marquardt damped while it is not positive
   definite or the cost does not decrease), the landmarks following to first order; landmarks whose minimum lies at
   infinity (inverse depth below 1e-7, or their own Newton step taking it to <= 1e-9) are flagged constant (not in
   XCB_BA_NEWTON_POLISH_FIXED); it stops early at a gradient max-norm of 1e-10 or when a step at the cost's rounding
   level in a row no longer halve it (three times).  XCB_BA_NEWTON_ADJOINT: at the converged
   state, solves H x = dL/dstate (gpose: [slots][6] = dL/d(dphi, dp) per slot of the batch, landmarks 0) and writes
   dL/dtheta = -(d2C / dtheta dstate) x: gtheta [nw][11] = fx, fy, cx, cy, B, omega (3), t (3) of the left-to-right
   extrinsic at the rectified rig; gisig [M] = per-row weight 1/sigma; gz [M][2] = per-row pixels.  H is applied
   exactly (dual numbers); the system is solved with the Cholesky factor of the exact reduced system (the landmarks
   by back-substitution) and at most two refinement steps while the relative residual is above `tol`, or, where the
   reduced system is not positive definite, by conjugate gradients preconditioned with the Gauss-Newton Schur
   system (at most `maxit` iterations).  stats [nw][4]: polish = Newton steps taken, final damping, final gradient
   max-norm, status; adjoint = refinement steps (or conjugate-gradient iterations), final relative residual, -,
   status.  Status: 0 ok, 1 Gauss-Newton system not positive definite, 2 (polish) no damping gave a decrease /
   (adjoint) non-positive curvature met: the state is not at a strict minimum, -1 window too large, -2 a landmark
   touches more than 16 keyframes, XCB_BA_STATUS_SCRATCH the scratch, less its last xcb_ba_newton_scratch_bytes(nw, 0)
   - 512 bytes (the copies of the reduced systems), holds fewer than 19 doubles per landmark after its first 256
   bytes. */
#define XCB_BA_NEWTON_POLISH 0
#define XCB_BA_NEWTON_ADJOINT 1
#define XCB_BA_NEWTON_POLISH_FIXED 2      /* as XCB_BA_NEWTON_POLISH, flagging no new constant landmarks */
size_t xcb_ba_newton_scratch_bytes(int nw, int Lt);
int xcb_ba_newton_windows_dev(const xcb_ba_windows* w, int max_slots, int mode, int steps, int maxit, double tol,
                              const double* gpose, double* gtheta, double* gisig, double* gz, double* stats,
                              void* scratch, size_t scratch_bytes, int grid, void* stream);

/* window.solve's LM (as xcb_ba_solve_windows_dev, float64) with the landmarks that the Newton calls on `scratch` found
   frozen held constant (no reference counterpart; the differentiable BA's forward).  window.solve keeps a landmark
   whose step would take its inverse depth to <= 1e-9 where it is, but its Schur complement assumes every landmark
   moves, so its fixed point is not a stationary point of the cost when such landmarks exist; holding them constant
   (their rows stay in the pose blocks and the gradient) makes the LM converge to one.  A landmark is flagged by
   XCB_BA_NEWTON_POLISH calls (whose Gauss-Newton step, decoupled from the poses, would take its inverse depth to
   <= 1e-9; a flag stays until the scratch is cleared).  scratch: the Newton scratch, at least
   xcb_ba_newton_scratch_bytes(nw, Lt) bytes (Lt: the batch's landmarks).  stats [nw][8] as xcb_ba_solve_windows_dev. */
int xcb_ba_solve_windows_free_dev(const xcb_ba_windows* w, int Lt, int max_slots, int iters, double lam0,
                                  double* stats, void* scratch, size_t scratch_bytes, int grid, void* stream);
/* final_linearisation's visual outputs (src/xclean/vio/window.py:985-1008, build_system at lam = 0): for every
   window of the batch, at its current state, written from out + w * out_stride (float64; out zero-filled by the
   caller): the Schur-reduced H (6P x 6P, row-major), b (6P), then, when the row holds them (out_stride >=
   36 P^2 + 6 P + 10 L + M for that window), per landmark [lm_ok, Hll_inv (3 x 3)] (10 L; masked-out landmarks stay
   0, Hll_inv only where lm_ok) and per observation its whitened squared residual ob_chi2 (M; inf where invalid or
   behind the camera, 0 for masked-out landmarks).  out_stride >= 36 max_slots^2 + 6 max_slots.  stats [nw][8]:
   [0], [1] = the robust cost.  No hold, no damping, the state unchanged.  The prior and IMU terms of the reference's
   _full_system are not part of it (this path has neither).  scratch as xcb_ba_solve_windows_dev. */
int xcb_ba_linearise_windows_dev(const xcb_ba_windows* w, int max_slots, double* out, int out_stride, double* stats,
                                 void* scratch, size_t scratch_bytes, int grid, void* stream);
/* window.posefree_cost and window.posefree_step (src/xclean/vio/window.py:683-765): the pose-free landmarks of one
   window (seen only in their host's left image; the batched solve carries them as ordinary landmarks with that one
   observation).  Window: P slots Rwb (P x 3 x 3) / pwb (P x 3), extrinsic Rbc / pbc; block: n landmarks lmp (n x 3),
   host (n, int64, in 0..P-1), rmeas / ris (n), z (n x 2), isg.  cost_out (may be NULL): the robust cost, terms added
   in landmark order (behind != 0: 1e6 per point behind its host).  lmp_out (n x 3) / Hinv_out (n x 3 x 3) / ok_out
   (n) (NULL together): the step at damping lam (lam = 0: final_linearisation's marginals, window.py:1003-1006);
   Hinv_out is written only where ok, as the reference does.  Bit-identical to the reference's float64 arithmetic.
   Host memory; waits for `stream` (NULL = the legacy default stream) before returning. */
int xcb_ba_posefree_host(int P, const double* Rwb, const double* pwb, const double* Rbc, const double* pbc, int n,
                         const double* lmp, const int64_t* host, const double* rmeas, const double* ris,
                         const double* z, double isg, double fx, double fy, double cx, double cy, double huber_k,
                         int behind, double lam, double* cost_out, double* lmp_out, double* Hinv_out, uint8_t* ok_out,
                         void* stream);

/* ----------------------------------------------------------------------------------------------------------------
   Local-BA stage kernels: one entry point per kernel of src/xclean/backend/kernels.py, same argument order and
   meaning, device pointers (float32 / int32, the reference's layouts), enqueued on `stream` (NULL = the legacy default
   stream).  Sums into Hll, bl, Hred and g are accumulated (the caller zeroes them), in an unspecified order.
   -> XCB_OK or XCB_ERR_ARG / XCB_ERR_CUDA (message in xcb_last_error()).
   ---------------------------------------------------------------------------------------------------------------- */
/* kernels.py:45-114 build_blocks: Euclidean points, T_cw (nk,12) row-major 3x4; Jpose (N,2,6), Jlm (N,2,3),
   resw (N,2), Hll (nl,9) +=, bl (nl,3) +=, Hpl (N,6,3) */
int xcb_bk_build_blocks(const float* Tcw, const float* pts, const int* okf, const int* olm, const float* ouv,
                        float* Jpose, float* Jlm, float* resw, float* Hll, float* bl, float* Hpl, int N, float fx,
                        float cx, float cy, float huber, void* stream);
/* kernels.py:135-166 depth_prior: inverse-range prior on Euclidean points */
int xcb_bk_depth_prior(const float* pts, const float* chost, const float* rho0, const float* invsig,
                       const float* valid, float* Hll, float* bl, int nl, float huber, void* stream);
/* kernels.py:169-191 inv3_damped: (Hll + lam max(tr/3, 1e-9) I)^-1 */
int xcb_bk_inv3_damped(const float* Hll, float* Hlli, int nl, float lam, void* stream);
/* kernels.py:203-232 schur_pairs: Hred[ki][kj] -= Hpl_i Hlli Hpl_j^T over the ordered pair list (pa, pb) */
int xcb_bk_schur_pairs(const float* Hpl, const float* Hlli, const int* okf, const int* olm, const int* pa,
                       const int* pb, float* Hred, long long npair, int d, int n, void* stream);
/* kernels.py:235-258 schur_grad: g[k] -= Hpl Hlli bl */
int xcb_bk_schur_grad(const float* Hpl, const float* Hlli, const float* bl, const int* okf, const int* olm, float* g,
                      int N, int d, void* stream);
/* kernels.py:261-285 pose_blocks: Hred[k][k] += J^T J, g[k] -= J^T res (kf < 0: skipped); J (N,r,d) */
int xcb_bk_pose_blocks(const float* Jp, const float* res, const int* kf, float* Hred, float* g, int N, int r, int d,
                       int n, void* stream);
/* kernels.py:291-346 chol_solve: H (n,n) overwritten by its lower Cholesky factor, x = H^-1 b, one CTA of `nthreads`;
   status (int32 on the device) is cleared, then set to k+1 for a non-positive pivot k (the pivot is then 1e-8) */
int xcb_bk_chol_solve(float* H, const float* b, float* x, int n, int* status, int nthreads, void* stream);
/* kernels.py:349-374 backsub: dxl = Hlli (bl - sum_obs Hpl^T dxp[okf]), observations sorted by landmark (offs) */
int xcb_bk_backsub(const float* Hpl, const float* Hlli, const float* bl, const float* dxp, const int* okf,
                   const int* offs, float* dxl, int nl, int d, void* stream);
/* kernels.py:417-580 build_blocks_id: host-anchored (x_n, y_n, rho) landmarks; in-window host slot hidx >= 0 (its
   pose inverted from Tcw), else hpose (nl,12) T_wc; Jp (N,2,2,6) [observer, host], resw (N,2), kslot (N,2),
   Hll (nl,9) +=, bl (nl,3) +=, Hpl (N,2,6,3) */
int xcb_bk_build_blocks_id(const float* Tcw, const float* hpose, const int* hidx, const float* mbear, const float* rhov,
                           const int* okf, const int* olm, const float* ouv, float* Jp, float* resw, int* kslot,
                           float* Hll, float* bl, float* Hpl, int N, float fx, float cx, float cy, float huber,
                           void* stream);
/* kernels.py:599-643 landmark_prior_id: bearing (not robustified) and inverse-depth (Huber) priors */
int xcb_bk_landmark_prior_id(const float* mb, const float* rhov, const float* m0, const float* rho0,
                             const float* invsig, const float* wbear, const float* valid, float* Hll, float* bl,
                             int nl, float huber, void* stream);
/* kernels.py:646-680 pose_blocks_id: both slot pairs of every observation */
int xcb_bk_pose_blocks_id(const float* Jp, const float* res, const int* kslot, float* Hred, float* g, int N, int d,
                          int n, void* stream);
/* kernels.py:683-717 schur_pairs_id */
int xcb_bk_schur_pairs_id(const float* Hpl, const float* Hlli, const int* kslot, const int* olm, const int* pa,
                          const int* pb, float* Hred, long long npair, int d, int n, void* stream);
/* kernels.py:720-745 schur_grad_id */
int xcb_bk_schur_grad_id(const float* Hpl, const float* Hlli, const float* bl, const int* kslot, const int* olm,
                         float* g, int N, int d, void* stream);
/* kernels.py:748-775 backsub_id */
int xcb_bk_backsub_id(const float* Hpl, const float* Hlli, const float* bl, const float* dxp, const int* kslot,
                      const int* offs, float* dxl, int nl, int d, void* stream);

/* ----------------------------------------------------------------------------------------------------------------
   Local BA solve on the device: the LM loop of src/xclean/backend/ba.py _solve_gpu (ba.py:930-1089, Euclidean
   points) and _solve_gpu_id (ba.py:1345-1497, host-anchored inverse depth), every iteration enqueued on `stream` with
   the LM decisions (reject -> restore the best state and lam x 4, non-finite step -> lam x 10, accept -> lam / 2) taken
   by device kernels: no host round trip until the end.  Jacobians and landmark blocks are float32 (the reference's
   stage kernels above), the reduced system, its Cholesky, the landmark back-substitution and the state are float64.
   Observations must be sorted by landmark (offs = CSR starts, nl + 1).  All pointers are device pointers.
   ---------------------------------------------------------------------------------------------------------------- */
#define XCB_LBA_EUCLID 0
#define XCB_LBA_INVDEPTH 1
#define XCB_LBA_MAX_SLOTS 64        /* keyframes per problem */
#define XCB_LBA_MAX_TOUCHED 32      /* distinct keyframes one landmark touches (observers + in-window host) */
typedef struct {
    int model;                      /* XCB_LBA_EUCLID / XCB_LBA_INVDEPTH */
    int nk, nl, N;                  /* keyframes, landmarks, observations */
    double fx, cx, cy, huber, rho_floor;
    double* Tcw;                    /* (nk,12) in/out: rows of T_cw's 3x4, float64 */
    double* lm;                     /* (nl,3) in/out: Euclidean points, or bearings (x_n, y_n, 1) */
    double* rho;                    /* (nl) in/out: inverse depths (XCB_LBA_INVDEPTH) */
    const int* okf;                 /* (N) observing keyframe slot */
    const int* olm;                 /* (N) landmark */
    const float* ouv;               /* (N,2) pixels */
    const int* offs;                /* (nl+1) observation range of each landmark */
    const int* hidx;                /* (nl) in-window host slot or -1 (XCB_LBA_INVDEPTH) */
    const float* hpose;             /* (nl,12) T_wc of out-of-window hosts (XCB_LBA_INVDEPTH) */
    const unsigned char* free_mask; /* (nk) 1 = the keyframe is updated */
    /* optional priors (NULL = none), float32:
       Euclidean (kernels.py depth_prior): p0 = host centre (nl,3), p1 = rho0, p2 = invsig, p3 = valid;
       inverse depth (kernels.py landmark_prior_id): p0 = m0 (nl,2), p1 = rho0, p2 = invsig, p3 = valid, p4 = wbear */
    const float *p0, *p1, *p2, *p3, *p4;
    /* optional gyro relative-rotation factors (ba.py _rot_factor_blocks): a, b slots, M (nrot,9), sigma */
    int nrot;
    const int* rot_a;
    const int* rot_b;
    const double* rot_M;
    const double* rot_sig;
} xcb_lba_problem;
size_t xcb_lba_workspace_bytes(const xcb_lba_problem* p);
/* stats (device, 10 doubles): chi2_0 (chi of the last accepted state), chi2_n, rms_0, rms_n, lam, accepted steps,
   rejected steps, non-finite steps, landmarks that touched more than XCB_LBA_MAX_TOUCHED keyframes (their surplus
   slots were left out; the Python driver rejects such problems first), - */
int xcb_lba_solve(const xcb_lba_problem* p, int iters, double lam0, double* stats, void* workspace,
                  size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif
#endif
