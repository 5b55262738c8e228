// front_ext.cu -- the frontend's multi-scale, oriented extras (sm_100a): FAST-9 corners with non-maximum suppression,
// an image pyramid, intensity-centroid orientation bins and steered rBRIEF.  They go beyond the reference, whose
// frontend is single-scale Shi-Tomasi with unoriented ORB (src/xclean/stages/features.py:27-28, :102-103;
// src/xclean/front/gpu_front.py:1712-1717).  They sit behind their own entry points, and the default path does not use
// them.  Level 0 with orientation bin 0 is the reference's descriptor bit for bit.
//
//   k_fast_score   thread per pixel: the FAST 9-of-16 segment test on the radius-3 Bresenham circle.  The score is the
//                  largest threshold at which the pixel is still a corner: the max over the 16 arcs of 9 pixels and both
//                  polarities of the arc's smallest difference, minus one.  -1 = no corner at `threshold`, or within
//                  3 px of the border.  cv2.FastFeatureDetector (TYPE_9_16) detects and scores exactly these
//   k_fast_rows    CTA per row: the corners that beat all 8 neighbours (non-corners count as 0), or every corner without
//                  suppression.  Pass 0 counts per row; pass 1 writes in row-major order after k_fast_scan's scan
//   k_fast_select  one CTA: of the corners at least `edge` px inside, the `quota` best by score, ties in row-major order
//                  (a score histogram gives the cut, two block scans place them); output in row-major order
//   k_pyr_down     thread per output pixel: bilinear resampling with 8-bit weights from exact rational source
//                  coordinates, which is cv2.resize(INTER_LINEAR_EXACT), the call cv2's ORB builds its pyramid with
//   k_ic_bins      warp per keypoint: the intensity centroid (m10, m01) over the disc u^2 + v^2 <= R (R + 1), R = 15.
//                  Exact sign tests against host-made directions give the orientation bin (30 bins of 12 degrees, bin k
//                  centred on 12 k).  The keypoint's level-0 position and level are written too
//   k_orb_steer    warp per keypoint: rBRIEF on the blurred pad-32 level image, with the test pattern rotated to the
//                  keypoint's bin (host-made tables; bin k equals cv2.ORB.compute with KeyPoint.angle = 12 k)
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "common.cuh"
#include "front_kernels.h"

extern void xcb_set_last_error(const std::string& m);

#define EXT_BINS 30
#define EXT_R 15
#define EXT_PAD 32
#define EXT_MAXL 8


// ------------------------------------------------------------------------------------------------------------ FAST
__device__ __forceinline__ int fmin_i(int a, int b) { return a < b ? a : b; }
__device__ __forceinline__ int fmax_i(int a, int b) { return a > b ? a : b; }

__global__ void k_fast_score(const u8* __restrict__ img, int H, int W, int threshold, int* __restrict__ score)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    int s = -1;
    if (x >= 3 && x < W - 3 && y >= 3 && y < H - 3) {
        // the radius-3 Bresenham circle, clockwise from the top
        const u8* c = img + (size_t)y * W + x;
        const int p = c[0];
        int d[16];
        d[0] = (int)c[-3 * W] - p;
        d[1] = (int)c[-3 * W + 1] - p;
        d[2] = (int)c[-2 * W + 2] - p;
        d[3] = (int)c[-W + 3] - p;
        d[4] = (int)c[3] - p;
        d[5] = (int)c[W + 3] - p;
        d[6] = (int)c[2 * W + 2] - p;
        d[7] = (int)c[3 * W + 1] - p;
        d[8] = (int)c[3 * W] - p;
        d[9] = (int)c[3 * W - 1] - p;
        d[10] = (int)c[2 * W - 2] - p;
        d[11] = (int)c[W - 3] - p;
        d[12] = (int)c[-3] - p;
        d[13] = (int)c[-W - 3] - p;
        d[14] = (int)c[-2 * W - 2] - p;
        d[15] = (int)c[-3 * W - 1] - p;
        // minima of every arc of 9 by doubling (arcs of 2, 4, 8, then the ninth), for d (bright) and -d (dark)
        int a2[16], b2[16], a4[16], b4[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            a2[k] = fmin_i(d[k], d[(k + 1) & 15]);
            b2[k] = fmin_i(-d[k], -d[(k + 1) & 15]);
        }
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            a4[k] = fmin_i(a2[k], a2[(k + 2) & 15]);
            b4[k] = fmin_i(b2[k], b2[(k + 2) & 15]);
        }
        int best = -(1 << 20);
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const int a8 = fmin_i(a4[k], a4[(k + 4) & 15]), b8 = fmin_i(b4[k], b4[(k + 4) & 15]);
            best = fmax_i(best, fmin_i(a8, d[(k + 8) & 15]));
            best = fmax_i(best, fmin_i(b8, -d[(k + 8) & 15]));
        }
        if (best - 1 >= threshold) s = best - 1;
    }
    score[(size_t)y * W + x] = s;
}

__device__ __forceinline__ bool fast_keep(const int* __restrict__ score, int H, int W, int x, int y, int nms)
{
    const int s = score[(size_t)y * W + x];
    if (s < 0) return false;
    if (!nms) return true;
    for (int a = -1; a <= 1; ++a)
        for (int b = -1; b <= 1; ++b) {
            if (!a && !b) continue;
            const int yy = y + a, xx = x + b;
            const int t = (yy >= 0 && yy < H && xx >= 0 && xx < W) ? max(score[(size_t)yy * W + xx], 0) : 0;
            if (!(s > t)) return false;
        }
    return true;
}

// pass 0: per-row counts; pass 1: the row's kept pixels from rowoff[y] on, in x order (at most cap in total)
__global__ void __launch_bounds__(256) k_fast_rows(const int* __restrict__ score, int H, int W, int nms, int pass,
                                                   int* __restrict__ rowcnt, const int* __restrict__ rowoff, int cap,
                                                   float* __restrict__ kp, float* __restrict__ resp)
{
    __shared__ int wsum[8];
    __shared__ int base;
    const int y = blockIdx.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) base = pass ? rowoff[y] : 0;
    __syncthreads();
    for (int x0 = 0; x0 < W; x0 += blockDim.x) {
        const int x = x0 + threadIdx.x;
        const bool k = x < W && fast_keep(score, H, W, x, y, nms);
        const unsigned m = __ballot_sync(0xffffffffu, k);
        if (lane == 0) wsum[wid] = __popc(m);
        __syncthreads();
        int before = 0, total = 0;
        for (int i = 0; i < 8; ++i) {
            if (i < wid) before += wsum[i];
            total += wsum[i];
        }
        if (pass && k) {
            const int o = base + before + __popc(m & ((1u << lane) - 1u));
            if (o < cap) {
                kp[2 * o] = (float)x;
                kp[2 * o + 1] = (float)y;
                resp[o] = (float)score[(size_t)y * W + x];
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) base += total;
        __syncthreads();
    }
    if (!pass && threadIdx.x == 0) rowcnt[y] = base;
}

// exclusive scan of the row counts (one CTA); the total into *n
__global__ void __launch_bounds__(1024) k_fast_scan(const int* __restrict__ rowcnt, int H, int* __restrict__ rowoff,
                                                    int* __restrict__ n)
{
    __shared__ int part[1024];
    const int per = (H + 1023) / 1024, b = threadIdx.x * per, e = min(H, b + per);
    int s = 0;
    for (int i = b; i < e; ++i) s += rowcnt[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const int v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    int r = part[threadIdx.x] - s;
    for (int i = b; i < e; ++i) {
        rowoff[i] = r;
        r += rowcnt[i];
    }
    if (threadIdx.x == 1023) *n = part[1023];
}

// block-wide exclusive count of `f` over the 1024 threads, and the total
__device__ __forceinline__ int block_excl(bool f, int* wsum, int& total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned m = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wsum[wid] = __popc(m);
    __syncthreads();
    int before = 0, t = 0;
    for (int i = 0; i < 32; ++i) {
        const int v = wsum[i];
        if (i < wid) before += v;
        t += v;
    }
    __syncthreads();
    total = t;
    return before + __popc(m & ((1u << lane) - 1u));
}

__global__ void __launch_bounds__(1024) k_fast_select(const float* __restrict__ rawkp, const float* __restrict__ rawresp,
                                                      const int* __restrict__ nraw, int cap_raw, int W, int H, int edge,
                                                      int quota, float* __restrict__ kp, float* __restrict__ resp,
                                                      int* __restrict__ count)
{
    __shared__ int hist[256];
    __shared__ int wsum[32];
    __shared__ int cut, take;
    const int n = min(*nraw, cap_raw);
    for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    auto inside = [&](int i) {
        const float x = rawkp[2 * i], y = rawkp[2 * i + 1];
        return x >= (float)edge && x < (float)(W - edge) && y >= (float)edge && y < (float)(H - edge);
    };
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (inside(i)) atomicAdd(&hist[min(max((int)rawresp[i], 0), 255)], 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        int cum = 0, c = -1, t = 0;
        for (int s = 255; s >= 0; --s) {
            if (cum + hist[s] >= quota) {
                c = s;
                t = quota - cum;
                break;
            }
            cum += hist[s];
        }
        cut = c;
        take = t;
    }
    __syncthreads();
    int base_keep = 0, base_tie = 0;
    for (int c0 = 0; c0 < n; c0 += blockDim.x) {
        const int i = c0 + threadIdx.x;
        const bool ins = i < n && inside(i);
        const int s = ins ? min(max((int)rawresp[i], 0), 255) : -1;
        const bool tie = ins && s == cut;
        int ntie, nkeep;
        const int trank = base_tie + block_excl(tie, wsum, ntie);
        const bool keep = ins && (s > cut || (tie && trank < take));
        const int pos = base_keep + block_excl(keep, wsum, nkeep);
        if (keep && pos < quota) {
            kp[2 * pos] = rawkp[2 * i];
            kp[2 * pos + 1] = rawkp[2 * i + 1];
            resp[pos] = rawresp[i];
        }
        base_keep += nkeep;
        base_tie += ntie;
    }
    if (threadIdx.x == 0) *count = min(base_keep, quota);
}

// --------------------------------------------------------------------------------------------------------- pyramid
// out = ((a (256 - fx) + b fx) (256 - fy) + (c (256 - fx) + d fx) fy + 2^15) >> 16, with the source index and weight
// of each output column (x0, wx) and row (y0, wy) from xcb_pyr_tables
__global__ void k_pyr_down(const u8* __restrict__ src, int Hs, int Ws, u8* __restrict__ dst, int Hd, int Wd,
                           const int* __restrict__ x0, const int* __restrict__ wx, const int* __restrict__ y0,
                           const int* __restrict__ wy)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= Wd) return;
    const int xa = min(max(x0[x], 0), Ws - 1), xb = min(xa + 1, Ws - 1);
    const int ya = min(max(y0[y], 0), Hs - 1), yb = min(ya + 1, Hs - 1);
    const int fx = wx[x], fy = wy[y];
    const int a = src[(size_t)ya * Ws + xa], b = src[(size_t)ya * Ws + xb];
    const int c = src[(size_t)yb * Ws + xa], d = src[(size_t)yb * Ws + xb];
    const int top = a * (256 - fx) + b * fx, bot = c * (256 - fx) + d * fx;
    dst[(size_t)y * Wd + x] = (u8)((top * (256 - fy) + bot * fy + 32768) >> 16);
}

// ----------------------------------------------------------------------------------------------------- orientation
// bin k when v = (m10, m01) is not clockwise of boundary k (at 12 k - 6 degrees), clockwise of boundary k + 1, and on
// the side of centre k; bin 0 when m10 = m01 = 0.  The same computed cross product decides both neighbouring bins, so
// the bins partition the plane.  Optional outputs: the level-0 position (kp x scale), the level, the moments.
__global__ void __launch_bounds__(256) k_ic_bins(const u8* __restrict__ img, int H, int W, const float* __restrict__ kp,
                                                 int n, const int* __restrict__ count, const int* __restrict__ umax,
                                                 const double* __restrict__ bdir, const double* __restrict__ cdir,
                                                 int* __restrict__ bins, long long* __restrict__ mom, float scale,
                                                 int level, float* __restrict__ kp0, int* __restrict__ lvl)
{
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    const int nn = count ? min(*count, n) : n;
    if (i >= nn) return;
    const int cx = __float2int_rn(kp[2 * i]), cy = __float2int_rn(kp[2 * i + 1]);
    long long m10 = 0, m01 = 0;
    if (lane <= 2 * EXT_R) {
        const int v = lane - EXT_R, yy = cy + v;
        const int um = umax[v < 0 ? -v : v];
        if (yy >= 0 && yy < H) {
            const u8* row = img + (size_t)yy * W;
            int s10 = 0, s0 = 0;
            for (int u = -um; u <= um; ++u) {
                const int xx = cx + u;
                const int I = (xx >= 0 && xx < W) ? row[xx] : 0;
                s10 += u * I;
                s0 += I;
            }
            m10 = s10;
            m01 = (long long)v * s0;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m10 += __shfl_xor_sync(0xffffffffu, m10, o);
        m01 += __shfl_xor_sync(0xffffffffu, m01, o);
    }
    if (lane == 0) {
        int bin = 0;
        if (m10 != 0 || m01 != 0) {
            const double X = (double)m10, Y = (double)m01;
            for (int k = 0; k < EXT_BINS; ++k) {
                const int k1 = (k + 1) % EXT_BINS;
                const double c0 = __dsub_rn(__dmul_rn(bdir[2 * k], Y), __dmul_rn(bdir[2 * k + 1], X));
                const double c1 = __dsub_rn(__dmul_rn(bdir[2 * k1], Y), __dmul_rn(bdir[2 * k1 + 1], X));
                const double dc = __dadd_rn(__dmul_rn(cdir[2 * k], X), __dmul_rn(cdir[2 * k + 1], Y));
                if (c0 >= 0.0 && c1 < 0.0 && dc > 0.0) {
                    bin = k;
                    break;
                }
            }
        }
        bins[i] = bin;
        if (mom) {
            mom[2 * i] = m10;
            mom[2 * i + 1] = m01;
        }
        if (kp0) {
            kp0[2 * i] = __fmul_rn(kp[2 * i], scale);
            kp0[2 * i + 1] = __fmul_rn(kp[2 * i + 1], scale);
        }
        if (lvl) lvl[i] = level;
    }
}

// --------------------------------------------------------------------------------------------------- steered rBRIEF
// pats [EXT_BINS][256][4] (x1, y1, x2, y2); the blurred image is padded by `pad`, the centre rint(kp + pad) as in the
// unrotated descriptor.  A test point outside the padded image reads 0 (never the case for keypoints inside the image
// and patterns within +-pad).
__global__ void __launch_bounds__(256) k_orb_steer(const u8* __restrict__ blur, int Hp, int Wp, int pad,
                                                   const float* __restrict__ kp, int n, const int* __restrict__ count,
                                                   const int* __restrict__ bins, const signed char* __restrict__ pats,
                                                   u8* __restrict__ desc)
{
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), by = threadIdx.x & 31;
    const int nn = count ? min(*count, n) : n;
    if (i >= nn) return;
    const int cx = __float2int_rn(__fadd_rn(kp[2 * i], (float)pad));
    const int cy = __float2int_rn(__fadd_rn(kp[2 * i + 1], (float)pad));
    const int bin = min(max(bins[i], 0), EXT_BINS - 1);
    const signed char* pt = pats + (size_t)bin * 1024;
    auto at = [&](int dx, int dy) -> int {
        const int x = cx + dx, y = cy + dy;
        return (x >= 0 && x < Wp && y >= 0 && y < Hp) ? blur[(size_t)y * Wp + x] : 0;
    };
    int val = 0;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        const signed char* q = pt + 4 * (8 * by + b);
        val |= (at(q[0], q[1]) < at(q[2], q[3])) << b;
    }
    desc[(size_t)i * 32 + by] = (u8)val;
}

// ------------------------------------------------------------------------------------------------ host-side tables
static int ext_fail(const std::string& m, int code)
{
    xcb_set_last_error(m);
    return code;
}

// source index and 8-bit weight of each destination sample: src = (d + 1/2) ns / nd - 1/2 exactly (rational), the
// weight round-half-even(frac * 256); clamped to index 0 / weight 0 below and index ns - 1 / weight 0 at the end
static void pyr_tables(int ns, int nd, int* idx, int* w)
{
    for (int d = 0; d < nd; ++d) {
        const long long N = (2ll * d + 1) * ns - nd, D = 2ll * nd;
        long long s = N >= 0 ? N / D : -((-N + D - 1) / D);
        const long long a = N - s * D;                 // in [0, D)
        const long long q = a * 256 / D, r = a * 256 % D;
        long long wt = q + ((2 * r > D || (2 * r == D && (q & 1))) ? 1 : 0);
        if (s < 0) {
            s = 0;
            wt = 0;
        }
        if (s >= ns - 1) {
            s = ns - 1;
            wt = 0;
        }
        idx[d] = (int)s;
        w[d] = (int)wt;
    }
}

static void ic_tables(int* umax, double* bdir, double* cdir)
{
    for (int v = 0; v <= EXT_R; ++v) {
        int u = 0;
        while ((u + 1) * (u + 1) + v * v <= EXT_R * (EXT_R + 1)) ++u;
        umax[v] = u;
    }
    const double d2r = M_PI / 180.0;
    for (int k = 0; k < EXT_BINS; ++k) {
        bdir[2 * k] = std::cos((double)(12 * k - 6) * d2r);
        bdir[2 * k + 1] = std::sin((double)(12 * k - 6) * d2r);
        cdir[2 * k] = std::cos((double)(12 * k) * d2r);
        cdir[2 * k + 1] = std::sin((double)(12 * k) * d2r);
    }
}

// ---------------------------------------------------------------------------------------------- C ABI: primitives
extern "C" int xcb_pyr_tables(int n_src, int n_dst, int32_t* idx, int32_t* w)
{
    if (n_src < 1 || n_dst < 1 || !idx || !w) return ext_fail("pyr_tables: bad argument", XCB_ERR_ARG);
    pyr_tables(n_src, n_dst, idx, w);
    return XCB_OK;
}

extern "C" int xcb_orient_tables(int32_t* umax, double* bdir, double* cdir)
{
    if (!umax || !bdir || !cdir) return ext_fail("orient_tables: null argument", XCB_ERR_ARG);
    ic_tables(umax, bdir, cdir);
    return XCB_OK;
}

static size_t al256(size_t b) { return (b + 255) / 256 * 256; }

extern "C" size_t xcb_fast_scratch_bytes(int width, int height)
{
    if (width < 1 || height < 1) return 0;
    return al256((size_t)width * height * 4) + 2 * al256((size_t)height * 4);
}

static cudaError_t launch_fast(const u8* img, int W, int H, int threshold, int nonmax, int cap, float* kp, float* resp,
                               int* count, int* score, int* rowcnt, int* rowoff, cudaStream_t st)
{
    k_fast_score<<<dim3((W + 127) / 128, H), 128, 0, st>>>(img, H, W, threshold, score);
    k_fast_rows<<<H, 256, 0, st>>>(score, H, W, nonmax, 0, rowcnt, nullptr, cap, kp, resp);
    k_fast_scan<<<1, 1024, 0, st>>>(rowcnt, H, rowoff, count);
    k_fast_rows<<<H, 256, 0, st>>>(score, H, W, nonmax, 1, rowcnt, rowoff, cap, kp, resp);
    return cudaGetLastError();
}

extern "C" int xcb_fast_dev(const uint8_t* img, int width, int height, int threshold, int nonmax, int cap, float* kp,
                            float* resp, int32_t* count, void* scratch, size_t scratch_bytes, void* stream)
{
    if (!img || !kp || !resp || !count || !scratch) return ext_fail("fast: null argument", XCB_ERR_ARG);
    if (width < 1 || height < 1 || height > 65535 || threshold < 0 || threshold > 255 || cap < 0)
        return ext_fail("fast: bad size (height <= 65535), threshold (0..255) or capacity", XCB_ERR_ARG);
    if (scratch_bytes < xcb_fast_scratch_bytes(width, height))
        return ext_fail("fast: scratch smaller than xcb_fast_scratch_bytes", XCB_ERR_CAPACITY);
    char* p = (char*)scratch;
    int* score = (int*)p;
    p += al256((size_t)width * height * 4);
    int* rowcnt = (int*)p;
    p += al256((size_t)height * 4);
    int* rowoff = (int*)p;
    const cudaError_t e = launch_fast(img, width, height, threshold, nonmax ? 1 : 0, cap, kp, resp, count, score,
                                      rowcnt, rowoff, (cudaStream_t)stream);
    if (e != cudaSuccess) return ext_fail(std::string("fast: ") + cudaGetErrorString(e), XCB_ERR_CUDA);
    return XCB_OK;
}

extern "C" int xcb_fast_select_dev(const float* kp_in, const float* resp_in, const int32_t* n_in, int cap_in,
                                   int width, int height, int edge, int quota, float* kp, float* resp,
                                   int32_t* count, void* stream)
{
    if (!kp_in || !resp_in || !n_in || !kp || !resp || !count || cap_in < 0 || quota < 0 || edge < 0)
        return ext_fail("fast_select: null argument or negative size", XCB_ERR_ARG);
    k_fast_select<<<1, 1024, 0, (cudaStream_t)stream>>>(kp_in, resp_in, n_in, cap_in, width, height, edge, quota, kp,
                                                        resp, count);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ext_fail(std::string("fast_select: ") + cudaGetErrorString(e), XCB_ERR_CUDA);
    return XCB_OK;
}

extern "C" int xcb_pyr_down_dev(const uint8_t* src, int ws, int hs, uint8_t* dst, int wd, int hd, const int32_t* x0,
                                const int32_t* wx, const int32_t* y0, const int32_t* wy, void* stream)
{
    if (!src || !dst || !x0 || !wx || !y0 || !wy || ws < 1 || hs < 1 || wd < 1 || hd < 1 || hd > 65535)
        return ext_fail("pyr_down: null argument, empty image or height > 65535", XCB_ERR_ARG);
    k_pyr_down<<<dim3((wd + 127) / 128, hd), 128, 0, (cudaStream_t)stream>>>(src, hs, ws, dst, hd, wd, x0, wx, y0, wy);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ext_fail(std::string("pyr_down: ") + cudaGetErrorString(e), XCB_ERR_CUDA);
    return XCB_OK;
}

extern "C" int xcb_ic_bins_dev(const uint8_t* img, int width, int height, const float* kp, int n,
                               const int32_t* count, const int32_t* umax, const double* bdir, const double* cdir,
                               int32_t* bins, int64_t* moments, void* stream)
{
    if (!img || (!kp && n) || !umax || !bdir || !cdir || (!bins && n) || n < 0 || width < 1 || height < 1)
        return ext_fail("ic_bins: null argument or bad size", XCB_ERR_ARG);
    if (n == 0) return XCB_OK;
    k_ic_bins<<<(n + 7) / 8, 256, 0, (cudaStream_t)stream>>>(img, height, width, kp, n, count, umax, bdir, cdir, bins,
                                                             (long long*)moments, 1.0f, 0, nullptr, nullptr);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ext_fail(std::string("ic_bins: ") + cudaGetErrorString(e), XCB_ERR_CUDA);
    return XCB_OK;
}

extern "C" int xcb_orb_steered_dev(const uint8_t* blur, int wp, int hp, int pad, const float* kp, int n,
                                   const int32_t* count, const int32_t* bins, const int8_t* patterns, uint8_t* desc,
                                   void* stream)
{
    if (!blur || (!kp && n) || (!bins && n) || !patterns || (!desc && n) || n < 0 || pad < 0 || wp < 1 || hp < 1)
        return ext_fail("orb_steered: null argument or bad size", XCB_ERR_ARG);
    if (n == 0) return XCB_OK;
    k_orb_steer<<<(n + 7) / 8, 256, 0, (cudaStream_t)stream>>>(blur, hp, wp, pad, kp, n, count, bins,
                                                               (const signed char*)patterns, desc);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ext_fail(std::string("orb_steered: ") + cudaGetErrorString(e), XCB_ERR_CUDA);
    return XCB_OK;
}

extern "C" int xcb_blur_dev(const uint8_t* img, int width, int height, const float* kf7, int vr, int vc, uint8_t* out,
                            void* stream)
{
    if (!img || !kf7 || !out || width < 2 || height < 2) return ext_fail("blur: null argument or bad size", XCB_ERR_ARG);
    const cudaError_t e = xcb_launch_blur(img, 1, height, width, kf7, vr, vc, out, (cudaStream_t)stream);
    if (e != cudaSuccess) return ext_fail(std::string("blur: ") + cudaGetErrorString(e), XCB_ERR_CUDA);
    return XCB_OK;
}

// ------------------------------------------------------------------------------------- C ABI: the per-frame handle
struct xcb_orbx {
    int W, H, L, nfeat, thr, edge, nonmax;
    int lw[EXT_MAXL], lh[EXT_MAXL], quota[EXT_MAXL], qoff[EXT_MAXL];
    float lscale[EXT_MAXL];
    size_t loff[EXT_MAXL], toff[EXT_MAXL];
    int vr[EXT_MAXL], vc[EXT_MAXL];
    bool blur_set[EXT_MAXL], pats_set;
    int cap_raw;
    u8 *lvl, *blur, *in;              // levels 1..L-1; the padded blurred level; the host entry's input
    int *score, *rowcnt, *rowoff, *nraw, *tabs, *umax;
    float *rawkp, *rawresp, *kf;
    double *bdir, *cdir;
    signed char* pats;
    float *kp, *kpl, *resp;           // outputs, [nfeat] slots, level l at qoff[l]
    int *level, *bins, *counts;
    u8* desc;
    cudaStream_t stream;
    std::string err;
};

static int ox_fail(xcb_orbx* h, int code, const std::string& m)
{
    if (h) h->err = m;
    xcb_set_last_error(m);
    return code;
}

extern "C" void xcb_orbx_destroy(xcb_orbx* h)
{
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    void* bufs[] = {h->lvl, h->blur, h->in, h->score, h->rowcnt, h->rowoff, h->nraw, h->tabs, h->umax, h->rawkp,
                    h->rawresp, h->kf, h->bdir, h->cdir, h->pats, h->kp, h->kpl, h->resp, h->level, h->bins,
                    h->counts, h->desc};
    for (void* b : bufs)
        if (b) cudaFree(b);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

extern "C" int xcb_orbx_create(int width, int height, int levels, double scale, int nfeatures, int fast_threshold,
                               int edge, int nonmax, xcb_orbx** out)
{
    if (!out) return ox_fail(nullptr, XCB_ERR_ARG, "orbx_create: null output");
    *out = nullptr;
    if (levels < 1 || levels > EXT_MAXL || !(scale > 1.0) || scale > 4.0 || nfeatures < 1 || fast_threshold < 0 ||
        fast_threshold > 255 || edge < EXT_R + 1 || width < 1 || height < 1 || height > 65535)
        return ox_fail(nullptr, XCB_ERR_ARG,
                       "orbx_create: levels 1..8, scale in (1, 4], nfeatures >= 1, threshold 0..255, edge >= 16");
    xcb_orbx* h = new xcb_orbx();
    h->W = width;
    h->H = height;
    h->L = levels;
    h->nfeat = nfeatures;
    h->thr = fast_threshold;
    h->edge = edge;
    h->nonmax = nonmax ? 1 : 0;
    // level sizes: rint(n / scale^l) in float32 (the sizes cv2's ORB gives its levels)
    for (int l = 0; l < levels; ++l) {
        const float s = (float)std::pow(scale, (double)l);
        h->lscale[l] = s;
        h->lw[l] = (int)std::nearbyint((float)width / s);
        h->lh[l] = (int)std::nearbyint((float)height / s);
        if (h->lw[l] < 2 * edge + 1 || h->lh[l] < 2 * edge + 1) {
            delete h;
            return ox_fail(nullptr, XCB_ERR_ARG, "orbx_create: level " + std::to_string(l) +
                                                     " smaller than 2 edge + 1 pixels");
        }
    }
    // per-level quotas: a geometric share of nfeatures (ratio 1 / scale), rounded; the last level takes the rest
    {
        const double f = 1.0 / scale;
        double share = nfeatures * (1.0 - f) / (1.0 - std::pow(f, (double)levels));
        int sum = 0;
        for (int l = 0; l < levels - 1; ++l) {
            h->quota[l] = std::min((int)std::nearbyint(share), nfeatures - sum);
            sum += h->quota[l];
            share *= f;
        }
        h->quota[levels - 1] = std::max(nfeatures - sum, 0);
        int o = 0;
        for (int l = 0; l < levels; ++l) {
            h->qoff[l] = o;
            o += h->quota[l];
        }
    }
    size_t lv = 0, tb = 0;
    for (int l = 1; l < levels; ++l) {
        h->loff[l] = lv;
        lv += al256((size_t)h->lw[l] * h->lh[l]);
        h->toff[l] = tb;
        tb += 2 * (size_t)(h->lw[l] + h->lh[l]);
    }
    h->cap_raw = width * height;
    const size_t npad = (size_t)(width + 2 * EXT_PAD) * (height + 2 * EXT_PAD);
    const size_t nf = (size_t)nfeatures;
    cudaError_t e = cudaSuccess;
    auto A = [&](void** p, size_t b) {
        if (e == cudaSuccess) e = cudaMalloc(p, b ? b : 256);
    };
    A((void**)&h->lvl, lv);
    A((void**)&h->blur, npad);
    A((void**)&h->in, (size_t)width * height);
    A((void**)&h->score, (size_t)width * height * 4);
    A((void**)&h->rowcnt, (size_t)height * 4);
    A((void**)&h->rowoff, (size_t)height * 4);
    A((void**)&h->nraw, 4 * EXT_MAXL);
    A((void**)&h->tabs, tb * 4);
    A((void**)&h->umax, 4 * (EXT_R + 1));
    A((void**)&h->rawkp, (size_t)h->cap_raw * 8);
    A((void**)&h->rawresp, (size_t)h->cap_raw * 4);
    A((void**)&h->kf, 7 * 4 * EXT_MAXL);
    A((void**)&h->bdir, 2 * EXT_BINS * 8);
    A((void**)&h->cdir, 2 * EXT_BINS * 8);
    A((void**)&h->pats, EXT_BINS * 1024);
    A((void**)&h->kp, nf * 8);
    A((void**)&h->kpl, nf * 8);
    A((void**)&h->resp, nf * 4);
    A((void**)&h->level, nf * 4);
    A((void**)&h->bins, nf * 4);
    A((void**)&h->counts, 4 * EXT_MAXL);
    A((void**)&h->desc, nf * 32);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        std::vector<int> t(tb ? tb : 1);
        for (int l = 1; l < levels; ++l) {
            int* p = t.data() + h->toff[l];
            pyr_tables(h->lw[l - 1], h->lw[l], p, p + h->lw[l]);
            pyr_tables(h->lh[l - 1], h->lh[l], p + 2 * h->lw[l], p + 2 * h->lw[l] + h->lh[l]);
        }
        int um[EXT_R + 1];
        double bd[2 * EXT_BINS], cd[2 * EXT_BINS];
        ic_tables(um, bd, cd);
        if (tb) e = cudaMemcpy(h->tabs, t.data(), tb * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(h->umax, um, sizeof(um), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(h->bdir, bd, sizeof(bd), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(h->cdir, cd, sizeof(cd), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemset(h->counts, 0, 4 * EXT_MAXL);
    }
    if (e != cudaSuccess) {
        const std::string m = std::string("orbx_create: ") + cudaGetErrorString(e);
        xcb_orbx_destroy(h);
        return ox_fail(nullptr, XCB_ERR_CUDA, m);
    }
    *out = h;
    return XCB_OK;
}

extern "C" const char* xcb_orbx_last_error(const xcb_orbx* h) { return h ? h->err.c_str() : xcb_last_error(); }

extern "C" int xcb_orbx_level(const xcb_orbx* h, int level, int* width, int* height, float* scale, int* quota,
                              int* offset)
{
    if (!h || level < 0 || level >= h->L) return ox_fail(nullptr, XCB_ERR_ARG, "orbx_level: bad handle or level");
    if (width) *width = h->lw[level];
    if (height) *height = h->lh[level];
    if (scale) *scale = h->lscale[level];
    if (quota) *quota = h->quota[level];
    if (offset) *offset = h->qoff[level];
    return XCB_OK;
}

extern "C" int xcb_orbx_set_blur(xcb_orbx* h, int level, int vr, int vc, const float* kf7)
{
    if (!h || level < 0 || level >= h->L || !kf7) return ox_fail(h, XCB_ERR_ARG, "orbx_set_blur: bad argument");
    const cudaError_t e = cudaMemcpy(h->kf + 7 * level, kf7, 7 * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return ox_fail(h, XCB_ERR_CUDA, std::string("orbx_set_blur: ") + cudaGetErrorString(e));
    h->vr[level] = vr;
    h->vc[level] = vc;
    h->blur_set[level] = true;
    return XCB_OK;
}

extern "C" int xcb_orbx_set_patterns(xcb_orbx* h, const int8_t* patterns)
{
    if (!h || !patterns) return ox_fail(h, XCB_ERR_ARG, "orbx_set_patterns: null argument");
    for (int i = 0; i < EXT_BINS * 1024; ++i)
        if (patterns[i] < -(EXT_PAD - 1) || patterns[i] > EXT_PAD - 1)
            return ox_fail(h, XCB_ERR_ARG, "orbx_set_patterns: a test point beyond the 32-pixel pad");
    const cudaError_t e = cudaMemcpy(h->pats, patterns, EXT_BINS * 1024, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return ox_fail(h, XCB_ERR_CUDA, std::string("orbx_set_patterns: ") + cudaGetErrorString(e));
    h->pats_set = true;
    return XCB_OK;
}

// the whole frame on `stream`: per level pyramid step, FAST, selection, orientation, blur, steered descriptors
extern "C" int xcb_orbx_detect_dev(xcb_orbx* h, const uint8_t* img, void* stream)
{
    if (!h || !img) return ox_fail(h, XCB_ERR_ARG, "orbx_detect: null argument");
    if (!h->pats_set) return ox_fail(h, XCB_ERR_NOT_CALIBRATED, "orbx_detect: steered patterns not set");
    for (int l = 0; l < h->L; ++l)
        if (!h->blur_set[l])
            return ox_fail(h, XCB_ERR_NOT_CALIBRATED, "orbx_detect: blur of level " + std::to_string(l) + " not set");
    cudaStream_t st = (cudaStream_t)stream;
    const u8* prev = img;
    for (int l = 0; l < h->L; ++l) {
        const int W = h->lw[l], H = h->lh[l];
        const u8* cur = img;
        if (l > 0) {
            u8* dst = h->lvl + h->loff[l];
            const int* t = h->tabs + h->toff[l];
            k_pyr_down<<<dim3((W + 127) / 128, H), 128, 0, st>>>(prev, h->lh[l - 1], h->lw[l - 1], dst, H, W, t, t + W,
                                                                  t + 2 * W, t + 2 * W + H);
            cur = dst;
        }
        cudaError_t e = launch_fast(cur, W, H, h->thr, h->nonmax, h->cap_raw, h->rawkp, h->rawresp, h->nraw + l,
                                    h->score, h->rowcnt, h->rowoff, st);
        const int q = h->quota[l], o = h->qoff[l];
        if (e == cudaSuccess) {
            k_fast_select<<<1, 1024, 0, st>>>(h->rawkp, h->rawresp, h->nraw + l, h->cap_raw, W, H, h->edge, q,
                                              h->kpl + 2 * o, h->resp + o, h->counts + l);
            e = xcb_launch_blur(cur, 1, H, W, h->kf + 7 * l, h->vr[l], h->vc[l], h->blur, st);
        }
        if (e == cudaSuccess && q > 0) {
            k_ic_bins<<<(q + 7) / 8, 256, 0, st>>>(cur, H, W, h->kpl + 2 * o, q, h->counts + l, h->umax, h->bdir,
                                                   h->cdir, h->bins + o, nullptr, h->lscale[l], l, h->kp + 2 * o,
                                                   h->level + o);
            k_orb_steer<<<(q + 7) / 8, 256, 0, st>>>(h->blur, H + 2 * EXT_PAD, W + 2 * EXT_PAD, EXT_PAD,
                                                     h->kpl + 2 * o, q, h->counts + l, h->bins + o, h->pats,
                                                     h->desc + (size_t)o * 32);
            e = cudaGetLastError();
        }
        if (e != cudaSuccess) return ox_fail(h, XCB_ERR_CUDA, std::string("orbx_detect: ") + cudaGetErrorString(e));
        prev = cur;
    }
    return XCB_OK;
}

// kernels one xcb_orbx_detect_dev call launches
extern "C" int xcb_orbx_launches(const xcb_orbx* h)
{
    if (!h) return 0;
    int n = 0;
    for (int l = 0; l < h->L; ++l) n += (l > 0 ? 1 : 0) + 4 + 2 + (h->quota[l] > 0 ? 2 : 0);
    return n;
}

extern "C" int xcb_orbx_outputs(xcb_orbx* h, float** kp, float** kp_level, float** resp, int32_t** level,
                                int32_t** bins, uint8_t** desc, int32_t** counts)
{
    if (!h) return ox_fail(nullptr, XCB_ERR_ARG, "orbx_outputs: null handle");
    if (kp) *kp = h->kp;
    if (kp_level) *kp_level = h->kpl;
    if (resp) *resp = h->resp;
    if (level) *level = h->level;
    if (bins) *bins = h->bins;
    if (desc) *desc = h->desc;
    if (counts) *counts = h->counts;
    return XCB_OK;
}

// host image in, every slot array out (nfeatures entries; level l's first counts[l] slots from its offset are valid);
// kp_level may be null
extern "C" int xcb_orbx_detect_host(xcb_orbx* h, const uint8_t* img, float* kp, float* kp_level, float* resp,
                                    int32_t* level, int32_t* bins, uint8_t* desc, int32_t* counts)
{
    if (!h || !img || !kp || !resp || !level || !bins || !desc || !counts)
        return ox_fail(h, XCB_ERR_ARG, "orbx_detect_host: null argument");
    cudaStream_t st = h->stream;
    const size_t nf = (size_t)h->nfeat;
    cudaError_t e = cudaMemcpyAsync(h->in, img, (size_t)h->W * h->H, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return ox_fail(h, XCB_ERR_CUDA, std::string("orbx H2D: ") + cudaGetErrorString(e));
    const int rc = xcb_orbx_detect_dev(h, h->in, st);
    if (rc != XCB_OK) return rc;
    struct Cp {
        void* dst;
        const void* src;
        size_t b;
    } cp[] = {{kp, h->kp, nf * 8},       {resp, h->resp, nf * 4}, {level, h->level, nf * 4},
              {bins, h->bins, nf * 4},   {desc, h->desc, nf * 32}, {counts, h->counts, (size_t)h->L * 4},
              {kp_level, h->kpl, kp_level ? nf * 8 : 0}};
    for (auto& c : cp)
        if (e == cudaSuccess && c.b) e = cudaMemcpyAsync(c.dst, c.src, c.b, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return ox_fail(h, XCB_ERR_CUDA, std::string("orbx D2H: ") + cudaGetErrorString(e));
    return XCB_OK;
}

// the slot arrays of the last detect (either entry, any stream) to the host: waits for the device; any may be null
extern "C" int xcb_orbx_read(xcb_orbx* h, float* kp, float* kp_level, float* resp, int32_t* level, int32_t* bins,
                             uint8_t* desc, int32_t* counts)
{
    if (!h) return ox_fail(nullptr, XCB_ERR_ARG, "orbx_read: null handle");
    cudaError_t e = cudaDeviceSynchronize();
    const size_t nf = (size_t)h->nfeat;
    struct Cp {
        void* dst;
        const void* src;
        size_t b;
    } cp[] = {{kp, h->kp, nf * 8},       {kp_level, h->kpl, nf * 8}, {resp, h->resp, nf * 4},
              {level, h->level, nf * 4}, {bins, h->bins, nf * 4},    {desc, h->desc, nf * 32},
              {counts, h->counts, (size_t)h->L * 4}};
    for (auto& c : cp)
        if (e == cudaSuccess && c.dst) e = cudaMemcpy(c.dst, c.src, c.b, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return ox_fail(h, XCB_ERR_CUDA, std::string("orbx_read: ") + cudaGetErrorString(e));
    return XCB_OK;
}

// a pyramid level of the last host-entry frame to the host (level 0 = that frame itself)
extern "C" int xcb_orbx_read_level(xcb_orbx* h, int level, uint8_t* out)
{
    if (!h || !out || level < 0 || level >= h->L) return ox_fail(h, XCB_ERR_ARG, "orbx_read_level: bad argument");
    const u8* src = level == 0 ? h->in : h->lvl + h->loff[level];
    cudaError_t e = cudaMemcpyAsync(out, src, (size_t)h->lw[level] * h->lh[level], cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return ox_fail(h, XCB_ERR_CUDA, std::string("orbx_read_level: ") + cudaGetErrorString(e));
    return XCB_OK;
}
