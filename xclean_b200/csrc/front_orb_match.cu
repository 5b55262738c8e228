// front_orb_match.cu -- ORB (no orientation) descriptors and brute-force Hamming matching (sm_100a).
//
//   blur + ORB = Frontend.describe (src/xclean/stages/features.py:405-421): cv2 ORB on the reflect-101 pad-32 image;
//                ORB's internal 7x7 sigma-2 Gaussian runs OpenCV's float separable filter on a sub-matrix
//                (row taps fused for x < blur_vr, symmetric column taps fused for x < blur_vc; calibrated at
//                start-up), rounded half to even and saturated to u8.  256 tests at rint(kp + 32) of the pair
//                table recovered from the cv2 build at start-up.  Reference device form: gpu_front.py:495-561.
//   Hamming    = mapmatch_fast._bf_mutual / Frontend.match_desc (mapmatch_fast.py:46-111, features.py:564-595):
//                per query the first minimum and the second smallest distance (cv2.BFMatcher.knnMatch k=2), per
//                train column the first minimum; mutual NN, b1 <= 104, b1 < 0.8 b2.  Reference device form:
//                gpu_front.py:947-987 + the host epilogue :1887-1893 (here on the device).
//
// B200 layout: the blur is one tiled kernel (u8 tile + halo staged in shared memory, the row pass kept in shared
// memory as float32, only the u8 result written), so the reference's (H+64) x (W+64) float32 intermediate never
// reaches HBM.  Descriptors are read as 16-byte vectors; each Hamming CTA streams the train descriptors through shared
// memory once for 128 query rows.
#include "common.cuh"
#include "front_kernels.h"

#define BLUR_TY 32
#define BLUR_TX 64

__global__ void __launch_bounds__(256) k_blur(const u8* __restrict__ imgs, int H, int W, const float* __restrict__ kf,
                                              int vr, int vc, u8* __restrict__ outs)
{
    const int Hp = H + 64, Wp = W + 64;
    const int f = blockIdx.z;
    const u8* I = imgs + (size_t)f * H * W;
    u8* out = outs + (size_t)f * Hp * Wp;
    const int y0 = blockIdx.y * BLUR_TY, x0 = blockIdx.x * BLUR_TX;
    __shared__ float src[BLUR_TY + 6][BLUR_TX + 6];
    __shared__ float rb[BLUR_TY + 6][BLUR_TX];
    __shared__ float k[7];
    if (threadIdx.x < 7) k[threadIdx.x] = kf[threadIdx.x];
    // stage: virtual padded rows y0-3 .. y0+BLUR_TY+2 and columns x0-3 .. x0+BLUR_TX+2, each reflected at the padded
    // image's border and then mapped to the source image by the reflect-101 pad of 32
    for (int i = threadIdx.x; i < (BLUR_TY + 6) * (BLUR_TX + 6); i += blockDim.x) {
        int vy = i / (BLUR_TX + 6), vx = i % (BLUR_TX + 6);
        int py = XCB_REFL(y0 - 3 + vy, Hp), px = XCB_REFL(x0 - 3 + vx, Wp);
        int sy = XCB_REFL(py - 32, H), sx = XCB_REFL(px - 32, W);
        src[vy][vx] = (float)I[(size_t)sy * W + sx];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < (BLUR_TY + 6) * BLUR_TX; i += blockDim.x) {
        int vy = i / BLUR_TX, tx = i % BLUR_TX;
        int x = x0 + tx;
        const float* p = &src[vy][tx];
        float s;
        if (x < vr) {
            s = __fmul_rn(p[0], k[0]);
#pragma unroll
            for (int q = 1; q < 7; ++q) s = __fmaf_rn(p[q], k[q], s);
        } else {
            s = __fmul_rn(k[0], p[0]);
#pragma unroll
            for (int q = 1; q < 7; ++q) s = __fadd_rn(s, __fmul_rn(k[q], p[q]));
        }
        rb[vy][tx] = s;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < BLUR_TY * BLUR_TX; i += blockDim.x) {
        int ty = i / BLUR_TX, tx = i % BLUR_TX;
        int y = y0 + ty, x = x0 + tx;
        if (y >= Hp || x >= Wp) continue;
        int vy = ty + 3;
        float s;
        if (x < vc) {
            s = __fmul_rn(k[3], rb[vy][tx]);
#pragma unroll
            for (int q = 1; q <= 3; ++q) s = __fmaf_rn(k[3 + q], __fadd_rn(rb[vy + q][tx], rb[vy - q][tx]), s);
        } else {
            s = __fadd_rn(__fmul_rn(k[3], rb[vy][tx]), 0.0f);
#pragma unroll
            for (int q = 1; q <= 3; ++q)
                s = __fadd_rn(s, __fmul_rn(k[3 + q], __fadd_rn(rb[vy + q][tx], rb[vy - q][tx])));
        }
        int v = __float2int_rn(s);
        out[(size_t)y * Wp + x] = (u8)(v < 0 ? 0 : (v > 255 ? 255 : v));
    }
}

cudaError_t xcb_launch_blur(const uint8_t* img, int F, int H, int W, const float* kf, int vr, int vc, uint8_t* out,
                            cudaStream_t st)
{
    int Hp = H + 64, Wp = W + 64;
    dim3 grid((Wp + BLUR_TX - 1) / BLUR_TX, (Hp + BLUR_TY - 1) / BLUR_TY, F);
    k_blur<<<grid, 256, 0, st>>>(img, H, W, kf, vr, vc, out);
    return cudaGetLastError();
}

// one warp per keypoint, one lane per descriptor byte
__global__ void __launch_bounds__(256) k_orb(const u8* __restrict__ blur, int Hp, int Wp, const float* __restrict__ kp,
                                             const int* __restrict__ counts, int cap, const signed char* __restrict__ pat,
                                             u8* __restrict__ desc)
{
    __shared__ signed char sp[1024];
    for (int i = threadIdx.x; i < 1024; i += blockDim.x) sp[i] = pat[i];
    __syncthreads();
    const int f = blockIdx.y;
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), by = threadIdx.x & 31;
    if (i >= counts[f] || i >= cap) return;
    const float* k = kp + ((size_t)f * cap + i) * 2;
    const int cx = __float2int_rn(__fadd_rn(k[0], 32.0f));
    const int cy = __float2int_rn(__fadd_rn(k[1], 32.0f));
    const u8* c = blur + (size_t)f * Hp * Wp + (size_t)cy * Wp + cx;
    int val = 0;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        const signed char* q = sp + 4 * (8 * by + b);
        int t0 = c[(int)q[1] * Wp + (int)q[0]], t1 = c[(int)q[3] * Wp + (int)q[2]];
        val |= (t0 < t1) << b;
    }
    desc[((size_t)f * cap + i) * 32 + by] = (u8)val;
}

cudaError_t xcb_launch_orb(const uint8_t* blur, int F, int Hp, int Wp, const float* kp, const int* counts, int cap,
                           const int8_t* pat, uint8_t* desc, cudaStream_t st)
{
    dim3 grid((cap + 7) / 8, F);
    k_orb<<<grid, 256, 0, st>>>(blur, Hp, Wp, kp, counts, cap, (const signed char*)pat, desc);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------------------------------
// Hamming, one pass over the distance matrix: a thread owns a query row and scans the train descriptors (staged in
// shared memory, read as broadcasts) in increasing index with the CPU's update (strictly smaller replaces the best),
// which gives best / second / first index directly.  The column side (each train descriptor's first-minimum query)
// reuses the same distances: (distance << 16 | query) packed so that an unsigned minimum picks the smallest distance
// and, among equal distances, the smallest query index; a warp reduces its 32 rows with redux.sync, the CTA in
// shared memory, the row blocks of a pair with one global atomicMin per column and block.
// ------------------------------------------------------------------------------------------------------------------
#define HAM_T 128
#define HAM_CHUNK 1024

__device__ __forceinline__ int ham4(const ulonglong2 a0, const ulonglong2 a1, const ulonglong2 b0,
                                    const ulonglong2 b1)
{
    return __popcll(a0.x ^ b0.x) + __popcll(a0.y ^ b0.y) + __popcll(a1.x ^ b1.x) + __popcll(a1.y ^ b1.y);
}

__global__ void __launch_bounds__(HAM_T) k_hamming(const u8* __restrict__ A, const u8* __restrict__ B,
                                                   long long strideA, long long strideB, const int* __restrict__ LA,
                                                   const int* __restrict__ NB, int maxL, int maxN,
                                                   int* __restrict__ o1, int* __restrict__ o2, int* __restrict__ oi,
                                                   unsigned* __restrict__ colmin)
{
    __shared__ ulonglong2 sb[HAM_CHUNK][2];
    __shared__ unsigned cm[HAM_CHUNK];
    const int p = blockIdx.y;
    const int L = LA[p], N = NB[p];
    if (blockIdx.x * HAM_T >= L) return;
    const int i = blockIdx.x * HAM_T + threadIdx.x, lane = threadIdx.x & 31;
    const bool act = i < L;
    const ulonglong2* Ap = (const ulonglong2*)(A + p * strideA);
    const ulonglong2* Bp = (const ulonglong2*)(B + p * strideB);
    ulonglong2 a0 = make_ulonglong2(0, 0), a1 = a0;
    if (act) { a0 = Ap[2 * i]; a1 = Ap[2 * i + 1]; }
    int b1 = 1 << 30, b2 = 1 << 30, bi = -1;
    unsigned* cg = colmin + (size_t)p * maxN;
    for (int j0 = 0; j0 < N; j0 += HAM_CHUNK) {
        const int nj = min(HAM_CHUNK, N - j0);
        __syncthreads();
        for (int t = threadIdx.x; t < 2 * nj; t += HAM_T) sb[t >> 1][t & 1] = Bp[2 * j0 + t];
        for (int t = threadIdx.x; t < nj; t += HAM_T) cm[t] = 0xffffffffu;
        __syncthreads();
        for (int j = 0; j < nj; ++j) {
            const int d = ham4(a0, a1, sb[j][0], sb[j][1]);
            if (d < b1) { b2 = b1; b1 = d; bi = j0 + j; }
            else if (d < b2) b2 = d;
            const unsigned wm = __reduce_min_sync(0xffffffffu, act ? ((unsigned)d << 16) | (unsigned)i : 0xffffffffu);
            if (lane == 0 && wm != 0xffffffffu) atomicMin(&cm[j], wm);
        }
        __syncthreads();
        for (int t = threadIdx.x; t < nj; t += HAM_T)
            if (cm[t] != 0xffffffffu) atomicMin(&cg[j0 + t], cm[t]);
    }
    if (act) {
        const size_t o = (size_t)p * maxL + i;
        o1[o] = b1; o2[o] = b2; oi[o] = bi;
    }
}

cudaError_t xcb_launch_hamming(const XcbHamPairs& p, int* b1, int* b2, int* bi, int* ci, cudaStream_t st)
{
    if (p.npair <= 0) return cudaSuccess;
    if (p.maxN > 0) {
        cudaError_t e = cudaMemsetAsync(ci, 0xff, (size_t)p.npair * p.maxN * sizeof(unsigned), st);
        if (e != cudaSuccess) return e;
    }
    if (p.maxL > 0) {
        dim3 gr((p.maxL + HAM_T - 1) / HAM_T, p.npair);
        k_hamming<<<gr, HAM_T, 0, st>>>(p.A, p.B, p.strideA, p.strideB, p.LA, p.NB, p.maxL, p.maxN, b1, b2, bi,
                                        (unsigned*)ci);
    }
    return cudaGetLastError();
}

// match epilogue, one CTA per pair: ok = mutual && b1 <= ham_max && b1 < ratio * b2 (float64, as Python compares an
// int with a float product), compacted in query order by a block scan
__global__ void __launch_bounds__(1024) k_match_epilogue(const int* __restrict__ LA, const int* __restrict__ NB,
                                                         int maxL, int maxN, const int* __restrict__ b1,
                                                         const int* __restrict__ b2, const int* __restrict__ bi,
                                                         const int* __restrict__ ci, int ham_max, double ratio,
                                                         long long* __restrict__ i0, long long* __restrict__ i1,
                                                         long long out_stride, int* __restrict__ nmatch)
{
    __shared__ int warp_tot[32];
    __shared__ int base;
    const int p = blockIdx.x;
    const int L = LA[p], N = NB[p];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    if (L < 2 || N < 2) {
        if (threadIdx.x == 0) nmatch[p] = 0;
        return;
    }
    for (int q0 = 0; q0 < L; q0 += 1024) {
        int q = q0 + threadIdx.x;
        int ok = 0, j = -1;
        if (q < L) {
            size_t o = (size_t)p * maxL + q;
            j = bi[o];
            if (j >= 0) {
                int d1 = b1[o], d2 = b2[o];
                ok = d1 <= ham_max && (double)d1 < ratio * (double)d2 &&
                     (ci[(size_t)p * maxN + j] & 0xffff) == q;
            }
        }
        unsigned bal = __ballot_sync(0xffffffffu, ok);
        int pre = __popc(bal & ((1u << lane) - 1u));
        if (lane == 0) warp_tot[wid] = __popc(bal);
        __syncthreads();
        if (wid == 0) {
            int v = warp_tot[lane];
            int inc = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int t = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += t;
            }
            warp_tot[lane] = inc - v;   // exclusive prefix
        }
        __syncthreads();
        int pos = base + warp_tot[wid] + pre;
        if (ok) {
            i0[(size_t)p * out_stride + pos] = q;
            i1[(size_t)p * out_stride + pos] = j;
        }
        __syncthreads();
        if (threadIdx.x == 1023) base = pos + ok;
        __syncthreads();
    }
    if (threadIdx.x == 0) nmatch[p] = base;
}

cudaError_t xcb_launch_match_epilogue(const XcbHamPairs& p, const int* b1, const int* b2, const int* bi,
                                      const int* ci, int ham_max, double ratio, long long* i0, long long* i1,
                                      long long out_stride, int* nmatch, cudaStream_t st)
{
    if (p.npair <= 0) return cudaSuccess;
    k_match_epilogue<<<p.npair, 1024, 0, st>>>(p.LA, p.NB, p.maxL, p.maxN, b1, b2, bi, ci, ham_max, ratio, i0, i1,
                                               out_stride, nmatch);
    return cudaGetLastError();
}
