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
// reaches HBM.  The Hamming distances are int8 tensor-core products of +-1 expanded descriptors; each CTA expands the
// train descriptors into shared memory once for 128 query rows, and the row and column minima come from one pass.
#include "common.cuh"
#include "front_kernels.h"

#define BLUR_TY 32
#define BLUR_TX 128

// one thread per padded-image column of a 128 x 32 tile: the tile and its 3-pixel halo are staged once in shared
// memory (float32), then each thread walks down its column: the row pass of each staged row (7 taps in OpenCV's
// order, fused for x < vr), a 7-row window in registers, the symmetric column pass (fused for x < vc), rounding half
// to even and saturation to u8
__global__ void __launch_bounds__(BLUR_TX) k_blur(const u8* __restrict__ imgs, int H, int W, const float* __restrict__ kf,
                                                 int vr, int vc, u8* __restrict__ outs)
{
    const int Hp = H + 64, Wp = W + 64;
    const int f = blockIdx.z, tx = threadIdx.x;
    const u8* I = imgs + (size_t)f * H * W;
    u8* out = outs + (size_t)f * Hp * Wp;
    const int y0 = blockIdx.y * BLUR_TY, x0 = blockIdx.x * BLUR_TX;
    __shared__ float src[BLUR_TY + 6][BLUR_TX + 6];
    // stage: virtual padded rows y0-3 .. y0+BLUR_TY+2 and columns x0-3 .. x0+BLUR_TX+2, each reflected at the padded
    // image's border and then mapped to the source image by the reflect-101 pad of 32
    const int sxa = XCB_REFL(XCB_REFL(x0 - 3 + tx, Wp) - 32, W);
    const int sxb = tx < 6 ? XCB_REFL(XCB_REFL(x0 - 3 + BLUR_TX + tx, Wp) - 32, W) : 0;
    for (int vy = 0; vy < BLUR_TY + 6; ++vy) {
        const u8* row = I + (size_t)XCB_REFL(XCB_REFL(y0 - 3 + vy, Hp) - 32, H) * W;
        src[vy][tx] = (float)row[sxa];
        if (tx < 6) src[vy][BLUR_TX + tx] = (float)row[sxb];
    }
    float k[7];
#pragma unroll
    for (int q = 0; q < 7; ++q) k[q] = kf[q];
    __syncthreads();
    const int x = x0 + tx;
    if (x >= Wp) return;
    const bool fr = x < vr, fc = x < vc;
    float h[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int vy = 0; vy < BLUR_TY + 6; ++vy) {
        const float* pp = &src[vy][tx];
        float sr;
        if (fr) {
            sr = __fmul_rn(pp[0], k[0]);
#pragma unroll
            for (int q = 1; q < 7; ++q) sr = __fmaf_rn(pp[q], k[q], sr);
        } else {
            sr = __fmul_rn(k[0], pp[0]);
#pragma unroll
            for (int q = 1; q < 7; ++q) sr = __fadd_rn(sr, __fmul_rn(k[q], pp[q]));
        }
#pragma unroll
        for (int i = 0; i < 6; ++i) h[i] = h[i + 1];
        h[6] = sr;
        if (vy >= 6) {
            const int y = y0 + vy - 6;        // output row: h[3] is its row pass, h[3 -+ q] the rows above / below
            float sc;
            if (fc) {
                sc = __fmul_rn(k[3], h[3]);
#pragma unroll
                for (int q = 1; q <= 3; ++q) sc = __fmaf_rn(k[3 + q], __fadd_rn(h[3 + q], h[3 - q]), sc);
            } else {
                sc = __fadd_rn(__fmul_rn(k[3], h[3]), 0.0f);
#pragma unroll
                for (int q = 1; q <= 3; ++q) sc = __fadd_rn(sc, __fmul_rn(k[3 + q], __fadd_rn(h[3 + q], h[3 - q])));
            }
            if (y < Hp) {
                const int v = __float2int_rn(sc);
                out[(size_t)y * Wp + x] = (u8)(v < 0 ? 0 : (v > 255 ? 255 : v));
            }
        }
    }
}

cudaError_t xcb_launch_blur(const uint8_t* img, int F, int H, int W, const float* kf, int vr, int vc, uint8_t* out,
                            cudaStream_t st)
{
    int Hp = H + 64, Wp = W + 64;
    dim3 grid((Wp + BLUR_TX - 1) / BLUR_TX, (Hp + BLUR_TY - 1) / BLUR_TY, F);
    k_blur<<<grid, BLUR_TX, 0, st>>>(img, H, W, kf, vr, vc, out);
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
// Hamming, one pass over the distance matrix: per query row the best / second / first index of the best (the CPU's
// sequential scan), per train column the first-minimum query, both from the same distances.
// ------------------------------------------------------------------------------------------------------------------
// The distance is a dot product of +-1 vectors, hamming = (256 - a.b) / 2, so
// legacy int8 mma.m16n8k32 (native on this part, unlike the single-bit XOR-popc form) gives a 16 x 8 block of
// distances per 8 instructions.  A warp owns 16 query rows (their +-1 expansion held in registers); a CTA expands a
// chunk of 128 train descriptors once into shared memory for its 8 warps.  Fragments (PTX ISA, m16n8k32 .s8): a0 / a2
// = row g, k = 4q.. / 16 + 4q..; a1 / a3 = row g + 8; b0 / b1 = column g, k = 4q.. / 16 + 4q..; d0, d1 = row g,
// columns 2q, 2q + 1; d2, d3 = row g + 8 (g = lane / 4, q = lane % 4).  In k-step ks, descriptor nibble 8 ks + q feeds
// the first half and nibble 8 ks + 4 + q the second, in the same order for queries and trains.  Rows: each lane scans
// its columns in increasing order with the CPU's update, then the four lanes of a row merge (ties to the smaller
// index).  Columns: packed (distance << 16 | query) minima over the warp's 16 rows by shuffles, over the CTA in shared
// memory, over the row blocks by global atomicMin.
#define HTC_WARPS 8
#define HTC_CHUNK 128
#define HTC_BSTRIDE 272     // bytes per expanded train descriptor: word 8 ks + q of column g hits bank (4 g + q + 8 ks) % 32

// 4 descriptor bits -> 4 int8: +1 where the bit is set, -1 elsewhere
__device__ __forceinline__ unsigned pm1_nibble(unsigned nib)
{
    return ~(((nib * 0x00204081u) & 0x01010101u) * 0xFEu);
}

// the row state is kept on dot products (distance = (256 - dot) / 2 falls as the dot rises): the CPU's update
// (a strictly smaller distance replaces the best) is a strictly larger dot
#define HTC_NONE (-(1 << 30))
__device__ __forceinline__ void ham_take(int dot, int j, int& b1, int& bi, int& b2)
{
    if (dot > b1) { b2 = b1; b1 = dot; bi = j; }
    else if (dot > b2) b2 = dot;
}

// merge the (best, index, second) of lane ^ off: the larger best dot wins, ties to the smaller index
__device__ __forceinline__ void ham_merge(int& b1, int& bi, int& b2, int off)
{
    const int c1 = __shfl_xor_sync(0xffffffffu, b1, off);
    const int ci = __shfl_xor_sync(0xffffffffu, bi, off);
    const int c2 = __shfl_xor_sync(0xffffffffu, b2, off);
    if (c1 > b1 || (c1 == b1 && ci >= 0 && (bi < 0 || ci < bi))) {
        b2 = max(b1, c2); b1 = c1; bi = ci;
    } else {
        b2 = max(b2, c1);
    }
}

__device__ __forceinline__ int ham_of_dot(int dot) { return dot == HTC_NONE ? 1 << 30 : (256 - dot) >> 1; }

__global__ void __launch_bounds__(HTC_WARPS * 32) k_hamming_tc(const u8* __restrict__ A, const u8* __restrict__ B,
                                                              long long strideA, long long strideB,
                                                              const int* __restrict__ LA, const int* __restrict__ NB,
                                                              int maxL, int maxN, int* __restrict__ o1,
                                                              int* __restrict__ o2, int* __restrict__ oi,
                                                              unsigned* __restrict__ colmin)
{
    __shared__ __align__(16) unsigned char sB[HTC_CHUNK * HTC_BSTRIDE];
    __shared__ unsigned cm[HTC_CHUNK];
    const int p = blockIdx.y;
    const int L = LA[p], N = NB[p];
    const int rb = blockIdx.x * 16 * HTC_WARPS;
    if (rb >= L) return;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, g = lane >> 2, q = lane & 3;
    const int r0 = rb + 16 * w + g, r1 = r0 + 8;
    // the warp's 16 query rows as +-1 fragments (rows past L: any values, never reported)
    unsigned a0[8], a1[8], a2[8], a3[8];
    {
        const uint4* Ap = (const uint4*)(A + p * strideA);
        uint4 x0 = make_uint4(0u, 0u, 0u, 0u), x1 = x0, y0 = x0, y1 = x0;
        if (r0 < L) { x0 = __ldg(Ap + 2 * r0); x1 = __ldg(Ap + 2 * r0 + 1); }
        if (r1 < L) { y0 = __ldg(Ap + 2 * r1); y1 = __ldg(Ap + 2 * r1 + 1); }
        const unsigned xr[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
        const unsigned yr[8] = {y0.x, y0.y, y0.z, y0.w, y1.x, y1.y, y1.z, y1.w};
#pragma unroll
        for (int ks = 0; ks < 8; ++ks) {       // descriptor word ks holds nibbles 8 ks .. 8 ks + 7
            a0[ks] = pm1_nibble((xr[ks] >> (4 * q)) & 0xFu);
            a2[ks] = pm1_nibble((xr[ks] >> (4 * q + 16)) & 0xFu);
            a1[ks] = pm1_nibble((yr[ks] >> (4 * q)) & 0xFu);
            a3[ks] = pm1_nibble((yr[ks] >> (4 * q + 16)) & 0xFu);
        }
    }
    int b1r0 = HTC_NONE, b2r0 = HTC_NONE, bir0 = -1, b1r1 = HTC_NONE, b2r1 = HTC_NONE, bir1 = -1;
    // column keys: distance << 16 | query = (256 - dot) << 15 | query; a row past L keys all ones (never the minimum)
    const unsigned pk0 = r0 < L ? (unsigned)r0 : 0xffffffffu, pk1 = r1 < L ? (unsigned)r1 : 0xffffffffu;
    const unsigned* Bw = (const unsigned*)(B + p * strideB);
    unsigned* cg = colmin + (size_t)p * maxN;
    for (int j0 = 0; j0 < N; j0 += HTC_CHUNK) {
        const int nj = min(HTC_CHUNK, N - j0), njp = (nj + 7) & ~7;
        __syncthreads();
        for (int t = tid; t < njp * 64; t += HTC_WARPS * 32) {      // (descriptor, nibble) -> one expanded word
            const int jj = t >> 6, nb = t & 63;
            const unsigned word = jj < nj ? __ldg(Bw + 8 * (j0 + jj) + (nb >> 3)) : 0u;
            ((unsigned*)(sB + jj * HTC_BSTRIDE))[nb] = pm1_nibble((word >> (4 * (nb & 7))) & 0xFu);
        }
        for (int t = tid; t < HTC_CHUNK; t += HTC_WARPS * 32) cm[t] = 0xffffffffu;
        __syncthreads();
        for (int jt = 0; jt < njp; jt += 8) {
            const unsigned* bw = (const unsigned*)(sB + (jt + g) * HTC_BSTRIDE);
            int d0 = 0, d1 = 0, d2 = 0, d3 = 0;
#pragma unroll
            for (int ks = 0; ks < 8; ++ks) {
                const unsigned b0 = bw[8 * ks + q], bb1 = bw[8 * ks + 4 + q];
                asm("mma.sync.aligned.m16n8k32.row.col.s32.s8.s8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                    "{%0,%1,%2,%3};"
                    : "+r"(d0), "+r"(d1), "+r"(d2), "+r"(d3)
                    : "r"(a0[ks]), "r"(a1[ks]), "r"(a2[ks]), "r"(a3[ks]), "r"(b0), "r"(bb1));
            }
            const int jA = j0 + jt + 2 * q;
            const bool vA = jA < N, vB = jA + 1 < N;
            if (vA) { ham_take(d0, jA, b1r0, bir0, b2r0); ham_take(d2, jA, b1r1, bir1, b2r1); }
            if (vB) { ham_take(d1, jA + 1, b1r0, bir0, b2r0); ham_take(d3, jA + 1, b1r1, bir1, b2r1); }
            unsigned mA = min(((unsigned)(256 - d0) << 15) | pk0, ((unsigned)(256 - d2) << 15) | pk1);
            unsigned mB = min(((unsigned)(256 - d1) << 15) | pk0, ((unsigned)(256 - d3) << 15) | pk1);
#pragma unroll
            for (int o = 4; o < 32; o <<= 1) {
                mA = min(mA, __shfl_xor_sync(0xffffffffu, mA, o));
                mB = min(mB, __shfl_xor_sync(0xffffffffu, mB, o));
            }
            if (g == 0) {
                if (vA && mA != 0xffffffffu) atomicMin(&cm[jt + 2 * q], mA);
                if (vB && mB != 0xffffffffu) atomicMin(&cm[jt + 2 * q + 1], mB);
            }
        }
        __syncthreads();
        for (int t = tid; t < nj; t += HTC_WARPS * 32)
            if (cm[t] != 0xffffffffu) atomicMin(&cg[j0 + t], cm[t]);
    }
    ham_merge(b1r0, bir0, b2r0, 1); ham_merge(b1r0, bir0, b2r0, 2);
    ham_merge(b1r1, bir1, b2r1, 1); ham_merge(b1r1, bir1, b2r1, 2);
    if (q == 0) {
        if (r0 < L) {
            const size_t o = (size_t)p * maxL + r0;
            o1[o] = ham_of_dot(b1r0); o2[o] = ham_of_dot(b2r0); oi[o] = bir0;
        }
        if (r1 < L) {
            const size_t o = (size_t)p * maxL + r1;
            o1[o] = ham_of_dot(b1r1); o2[o] = ham_of_dot(b2r1); oi[o] = bir1;
        }
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
        dim3 gr((p.maxL + 16 * HTC_WARPS - 1) / (16 * HTC_WARPS), p.npair);
        k_hamming_tc<<<gr, HTC_WARPS * 32, 0, st>>>(p.A, p.B, p.strideA, p.strideB, p.LA, p.NB, p.maxL, p.maxN, b1, b2,
                                                    bi, (unsigned*)ci);
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
