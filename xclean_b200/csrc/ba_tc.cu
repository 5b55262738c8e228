// ba_tc.cu -- the dense Gram product D = U U^T on the tensor cores (tcgen05, kind::tf32 with a hi / lo split), the
// contraction the large-window build uses for the Schur term (S -= W V^-1 W^T = U U^T with U = W chol(V^-1)).
#include <string>

#include "ba_tc.cuh"
#include "common.cuh"

extern void xcb_set_last_error(const std::string& m);

// one CTA of 128 threads: U (n x K row-major, n <= 128) streamed through two stages of TF32 hi / lo tiles of 32
// columns; D (n x n row-major) from the tensor-memory accumulator
__global__ void __launch_bounds__(128, 1) k_gram_tc(const float* __restrict__ U, int n, int K, float* __restrict__ D,
                                                   unsigned int* err)
{
    extern __shared__ __align__(1024) float tsm[];
    __shared__ __align__(8) uint64_t bar[3];          // two tile stages, the final drain
    __shared__ uint32_t tmem_base;
    __shared__ int fail;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) tc_alloc(&tmem_base, 128);
    if (tid == 0) {
        tc_mbar_init(&bar[0]);
        tc_mbar_init(&bar[1]);
        tc_mbar_init(&bar[2]);
        fail = 0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;
    const int ntile = (K + TC_KT - 1) / TC_KT;
    for (int t = 0; t < ntile; ++t) {
        const int st = t & 1;
        if (t >= 2 && tid == 0 && !tc_mbar_wait(&bar[st], (uint32_t)(((t >> 1) - 1) & 1))) fail = 1;
        __syncthreads();
        if (fail) break;
        float* hi = tsm + st * 2 * TC_TILE_FLOATS;
        float* lo = hi + TC_TILE_FLOATS;
        for (int q = tid; q < TC_M * TC_KT; q += blockDim.x) {
            const int r = q / TC_KT, k = q % TC_KT, kk = t * TC_KT + k;
            const float x = (r < n && kk < K) ? U[(size_t)r * K + kk] : 0.0f;
            float h, l;
            tc_split(x, h, l);
            hi[tc_off(r, k)] = h;
            lo[tc_off(r, k)] = l;
        }
        tc_fence_proxy();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            tc_issue(tmem, hi, lo, t > 0, &bar[st]);
        }
    }
    if (tid == 0 && !fail) {
        if (ntile >= 1 && !tc_mbar_wait(&bar[(ntile - 1) & 1], (uint32_t)(((ntile - 1) >> 1) & 1))) fail = 1;
        if (ntile >= 2 && !tc_mbar_wait(&bar[(ntile - 2) & 1], (uint32_t)(((ntile - 2) >> 1) & 1))) fail = 1;
    }
    if (tid == 0 && ntile >= 1 && !tc_drain(&bar[2])) fail = 1;
    __syncthreads();
    tc_fence_after();
    if (!fail) {
        const int row = 32 * warp + lane;
        for (int c0 = 0; c0 < TC_M; c0 += 16) {
            float v[16];
            if (ntile > 0) {
                tc_ld16(tmem, warp, c0, v);
            } else {
#pragma unroll
                for (int i = 0; i < 16; ++i) v[i] = 0.0f;
            }
            if (row < n)
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    if (c0 + i < n) D[(size_t)row * n + c0 + i] = v[i];
        }
    } else if (tid == 0 && err) {
        atomicOr(err, XCB_DEVERR_TC_WAIT);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tc_dealloc(tmem, 128);
}

extern "C" int xcb_ba_gram_tc(const float* U, int n, int K, float* D, unsigned int* err, void* stream)
{
    if ((!U && K > 0) || !D || n < 1 || n > TC_M || K < 0) {
        xcb_set_last_error("ba_gram_tc: D null, U null with K > 0, n outside 1..128 or K negative");
        return XCB_ERR_ARG;
    }
    static XcbAttrOnce attr;
    cudaError_t e = xcb_smem_attr_once(attr, (const void*)k_gram_tc, 4 * TC_TILE_FLOATS * (int)sizeof(float));
    if (e == cudaSuccess) {
        k_gram_tc<<<1, 128, 4 * TC_TILE_FLOATS * sizeof(float), (cudaStream_t)stream>>>(U, n, K, D, err);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        xcb_set_last_error(std::string("ba_gram_tc: ") + cudaGetErrorString(e));
        return XCB_ERR_CUDA;
    }
    return XCB_OK;
}
