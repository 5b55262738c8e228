// front_detect.cu -- Shi-Tomasi response, noise floor, cell-scope candidates and the exact greedy pick (sm_100a).
//
// Bit-exactness contract (compiled with --fmad=false; every rounding step is an explicit intrinsic):
//   response  = cv2.cornerMinEigenVal(gray, 3, 3)          (src/xclean/stages/features.py:299; the reference's device
//               form is gpu_front.py:99-202).  OpenCV's arithmetic: separable Sobel with a fused multiply-add chain in
//               the SIMD body of the smoothing row filter (x < dy_vend) and of the derivative column filter
//               (x < dx_vend), float32 products, 3x3 box sum in double with ColumnSum's running sum per column, the
//               min eigenvalue in float32.  The split points are calibrated against cv2 at start-up.
//   floor     = features.noise_floor_8u (features.py:57-73), numpy's float32 pairwise summation tree.
//   picks     = Frontend._response cell scope + Frontend._detect greedy + _subpix (features.py:288-403).
//
// B200 layout: frames are batched along grid.y; the response is ONE kernel per batch (u8 in, float32 R out: the
// reference's dx/dy/row-sum/cov intermediates, ~100 B/px, never touch HBM).  Candidates are gathered one CTA per
// greedy cell row (coalesced rows) into per-cell lists, each list then sorted by rank, so the greedy kernel advances a
// list head instead of rescanning; the greedy state, the ranking (a bitonic sort of the picks) and the sub-pixel step
// share one CTA per frame in shared memory.
#include "common.cuh"
#include "front_kernels.h"

// ------------------------------------------------------------------------------------------------------------------
// 1. response: one thread per (frame, column); the column walk reproduces ColumnSum's running double sums exactly.
// ------------------------------------------------------------------------------------------------------------------
struct SobelRow {
    float rx, ry;
};

// row-filter outputs of OpenCV's Sobel at column c of one image row from its pixels a = row[c - 1], b = row[c],
// d = row[c + 1] (reflected): rx = derivative taps (-1 0 1), ry = smoothing taps (1 2 1) * scale, fused for c < dy_vend
__device__ __forceinline__ SobelRow sobel_row_v(float a, float b, float d, int c, float ks, float k2s, int dy_vend)
{
    SobelRow o;
    o.rx = __fsub_rn(d, a);
    if (c < dy_vend) {
        float s = __fmul_rn(a, ks);
        s = __fmaf_rn(b, k2s, s);
        s = __fmaf_rn(d, ks, s);
        o.ry = s;
    } else {
        float s = __fmul_rn(ks, a);
        s = __fadd_rn(s, __fmul_rn(k2s, b));
        s = __fadd_rn(s, __fmul_rn(ks, d));
        o.ry = s;
    }
    return o;
}

__device__ __forceinline__ SobelRow sobel_row(const u8* row, int W, int c, float ks, float k2s, int dy_vend)
{
    return sobel_row_v((float)row[XCB_REFL(c - 1, W)], (float)row[c], (float)row[XCB_REFL(c + 1, W)], c, ks, k2s,
                       dy_vend);
}

// Sobel (dx, dy) at column c from the row-filter outputs of the rows above, at and below -> the three products
// dx*dx, dx*dy, dy*dy (float32)
__device__ __forceinline__ void sobel_products3(const SobelRow& r0, const SobelRow& r1, const SobelRow& r2, int c,
                                                float ks, float k2s, int dx_vend, float p[3])
{
    float t = __fadd_rn(r0.rx, r2.rx);
    float dx = (c < dx_vend) ? __fmaf_rn(t, ks, __fmul_rn(r1.rx, k2s))
                             : __fadd_rn(__fmul_rn(t, ks), __fmul_rn(r1.rx, k2s));
    float dy = __fsub_rn(r2.ry, r0.ry);
    p[0] = __fmul_rn(dx, dx);
    p[1] = __fmul_rn(dx, dy);
    p[2] = __fmul_rn(dy, dy);
}

// Sobel products at (y, c)
__device__ __forceinline__ void sobel_products(const u8* I, int H, int W, int y, int c, float ks, float k2s,
                                               int dy_vend, int dx_vend, float p[3])
{
    SobelRow r0 = sobel_row(I + (size_t)XCB_REFL(y - 1, H) * W, W, c, ks, k2s, dy_vend);
    SobelRow r1 = sobel_row(I + (size_t)y * W, W, c, ks, k2s, dy_vend);
    SobelRow r2 = sobel_row(I + (size_t)XCB_REFL(y + 1, H) * W, W, c, ks, k2s, dy_vend);
    sobel_products3(r0, r1, r2, c, ks, k2s, dx_vend, p);
}

// box-filter row sums (double) of the three products at row y, column x
__device__ __forceinline__ void row_sums(const u8* I, int H, int W, int y, int x, float ks, float k2s, int dy_vend,
                                         int dx_vend, double rs[3])
{
    float pm[3], p0[3], pp[3];
    sobel_products(I, H, W, y, XCB_REFL(x - 1, W), ks, k2s, dy_vend, dx_vend, pm);
    sobel_products(I, H, W, y, x, ks, k2s, dy_vend, dx_vend, p0);
    sobel_products(I, H, W, y, XCB_REFL(x + 1, W), ks, k2s, dy_vend, dx_vend, pp);
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) rs[ch] = __dadd_rn(__dadd_rn((double)pm[ch], (double)p0[ch]), (double)pp[ch]);
}

__global__ void __launch_bounds__(128, 7) k_response(const u8* __restrict__ imgs, int H, int W, int dy_vend,
                                                  int dx_vend, float* __restrict__ Rall, int* __restrict__ anypos)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int f = blockIdx.y;
    const u8* I = imgs + (size_t)f * H * W;
    float* R = Rall + (size_t)f * H * W;
    const float ks = (float)(1.0 / (4 * 3 * 255.0));
    const float k2s = (float)(2.0 * (1.0 / (4 * 3 * 255.0)));
    int pos = 0;
    if (x < W) {
        double a[3], b[3], S[3], c[3];
        row_sums(I, H, W, XCB_REFL(-1, H), x, ks, k2s, dy_vend, dx_vend, a);
        row_sums(I, H, W, 0, x, ks, k2s, dy_vend, dx_vend, b);
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) S[ch] = __dadd_rn(__dadd_rn(0.0, a[ch]), b[ch]);
        // the row-filter outputs of image rows y and y + 1 at columns x - 1, x, x + 1 roll down with y, so each step
        // filters one new row, whose nine pixels were loaded a step earlier (the last step, whose rows reflect back
        // up, is computed in full)
        const int cols[3] = {XCB_REFL(x - 1, W), x, XCB_REFL(x + 1, W)};
        int po[3][3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            po[k][0] = XCB_REFL(cols[k] - 1, W); po[k][1] = cols[k]; po[k][2] = XCB_REFL(cols[k] + 1, W);
        }
        SobelRow q0[3], q1[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            q0[k] = sobel_row(I, W, cols[k], ks, k2s, dy_vend);
            q1[k] = sobel_row(I + (size_t)XCB_REFL(1, H) * W, W, cols[k], ks, k2s, dy_vend);
        }
        u8 nb[3][3];
        {
            const u8* rn = I + (size_t)XCB_REFL(2, H) * W;
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
                for (int e = 0; e < 3; ++e) nb[k][e] = rn[po[k][e]];
        }
#pragma unroll 2
        for (int y = 0; y < H; ++y) {
            if (y < H - 1 && H >= 3) {
                u8 cb[3][3];
#pragma unroll
                for (int k = 0; k < 3; ++k)
#pragma unroll
                    for (int e = 0; e < 3; ++e) cb[k][e] = nb[k][e];
                if (y + 1 < H - 1) {
                    const u8* rn = I + (size_t)XCB_REFL(y + 3, H) * W;
#pragma unroll
                    for (int k = 0; k < 3; ++k)
#pragma unroll
                        for (int e = 0; e < 3; ++e) nb[k][e] = rn[po[k][e]];
                }
                float pr[3][3];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const SobelRow q2 = sobel_row_v((float)cb[k][0], (float)cb[k][1], (float)cb[k][2], cols[k], ks,
                                                    k2s, dy_vend);
                    sobel_products3(q0[k], q1[k], q2, cols[k], ks, k2s, dx_vend, pr[k]);
                    q0[k] = q1[k];
                    q1[k] = q2;
                }
#pragma unroll
                for (int ch = 0; ch < 3; ++ch)
                    c[ch] = __dadd_rn(__dadd_rn((double)pr[0][ch], (double)pr[1][ch]), (double)pr[2][ch]);
            } else {
                row_sums(I, H, W, XCB_REFL(y + 1, H), x, ks, k2s, dy_vend, dx_vend, c);
            }
            float cov[3];
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) {
                double s0 = __dadd_rn(S[ch], c[ch]);
                cov[ch] = __double2float_rn(s0);
                S[ch] = __dsub_rn(s0, a[ch]);
                a[ch] = b[ch];
                b[ch] = c[ch];
            }
            float ea = __fmul_rn(cov[0], 0.5f), eb = cov[1], ec = __fmul_rn(cov[2], 0.5f);
            float t = __fsub_rn(ea, ec);
            float v = __fadd_rn(__fmul_rn(t, t), __fmul_rn(eb, eb));
            float r = __fsub_rn(__fadd_rn(ea, ec), __fsqrt_rn(v));
            R[(size_t)y * W + x] = r;
            pos |= r > 0.0f;
        }
    }
    if (__any_sync(0xffffffffu, pos) && (threadIdx.x & 31) == 0) atomicOr(anypos + f, 1);
}

cudaError_t xcb_launch_response(const uint8_t* img, int F, int H, int W, int dy_vend, int dx_vend, float* R,
                                int* anypos, cudaStream_t st)
{
    dim3 grid((W + 127) / 128, F);
    k_response<<<grid, 128, 0, st>>>(img, H, W, dy_vend, dx_vend, R, anypos);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------------------------------
// 2. noise floor: leaves of numpy's pairwise tree in parallel, then the tree level by level (one CTA per frame)
// ------------------------------------------------------------------------------------------------------------------
// |Laplacian-like filter| at the pixel p points to (an integer, exact in float32)
__device__ __forceinline__ float lap_abs_at(const u8* p, int W)
{
    const u8* r0 = p - W;
    const u8* r2 = p + W;
    int v = (int)r0[-1] - 2 * (int)r0[0] + (int)r0[1] - 2 * (int)p[-1] + 4 * (int)p[0] - 2 * (int)p[1] + (int)r2[-1]
            - 2 * (int)r2[0] + (int)r2[1];
    return (float)(v < 0 ? -v : v);
}

#define NOISE_LEAF 128      // numpy's pairwise block: a leaf holds at most 128 elements
#define NOISE_WARPS 8

// one warp per leaf: the lanes evaluate the leaf's elements (consecutive interior pixels: coalesced rows) into shared
// memory, then numpy's order inside a leaf: eight running sums over elements j, j + 8, ... (lane j), combined as
// ((r0 + r1) + (r2 + r3)) + ((r4 + r5) + (r6 + r7)), then the tail; fewer than 8 elements: one sequential sum
__global__ void __launch_bounds__(NOISE_WARPS * 32) k_noise_leaves(const u8* __restrict__ imgs, int H, int W,
                                                                   const long long* __restrict__ lstart,
                                                                   const int* __restrict__ llen, int nleaf,
                                                                   int nnode, float* __restrict__ nodeval)
{
    __shared__ float ev[NOISE_WARPS][NOISE_LEAF];
    const int wl = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int l = blockIdx.x * NOISE_WARPS + wl;
    const int f = blockIdx.y;
    if (l >= nleaf) return;
    const u8* I = imgs + (size_t)f * H * W;
    const long long st = lstart[l];
    const int n = min(llen[l], NOISE_LEAF);
    const int wi = W - 2;
    const int y0 = 1 + (int)(st / wi), x0 = (int)(st % wi);
    float* e = ev[wl];
    for (int i = lane; i < n; i += 32) {
        int xx = x0 + i, y = y0;
        while (xx >= wi) { xx -= wi; ++y; }
        e[i] = lap_abs_at(I + (size_t)y * W + 1 + xx, W);
    }
    __syncwarp();
    float res = 0.0f;
    if (n < 8) {
        if (lane == 0) {
            res = -0.0f;
            for (int i = 0; i < n; ++i) res = __fadd_rn(res, e[i]);
        }
    } else {
        const int lim = n - (n % 8);
        float r = 0.0f;
        if (lane < 8) {
            r = e[lane];
            for (int i = 8 + lane; i < lim; i += 8) r = __fadd_rn(r, e[i]);
        }
        float q[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) q[j] = __shfl_sync(0xffffffffu, r, j);
        if (lane == 0) {
            res = __fadd_rn(__fadd_rn(__fadd_rn(q[0], q[1]), __fadd_rn(q[2], q[3])),
                            __fadd_rn(__fadd_rn(q[4], q[5]), __fadd_rn(q[6], q[7])));
            for (int i = lim; i < n; ++i) res = __fadd_rn(res, e[i]);
        }
    }
    if (lane == 0) nodeval[(size_t)f * nnode + l] = res;
}

__global__ void k_noise_tree(float* __restrict__ nodeval, int nnode, const int* __restrict__ left,
                             const int* __restrict__ right, const int* __restrict__ lvl, int nlvl, int root, double K,
                             double Q, double* __restrict__ floor_d, float* __restrict__ floor_f)
{
    int f = blockIdx.x;
    float* val = nodeval + (size_t)f * nnode;
    for (int h = 0; h < nlvl; ++h) {
        for (int i = lvl[h] + threadIdx.x; i < lvl[h + 1]; i += blockDim.x) val[i] = __fadd_rn(val[left[i]], val[right[i]]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double sn = __dmul_rn(K, (double)val[root]);
        double fl = __ddiv_rn(__dmul_rn(__dmul_rn(Q, sn), sn), 65025.0);
        floor_d[f] = fl;
        floor_f[f] = __double2float_rn(fl);
    }
}

cudaError_t xcb_launch_noise(const uint8_t* img, int F, int H, int W, const XcbNoiseTree& t, float* nodeval,
                             double K, double Q, double* floor_d, float* floor_f, cudaStream_t st)
{
    dim3 g1((t.nleaf + NOISE_WARPS - 1) / NOISE_WARPS, F);
    k_noise_leaves<<<g1, NOISE_WARPS * 32, 0, st>>>(img, H, W, t.lstart, t.llen, t.nleaf, t.nnode, nodeval);
    k_noise_tree<<<F, 1024, 0, st>>>(nodeval, t.nnode, t.left, t.right, t.lvl, t.nlvl, t.root, K, Q, floor_d, floor_f);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------------------------------
// 3. thresholds (0.01 x the c x c cell max of the zero-padded response) and the per-cell candidate lists
// ------------------------------------------------------------------------------------------------------------------
// one CTA per threshold-cell row: column maxima over the row's c image rows (coalesced), then one thread per cell;
// a cell reaching past the image (the zero pad) also takes max(., 0)
#define CMAX_T 256
#define CMAX_MAXW 8192
__global__ void __launch_bounds__(CMAX_T) k_cellmax(const float* __restrict__ Rall, int H, int W, int c, int gwc,
                                                    int ghc, float* __restrict__ thr)
{
    __shared__ float colmax[CMAX_MAXW];
    const int gy = blockIdx.x, f = blockIdx.y, tid = threadIdx.x;
    const float* R = Rall + (size_t)f * H * W;
    const int y0 = gy * c, y1 = min(y0 + c, H);
    for (int x = tid; x < W; x += CMAX_T) {
        float m = -CUDART_INF_F;
        for (int y = y0; y < y1; ++y) m = fmaxf(m, R[(size_t)y * W + x]);
        colmax[x] = m;
    }
    __syncthreads();
    for (int gx = tid; gx < gwc; gx += CMAX_T) {
        const int x0 = gx * c, x1 = min(x0 + c, W);
        float m = -CUDART_INF_F;
        for (int x = x0; x < x1; ++x) m = fmaxf(m, colmax[x]);
        if (y0 + c > H || x0 + c > W) m = fmaxf(m, 0.0f);
        thr[(size_t)f * gwc * ghc + (size_t)gy * gwc + gx] = __fmul_rn(0.01f, m);
    }
}

// candidates (3x3 local max of the response, >= its threshold cell's 0.01 max, >= the noise floor, inside the border):
// one CTA per (greedy cell row, frame), threads over columns so every row is read coalesced; a candidate is appended
// to its cell's list through a shared-memory counter, then each cell's list (keys are unique) is ranked into the
// sorted list (one warp per cell)
#define CAND_T 256
#define CAND_MAXCX 1024
__global__ void __launch_bounds__(CAND_T) k_cell_candidates(const float* __restrict__ Rall, int H, int W, int b, int ncx,
                                                            int ncell, const int* __restrict__ ybeg,
                                                            const int* __restrict__ xbeg, const int* __restrict__ coff,
                                                            int c, int gwc, int ghc, const float* __restrict__ thr,
                                                            const float* __restrict__ floor_f,
                                                            const int* __restrict__ anypos, u64* raw,
                                                            u64* __restrict__ sorted, int* __restrict__ ccount,
                                                            long long list_stride)
{
    __shared__ int cnt[CAND_MAXCX];
    __shared__ int sxb[CAND_MAXCX + 1];
    const int cy = blockIdx.x, f = blockIdx.y, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int i = tid; i < ncx; i += CAND_T) cnt[i] = 0;
    for (int i = tid; i <= ncx; i += CAND_T) sxb[i] = xbeg[i];
    __syncthreads();
    const int c0 = cy * ncx;
    u64* fraw = raw + (size_t)f * list_stride;
    if (anypos[f]) {               // rmax <= 0: no candidates (Frontend._response)
        const float* R = Rall + (size_t)f * H * W;
        const float* T = thr + (size_t)f * gwc * ghc;
        const float fl = floor_f[f];
        const int ya = max(ybeg[cy], b), yb = min(ybeg[cy + 1], H - b);
        for (int x = b + tid; x < W - b; x += CAND_T) {
            int lo = 0, hi = ncx - 1;            // the cell column holding x: the last start <= x
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (sxb[mid] <= x) lo = mid; else hi = mid - 1;
            }
            const int tx = x / c;
            u64* lraw = fraw + coff[c0 + lo];
            for (int y = ya; y < yb; ++y) {
                const float* q = R + (size_t)y * W + x;
                const float v = q[0];
                float m = v;
#pragma unroll
                for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
                    for (int dx = -1; dx <= 1; ++dx) m = fmaxf(m, q[dy * W + dx]);
                if (v >= m && v >= T[(y / c) * gwc + tx] && v >= fl) lraw[atomicAdd(&cnt[lo], 1)] = xcb_key(v, y, x);
            }
        }
    }
    __syncthreads();
    for (int cx = wid; cx < ncx; cx += CAND_T / 32) {
        const int cell = c0 + cx, n = cnt[cx];
        const u64* lraw = fraw + coff[cell];
        u64* ls = sorted + (size_t)f * list_stride + coff[cell];
        for (int i = lane; i < n; i += 32) {
            const u64 k = lraw[i];
            int rank = 0;
            for (int j = 0; j < n; ++j) rank += lraw[j] > k;
            ls[rank] = k;
        }
        if (lane == 0) ccount[(size_t)f * ncell + cell] = n;
    }
}

cudaError_t xcb_launch_candidates(const float* R, int F, int H, int W, const XcbDetectGeom& g, const float* floor_f,
                                  const int* anypos, float* thr, unsigned long long* raw, unsigned long long* sorted,
                                  int* ccount, cudaStream_t st)
{
    if (W > CMAX_MAXW) return cudaErrorInvalidValue;
    dim3 g1(g.ghc, F);
    k_cellmax<<<g1, CMAX_T, 0, st>>>(R, H, W, g.c, g.gwc, g.ghc, thr);
    if (g.ncx > CAND_MAXCX) return cudaErrorInvalidValue;
    dim3 g2(g.gh, F);
    k_cell_candidates<<<g2, CAND_T, 0, st>>>(R, H, W, g.border, g.ncx, g.ncell, g.ybeg, g.xbeg, g.coff, g.c, g.gwc,
                                             g.ghc, thr, floor_f, anypos, raw, sorted, ccount, (long long)H * W);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------------------------------
// 4. the exact greedy (one CTA per frame): strongest first, one pick per cell, none within r (strict <) of a
//    higher-ranked pick.  Each cell holds its best unskipped candidate; a cell commits when no neighbouring undecided
//    cell holds a higher-ranked candidate, and skips a candidate within r of a committed higher-ranked neighbour pick.
//    The globally highest undecided candidate is never waiting, so every round decides something and the committed
//    set equals the sequential loop's; ranking the picks and keeping the first n gives its first n picks.
// ------------------------------------------------------------------------------------------------------------------
#define ST_UNDECIDED 0
#define ST_PICK 1
#define ST_NONE 2
#define GREEDY_THREADS 1024

// shared-memory layout of k_greedy: key u64 [ncell] | head int [ncell] | state u8 [ncell] | picks u64 [p2]
__host__ __device__ __forceinline__ size_t greedy_picks_offset(int ncell)
{
    return ((size_t)ncell * 13 + 15) & ~(size_t)15;
}

size_t xcb_greedy_smem(int ncell)
{
    int p2 = 1;
    while (p2 < ncell) p2 <<= 1;
    return greedy_picks_offset(ncell) + (size_t)p2 * 8;
}

// the B200 opt-in maximum is 227 KB per block including the kernel's static shared variables
int xcb_greedy_smem_limit() { return 226 * 1024; }

__global__ void __launch_bounds__(GREEDY_THREADS) k_greedy(const float* __restrict__ Rall, int H, int W, int ncx,
                                                           int gh, int ncell, double r2,
                                                           const int* __restrict__ coff,
                                                           const u64* __restrict__ sorted_all,
                                                           const int* __restrict__ ccount_all, long long list_stride,
                                                           int budget, int cap, int max_rounds, float* __restrict__ kp,
                                                           int* __restrict__ counts, int* __restrict__ rounds_out,
                                                           unsigned int* __restrict__ err)
{
    extern __shared__ __align__(16) unsigned char smem[];
    int p2 = 1;
    while (p2 < ncell) p2 <<= 1;
    volatile u64* key = (volatile u64*)smem;
    volatile int* head = (volatile int*)(smem + (size_t)ncell * 8);
    volatile u8* state = (volatile u8*)(smem + (size_t)ncell * 12);
    u64* picks = (u64*)(smem + greedy_picks_offset(ncell));
    __shared__ int unresolved, npick;

    const int f = blockIdx.x, tid = threadIdx.x;
    const u64* lists = sorted_all + (size_t)f * list_stride;
    const int* cnt = ccount_all + (size_t)f * ncell;

    for (int c = tid; c < ncell; c += GREEDY_THREADS) {
        head[c] = 0;
        if (cnt[c] > 0) { key[c] = lists[coff[c]]; state[c] = ST_UNDECIDED; }
        else { key[c] = 0; state[c] = ST_NONE; }
    }
    if (tid == 0) npick = 0;
    __syncthreads();

    int round = 0;
    for (;;) {
        if (tid == 0) unresolved = 0;
        __syncthreads();
        for (int c = tid; c < ncell; c += GREEDY_THREADS) {
            if (state[c] != ST_UNDECIDED) continue;
            const int gx = c % ncx, gy = c / ncx;
            for (;;) {
                const u64 kk = key[c];
                const int qx = xcb_key_x(kk), qy = xcb_key_y(kk);
                bool blocked = false, wait = false;
                for (int ny = gy - 1; ny <= gy + 1 && !blocked; ++ny) {
                    if (ny < 0 || ny >= gh) continue;
                    for (int nx = gx - 1; nx <= gx + 1; ++nx) {
                        if (nx < 0 || nx >= ncx) continue;
                        const int nb = ny * ncx + nx;
                        if (nb == c) continue;
                        const int s = state[nb];
                        if (s == ST_PICK) {
                            __threadfence_block();
                            const u64 pk = key[nb];
                            if (pk > kk) {
                                long long ddx = (long long)xcb_key_x(pk) - qx, ddy = (long long)xcb_key_y(pk) - qy;
                                if ((double)(ddx * ddx + ddy * ddy) < r2) { blocked = true; break; }
                            }
                        } else if (s == ST_UNDECIDED) {
                            if (key[nb] > kk) wait = true;
                        }
                    }
                }
                if (blocked) {
                    const int h = head[c] + 1;
                    head[c] = h;
                    if (h >= cnt[c]) { __threadfence_block(); state[c] = ST_NONE; break; }
                    key[c] = lists[coff[c] + h];
                    continue;
                }
                if (wait) { atomicAdd(&unresolved, 1); break; }
                __threadfence_block();
                state[c] = ST_PICK;
                break;
            }
        }
        __syncthreads();
        ++round;
        const int u = unresolved;
        if (u == 0) break;
        if (round >= max_rounds) {
            if (tid == 0) atomicOr(err, XCB_DEVERR_GREEDY_ROUNDS);
            break;
        }
        __syncthreads();
    }
    __syncthreads();
    // picks -> power-of-two buffer, zero padded; bitonic sort descending (keys are unique and non-zero)
    for (int c = tid; c < ncell; c += GREEDY_THREADS)
        if (state[c] == ST_PICK) picks[atomicAdd(&npick, 1)] = key[c];
    __syncthreads();
    const int P = npick;
    for (int i = P + tid; i < p2; i += GREEDY_THREADS) picks[i] = 0ull;
    __syncthreads();
    for (int k = 2; k <= p2; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < p2; i += GREEDY_THREADS) {
                int ixj = i ^ j;
                if (ixj > i) {
                    u64 a = picks[i], bb = picks[ixj];
                    bool desc = (i & k) == 0;
                    if (desc ? (a < bb) : (a > bb)) { picks[i] = bb; picks[ixj] = a; }
                }
            }
            __syncthreads();
        }
    }
    int n_out = P < budget ? P : budget;
    if (n_out > cap) n_out = cap;
    const float* R = Rall + (size_t)f * H * W;
    float* kpo = kp + (size_t)f * cap * 2;
    for (int i = tid; i < n_out; i += GREEDY_THREADS) {
        const u64 k = picks[i];
        const int x = xcb_key_x(k), y = xcb_key_y(k);
        double fx = (double)x, fy = (double)y;
        if (x > 0 && x < W - 1 && y > 0 && y < H - 1) {
            const float* q = R + (size_t)y * W + x;
            double cc = q[0], l = q[-1], rr = q[1], u = q[-W], d = q[W];
            double c2 = __dmul_rn(2.0, cc);
            double denx = __dadd_rn(__dsub_rn(l, c2), rr);
            double deny = __dadd_rn(__dsub_rn(u, c2), d);
            double dx = denx < 0.0 ? __ddiv_rn(__dmul_rn(0.5, __dsub_rn(l, rr)), denx) : 0.0;
            double dy = deny < 0.0 ? __ddiv_rn(__dmul_rn(0.5, __dsub_rn(u, d)), deny) : 0.0;
            dx = fmin(fmax(dx, -0.5), 0.5);
            dy = fmin(fmax(dy, -0.5), 0.5);
            fx = __dadd_rn(fx, dx);
            fy = __dadd_rn(fy, dy);
        }
        kpo[2 * i] = __double2float_rn(fx);
        kpo[2 * i + 1] = __double2float_rn(fy);
    }
    if (tid == 0) {
        counts[f] = n_out;
        if (rounds_out) rounds_out[f] = round;
    }
}

cudaError_t xcb_greedy_init_attrs()
{
    return cudaFuncSetAttribute(k_greedy, cudaFuncAttributeMaxDynamicSharedMemorySize, xcb_greedy_smem_limit());
}

cudaError_t xcb_launch_greedy(const float* R, int F, int H, int W, const XcbDetectGeom& g,
                              const unsigned long long* sorted, const int* ccount, int budget, int cap, float* kp,
                              int* counts, int* rounds, unsigned int* err, cudaStream_t st)
{
    size_t sm = xcb_greedy_smem(g.ncell);
    // every round decides at least one candidate: the bound is the candidate count, at most H * W
    int max_rounds = H * W + 1;
    k_greedy<<<F, GREEDY_THREADS, sm, st>>>(R, H, W, g.ncx, g.gh, g.ncell, g.r2, g.coff, sorted, ccount,
                                            (long long)H * W, budget, cap, max_rounds, kp, counts, rounds, err);
    return cudaGetLastError();
}
