// front_mapmatch.cu -- gated map matching on the device: MapMatcher.match (src/xclean/front/mapmatch.py:148-169 with
// its numba _gated, mapmatch.py:49-131, and grid, :141-146; the same outputs as front/mapmatch_fast.MapMatcher.match,
// mapmatch_fast.py:113-184) for one frame from host arrays, or for a batch of frames resident in device memory.
//
// Three launches per call (grid.y = frame):
//   k_mm_grid    one CTA per frame builds the 16-px keypoint grid: cell counts by shared-memory atomics, a block scan
//                into cell starts, then each keypoint's index stored in its cell's range (any order inside a cell).
//   k_mm_gate    two lanes per landmark: the gate preamble (det, Sinv, half-widths, the box of cells under the
//                ellipse), then the lanes walk the box's cell rows side by side (one contiguous range of entries per
//                row), apply the Mahalanobis gate, take the minimum Hamming distance over the landmark's descriptors and
//                keep a lane-local best / second best, merged across the two lanes; chance bound and Lowe ratio; an
//                accepted landmark claims its keypoint, counts itself on it and leaves its id in one of the keypoint's
//                four claimant slots.
//   k_mm_mutual  one thread per landmark: a keypoint with a single claimant goes to it; the reference's owner fold
//                over the claimants in landmark order is replayed from the slots (up to four claimants) or by the warp
//                over all of the frame's claims (more).
//
// Why the gate may merge in any order: the reference visits the box's cells row by row and a cell's keypoints in index
// order, and only an equal best distance with a smaller d2 displaces the running best.  Any tie at the best distance
// also sets the second-best distance to that value, and then the ratio test (best < 0.8 second) rejects the landmark.
// An accepted landmark therefore has exactly one keypoint at its best distance, whatever the visit order, and its d2
// (NaN included) is that keypoint's.  The owner fold of the mutual step is order-dependent (NaN d2 included) and is
// replayed in landmark order as written.
//
// Every floating-point step is an explicit round-to-nearest intrinsic in the reference's evaluation order (the file is
// also built with --fmad=false).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <string>

#include "common.cuh"

extern void xcb_set_last_error(const std::string& m);

#define MM_GRID 16            // mapmatch.py:30
#define MM_GRID_T 1024        // threads of k_mm_grid
#define MM_WARPS 8            // warps per CTA of k_mm_gate / k_mm_mutual
#define MM_GROUP_DEFAULT 2    // lanes per landmark in k_mm_gate (1, 2, 4 or 8: the tuner's choice per device and
                              // shape; 2 measured faster than 4 and 8 on B200: more landmarks in flight)
#define MM_SLOTS 4            // claimant ids kept per keypoint (more claimants: the ordered scan of all claims)
// x / 16 and x * 0.0625 are the same correctly rounded double for every x (scaling by a power of two)
#define MM_INV_GRID 0.0625
#define MM_MAX_CELLS 49152    // cell counts of one frame live in shared memory (192 KB)
#define MM_NONE 9999          // mapmatch.py:57-59 "no distance"

struct MMArgs {
    const void* kp;           // [F][kp_stride][2] float32 or float64 (x, y)
    const int* nkp;           // [F] keypoint counts on the device, or NULL: nkp1 for every frame
    int nkp1, kp_stride;
    const u8* desc;           // [F][kp_stride][32]
    const double* uv;         // [F][lm_stride][2] predicted projections
    const double* S;          // [F][lm_stride][2][2] innovation covariances
    const u8* lmd;            // [F][lm_stride][D][32] landmark descriptors
    const i64* lnd;           // [F][lm_stride] valid descriptors per landmark (values above D read as D)
    const int* nlm;           // [F] landmark counts on the device, or NULL: nlm1
    int nlm1, lm_stride, D;
    double chi2, ratio;
    int ham_max, gw, gh, ncell;
    int* cstart;              // [F][ncell + 1]
    int* slot;                // [F][kp_stride]
    int* ent;                 // [F][kp_stride] keypoint indices grouped by cell
    int* claim;               // [F][lm_stride] keypoint claimed after the gate, or -1
    int* kcnt;                // [F][kp_stride] landmarks claiming each keypoint
    int* kslot;               // [F][kp_stride][MM_SLOTS] the first MM_SLOTS of them, in arrival order
    i64* out_kp;              // [F][lm_stride]
    i64* out_d;
    double* out_d2;
};

// float64 -> int64 as x86-64 converts it (numpy astype(np.int64), numba int()): NaN and out-of-range -> INT64_MIN
__device__ __forceinline__ i64 mm_f2i(double v)
{
    if (!(v >= -9223372036854775808.0 && v < 9223372036854775808.0)) return (i64)0x8000000000000000ull;
    return (i64)v;
}

__device__ __forceinline__ int mm_clampi(i64 v, int hi) { return (int)(v < 0 ? 0 : (v > hi ? hi : v)); }

template <typename KT>
__device__ __forceinline__ void mm_kp(const MMArgs& a, size_t i, double& x, double& y)
{
    const KT* p = (const KT*)a.kp + 2 * i;
    x = (double)p[0];
    y = (double)p[1];
}

// the keypoint's cell (mapmatch.py:141-144): clip(x // 16) + gw clip(y // 16)
template <typename KT>
__device__ __forceinline__ int mm_cell(const MMArgs& a, size_t i)
{
    double x, y;
    mm_kp<KT>(a, i, x, y);
    const int cx = mm_clampi(mm_f2i(floor(__dmul_rn(x, MM_INV_GRID))), a.gw - 1);
    const int cy = mm_clampi(mm_f2i(floor(__dmul_rn(y, MM_INV_GRID))), a.gh - 1);
    return cy * a.gw + cx;
}

__device__ __forceinline__ int mm_nkp(const MMArgs& a, int f)
{
    const int n = a.nkp ? a.nkp[f] : a.nkp1;
    return n < 0 ? 0 : (n > a.kp_stride ? a.kp_stride : n);
}

__device__ __forceinline__ int mm_nlm(const MMArgs& a, int f)
{
    const int n = a.nlm ? a.nlm[f] : a.nlm1;
    return n < 0 ? 0 : (n > a.lm_stride ? a.lm_stride : n);
}

// ------------------------------------------------------------------------------------------------ grid (one CTA/frame)
template <typename KT>
__global__ void __launch_bounds__(MM_GRID_T) k_mm_grid(MMArgs a)
{
    extern __shared__ int s_cnt[];          // [ncell + 1]
    __shared__ int s_wsum[MM_GRID_T / 32];
    const int f = blockIdx.x, tid = threadIdx.x, n = mm_nkp(a, f), nc = a.ncell;
    const size_t kb = (size_t)f * a.kp_stride;
    for (int c = tid; c <= nc; c += MM_GRID_T) s_cnt[c] = 0;
    __syncthreads();
    for (int k = tid; k < n; k += MM_GRID_T) {
        a.slot[kb + k] = atomicAdd(&s_cnt[mm_cell<KT>(a, kb + k)], 1);
        a.kcnt[kb + k] = 0;
    }
    __syncthreads();
    // exclusive scan of the counts: a contiguous run of cells per thread, then the run totals across the block
    const int per = (nc + MM_GRID_T - 1) / MM_GRID_T, c0 = tid * per, c1 = min(nc, c0 + per);
    int run = 0;
    for (int c = c0; c < c1; ++c) run += s_cnt[c];
    int incl = run;
    const int lane = tid & 31, w = tid >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) s_wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
        int v = s_wsum[lane], iv = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, iv, o);
            if (lane >= o) iv += t;
        }
        s_wsum[lane] = iv - v;             // exclusive warp offsets
    }
    __syncthreads();
    int acc = s_wsum[w] + incl - run;
    for (int c = c0; c < c1; ++c) {
        const int v = s_cnt[c];
        s_cnt[c] = acc;
        acc += v;
    }
    if (tid == MM_GRID_T - 1) s_cnt[nc] = acc;
    __syncthreads();
    int* cs = a.cstart + (size_t)f * (nc + 1);
    for (int c = tid; c <= nc; c += MM_GRID_T) cs[c] = s_cnt[c];
    for (int k = tid; k < n; k += MM_GRID_T) {
        const int c = mm_cell<KT>(a, kb + k);
        a.ent[kb + s_cnt[c] + a.slot[kb + k]] = k;
    }
}

__device__ __forceinline__ int mm_ham(const uint4* p, const uint4* q)
{
    const uint4 a0 = p[0], a1 = p[1], b0 = __ldg(q), b1 = __ldg(q + 1);
    return __popc(a0.x ^ b0.x) + __popc(a0.y ^ b0.y) + __popc(a0.z ^ b0.z) + __popc(a0.w ^ b0.w)
           + __popc(a1.x ^ b1.x) + __popc(a1.y ^ b1.y) + __popc(a1.z ^ b1.z) + __popc(a1.w ^ b1.w);
}

// ----------------------------------------------------------------------------- gate (2 lanes per landmark, 128 per CTA)
template <typename KT, int MM_GROUP>
__global__ void __launch_bounds__(MM_WARPS * 32, 4) k_mm_gate(MMArgs a)
{
    constexpr int MM_LPB = MM_WARPS * 32 / MM_GROUP;     // landmarks per CTA
    const int lane = threadIdx.x & 31, gl = lane & (MM_GROUP - 1), f = blockIdx.y;
    const int l = blockIdx.x * MM_LPB + (threadIdx.x / MM_GROUP);
    const bool in = l < mm_nlm(a, f);
    const size_t li = (size_t)f * a.lm_stride + (in ? l : 0);
    const size_t kb = (size_t)f * a.kp_stride;
    int best = MM_NONE, second = MM_NONE, bk = -1;
    double bd2 = XCB_INF;
    if (in) {
        if (gl == 0) {
            a.out_kp[li] = -1;
            a.out_d[li] = MM_NONE;
            a.out_d2[li] = XCB_INF;
            a.claim[li] = -1;
        }
        // preamble (mapmatch.py:158-166): det, Sinv where det > 0 (else no descriptors), half = sqrt(max(chi2 S_ii, 0))
        const double s00 = a.S[4 * li], s01 = a.S[4 * li + 1], s10 = a.S[4 * li + 2], s11 = a.S[4 * li + 3];
        const double u = a.uv[2 * li], v = a.uv[2 * li + 1];
        i64 nd = a.lnd[li];
        if (nd > a.D) nd = a.D;
        const double det = __dsub_rn(__dmul_rn(s00, s11), __dmul_rn(s01, s10));
        if (!(det > 0)) nd = 0;
        if (nd > 0 && isfinite(u) && isfinite(v)) {
            const double i00 = __ddiv_rn(s11, det), i11 = __ddiv_rn(s00, det);
            const double i01 = __ddiv_rn(-s01, det), i10 = __ddiv_rn(-s10, det);
            const double h0 = __dmul_rn(a.chi2, s00), h1 = __dmul_rn(a.chi2, s11);
            const double hx = __dsqrt_rn((h0 >= 0.0 || isnan(h0)) ? h0 : 0.0);
            const double hy = __dsqrt_rn((h1 >= 0.0 || isnan(h1)) ? h1 : 0.0);
            // the box of cells (mapmatch.py:58-72), int64 as the reference computes it, then clamped
            i64 x0 = mm_f2i(floor(__dmul_rn(__dsub_rn(u, hx), MM_INV_GRID)));
            i64 x1 = mm_f2i(floor(__dmul_rn(__dadd_rn(u, hx), MM_INV_GRID)));
            i64 y0 = mm_f2i(floor(__dmul_rn(__dsub_rn(v, hy), MM_INV_GRID)));
            i64 y1 = mm_f2i(floor(__dmul_rn(__dadd_rn(v, hy), MM_INV_GRID)));
            if (x0 < 0) x0 = 0;
            if (y0 < 0) y0 = 0;
            if (x1 > a.gw - 1) x1 = a.gw - 1;
            if (y1 > a.gh - 1) y1 = a.gh - 1;
            if (x0 <= x1 && y0 <= y1) {    // then 0 <= x0 <= x1 < gw and 0 <= y0 <= y1 < gh
                const int* cs = a.cstart + (size_t)f * (a.ncell + 1);
                const int* en = a.ent + kb;
                const uint4* ld = (const uint4*)(a.lmd + li * (size_t)a.D * 32);
                const int nrows = (int)(y1 - y0) + 1;
                // the rows of the box side by side: with m rows in a pass, lane gl walks row gl % m from entry
                // gl / m with a stride of the number of lanes on that row
                for (int r0 = 0; r0 < nrows; r0 += MM_GROUP) {
                    const int m = min(MM_GROUP, nrows - r0), rr = gl % m;
                    const int sub = gl / m, stride = (MM_GROUP - rr + m - 1) / m;
                    const int row = ((int)y0 + r0 + rr) * a.gw;
                    const int t1 = cs[row + (int)x1 + 1];
                    for (int t = cs[row + (int)x0] + sub; t < t1; t += stride) {
                        const int k = en[t];
                        double x, y;
                        mm_kp<KT>(a, kb + k, x, y);
                        const double dx = __dsub_rn(x, u), dy = __dsub_rn(y, v);
                        const double d2 = __dadd_rn(__dmul_rn(dx, __dadd_rn(__dmul_rn(i00, dx), __dmul_rn(i01, dy))),
                                                    __dmul_rn(dy, __dadd_rn(__dmul_rn(i10, dx), __dmul_rn(i11, dy))));
                        if (d2 > a.chi2) continue;
                        const uint4* kd = (const uint4*)(a.desc + (kb + k) * 32);
                        int h = MM_NONE;
                        for (int j = 0; j < (int)nd; ++j) h = min(h, mm_ham(ld + 2 * j, kd));
                        if (h < best) {
                            second = best;
                            best = h;
                            bk = k;
                            bd2 = d2;
                        } else if (h < second) {
                            second = h;
                        }
                    }
                }
            }
        }
    }
    // merge the landmark's lanes: best = minimum, second = second smallest of the union, keypoint of the (best,
    // index) minimum (an accepted landmark has a single keypoint at its best distance)
#pragma unroll
    for (int o = MM_GROUP / 2; o > 0; o >>= 1) {
        const int ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int os = __shfl_xor_sync(0xffffffffu, second, o);
        const int ok = __shfl_xor_sync(0xffffffffu, bk, o);
        const double od2 = __shfl_xor_sync(0xffffffffu, bd2, o);
        second = min(max(best, ob), min(second, os));
        if (ob < best || (ob == best && ok < bk)) {
            best = ob;
            bk = ok;
            bd2 = od2;
        }
    }
    if (!in || gl != 0 || bk < 0 || best > a.ham_max) return;
    if (second < MM_NONE && !((double)best < __dmul_rn(a.ratio, (double)second))) return;
    a.claim[li] = bk;
    a.out_d[li] = best;
    a.out_d2[li] = bd2;
    const int pos = atomicAdd(&a.kcnt[kb + bk], 1);
    if (pos < MM_SLOTS) a.kslot[(kb + bk) * MM_SLOTS + pos] = l;
}

// ---------------------------------------------------------------------------- mutual best (one thread per landmark)
// mapmatch.py:113-131: claimants in landmark order; a later one takes the keypoint only with a smaller distance, or an
// equal distance and a smaller d2.  A keypoint with one claimant goes to it; with up to MM_SLOTS claimants the thread
// sorts their ids and replays the fold; with more, the warp replays it over the frame's claims, 32 landmarks per step,
// until it has seen all of the keypoint's claimants.
__global__ void __launch_bounds__(MM_WARPS * 32) k_mm_mutual(MMArgs a)
{
    const int lane = threadIdx.x & 31, f = blockIdx.y, L = mm_nlm(a, f);
    const int l = blockIdx.x * (MM_WARPS * 32) + threadIdx.x;
    const size_t lb = (size_t)f * a.lm_stride, kb = (size_t)f * a.kp_stride;
    const int k = l < L ? a.claim[lb + l] : -1;
    int cnt = 0;
    if (k >= 0) {
        cnt = a.kcnt[kb + k];
        if (cnt == 1) {
            a.out_kp[lb + l] = k;
        } else if (cnt <= MM_SLOTS) {
            int id[MM_SLOTS];
#pragma unroll
            for (int j = 0; j < MM_SLOTS; ++j) id[j] = j < cnt ? a.kslot[(kb + k) * MM_SLOTS + j] : INT_MAX;
#pragma unroll
            for (int i = 1; i < MM_SLOTS; ++i)        // landmark order
#pragma unroll
                for (int j = MM_SLOTS - 1; j >= i; --j)
                    if (id[j] < id[j - 1]) {
                        const int t = id[j];
                        id[j] = id[j - 1];
                        id[j - 1] = t;
                    }
            int owner = id[0];
            i64 od = a.out_d[lb + owner];
            double od2 = a.out_d2[lb + owner];
#pragma unroll
            for (int j = 1; j < MM_SLOTS; ++j) {
                if (j >= cnt) break;
                const i64 d = a.out_d[lb + id[j]];
                const double d2 = a.out_d2[lb + id[j]];
                if (d < od || (d == od && d2 < od2)) {
                    owner = id[j];
                    od = d;
                    od2 = d2;
                }
            }
            if (owner == l) a.out_kp[lb + l] = k;
        }
    }
    unsigned todo = __ballot_sync(0xffffffffu, cnt > MM_SLOTS);
    while (todo) {
        const int src = __ffs(todo) - 1;
        todo &= todo - 1;
        const int kk = __shfl_sync(0xffffffffu, k, src), n = __shfl_sync(0xffffffffu, cnt, src);
        const int me = l - lane + src;
        int owner = -1, seen = 0;
        i64 od = 0;
        double od2 = 0.0;
        for (int base = 0; base < L && seen < n; base += 32) {
            const int j = base + lane;
            unsigned m = __ballot_sync(0xffffffffu, j < L && a.claim[lb + j] == kk);
            seen += __popc(m);
            while (m) {
                const int l2 = base + __ffs(m) - 1;
                m &= m - 1;
                const i64 d = a.out_d[lb + l2];
                const double d2 = a.out_d2[lb + l2];
                if (owner < 0 || d < od || (d == od && d2 < od2)) {
                    owner = l2;
                    od = d;
                    od2 = d2;
                }
            }
        }
        if (lane == src && owner == me) a.out_kp[lb + me] = kk;
    }
}

// ================================================================================================== handle + C ABI
struct xcb_mm {
    int W, H, gw, gh, ncell, maxF, cap_kp, cap_lm;
    int lanes;                // lanes per landmark in k_mm_gate (XCB_TUNE_MM_LANES)
    cudaStream_t stream;
    int* d_cstart;
    int* d_slot;
    int* d_ent;
    int* d_claim;
    int* d_kcnt;
    int* d_kslot;
    // host entry: one pinned staging block and its device twin for the inputs, the same for the outputs
    size_t in_cap, out_cap;
    char *h_in, *d_in, *h_out, *d_out;
    std::string err;
};

static int mm_fail(xcb_mm* m, int code, const std::string& msg)
{
    if (m) m->err = msg;
    xcb_set_last_error(msg);
    return code;
}

#define MCK(call, where)                                                                                  \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess) return mm_fail(m, XCB_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e_)); \
    } while (0)

static void mm_free_scratch(xcb_mm* m)
{
    cudaFree(m->d_cstart);
    cudaFree(m->d_slot);
    cudaFree(m->d_ent);
    cudaFree(m->d_claim);
    cudaFree(m->d_kcnt);
    cudaFree(m->d_kslot);
    m->d_kcnt = nullptr;
    m->d_kslot = nullptr;
    m->d_cstart = nullptr;
    m->d_slot = nullptr;
    m->d_ent = nullptr;
    m->d_claim = nullptr;
}

static int mm_alloc_scratch(xcb_mm* m, int cap_kp, int cap_lm)
{
    mm_free_scratch(m);
    const size_t F = (size_t)m->maxF, nk = (size_t)std::max(cap_kp, 1), nl = (size_t)std::max(cap_lm, 1);
    MCK(cudaMalloc(&m->d_cstart, F * (m->ncell + 1) * sizeof(int)), "mapmatch scratch");
    MCK(cudaMalloc(&m->d_slot, F * nk * sizeof(int)), "mapmatch scratch");
    MCK(cudaMalloc(&m->d_ent, F * nk * sizeof(int)), "mapmatch scratch");
    MCK(cudaMalloc(&m->d_claim, F * nl * sizeof(int)), "mapmatch scratch");
    MCK(cudaMalloc(&m->d_kcnt, F * nk * sizeof(int)), "mapmatch scratch");
    MCK(cudaMalloc(&m->d_kslot, F * nk * MM_SLOTS * sizeof(int)), "mapmatch scratch");
    m->cap_kp = cap_kp;
    m->cap_lm = cap_lm;
    return XCB_OK;
}

extern "C" int xcb_mm_create(int width, int height, int max_frames, int max_kp, int max_lm, xcb_mm** out)
{
    if (!out) return mm_fail(nullptr, XCB_ERR_ARG, "mm_create: null output");
    *out = nullptr;
    if (width < 1 || height < 1 || max_frames < 1 || max_kp < 0 || max_lm < 0)
        return mm_fail(nullptr, XCB_ERR_ARG, "mm_create: bad size");
    const long long gw = (width + MM_GRID - 1) / MM_GRID, gh = (height + MM_GRID - 1) / MM_GRID;
    if (gw * gh > MM_MAX_CELLS) return mm_fail(nullptr, XCB_ERR_ARG, "mm_create: more than 49152 grid cells");
    xcb_mm* m = new xcb_mm();
    m->W = width;
    m->H = height;
    m->gw = (int)gw;
    m->gh = (int)gh;
    m->ncell = (int)(gw * gh);
    m->maxF = max_frames;
    m->lanes = MM_GROUP_DEFAULT;
    // the shared-memory opt-in is per kernel, not per handle: raise it to the largest grid any handle has asked for
    static XcbAttrOnce s_attr_f, s_attr_d;
    const int smem = (m->ncell + 1) * (int)sizeof(int);
    int rc = XCB_OK;
    if (xcb_smem_attr_once(s_attr_f, (const void*)k_mm_grid<float>, smem) != cudaSuccess
        || xcb_smem_attr_once(s_attr_d, (const void*)k_mm_grid<double>, smem) != cudaSuccess)
        rc = mm_fail(m, XCB_ERR_CUDA, "mm_create: shared-memory opt-in failed");
    if (!rc && cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess)
        rc = mm_fail(m, XCB_ERR_CUDA, "mm_create: stream");
    if (!rc) rc = mm_alloc_scratch(m, max_kp, max_lm);
    if (rc) {
        mm_free_scratch(m);
        if (m->stream) cudaStreamDestroy(m->stream);
        delete m;
        return rc;
    }
    *out = m;
    return XCB_OK;
}

extern "C" int xcb_mm_destroy(xcb_mm* m)
{
    if (!m) return XCB_OK;
    cudaStreamSynchronize(m->stream);
    mm_free_scratch(m);
    cudaFreeHost(m->h_in);
    cudaFreeHost(m->h_out);
    cudaFree(m->d_in);
    cudaFree(m->d_out);
    cudaStreamDestroy(m->stream);
    delete m;
    return XCB_OK;
}

extern "C" const char* xcb_mm_last_error(xcb_mm* m) { return m ? m->err.c_str() : xcb_last_error(); }

extern "C" int xcb_mm_set_tuning(xcb_mm* m, int knob, int value)
{
    if (!m) return mm_fail(nullptr, XCB_ERR_ARG, "mm_set_tuning: null matcher");
    if (knob != XCB_TUNE_MM_LANES) return mm_fail(m, XCB_ERR_ARG, "mm_set_tuning: not a matcher knob");
    if (value == 0) value = MM_GROUP_DEFAULT;
    if (value != 1 && value != 2 && value != 4 && value != 8)
        return mm_fail(m, XCB_ERR_ARG, "mm_set_tuning: lanes per landmark must be 1, 2, 4 or 8");
    m->lanes = value;
    return XCB_OK;
}

extern "C" int xcb_mm_grid_dims(xcb_mm* m, int* gw, int* gh)
{
    if (!m || !gw || !gh) return mm_fail(m, XCB_ERR_ARG, "mm_grid_dims: null argument");
    *gw = m->gw;
    *gh = m->gh;
    return XCB_OK;
}

static int mm_launch(xcb_mm* m, MMArgs& a, int F, bool kp_f32, cudaStream_t st)
{
    a.gw = m->gw;
    a.gh = m->gh;
    a.ncell = m->ncell;
    a.ratio = 0.8;             // features.py RATIO
    a.ham_max = 104;           // features.py HAMMING_CHANCE
    a.cstart = m->d_cstart;
    a.slot = m->d_slot;
    a.ent = m->d_ent;
    a.claim = m->d_claim;
    a.kcnt = m->d_kcnt;
    a.kslot = m->d_kslot;
    const size_t smem = (size_t)(m->ncell + 1) * sizeof(int);
    const int grp = m->lanes, lpb = MM_WARPS * 32 / grp;
    const dim3 lg((a.lm_stride + lpb - 1) / lpb, F), lm((a.lm_stride + MM_WARPS * 32 - 1) / (MM_WARPS * 32), F);
#define MM_GATE(KT)                                                                                               \
    switch (grp) {                                                                                                \
        case 1: k_mm_gate<KT, 1><<<lg, MM_WARPS * 32, 0, st>>>(a); break;                                         \
        case 4: k_mm_gate<KT, 4><<<lg, MM_WARPS * 32, 0, st>>>(a); break;                                         \
        case 8: k_mm_gate<KT, 8><<<lg, MM_WARPS * 32, 0, st>>>(a); break;                                         \
        default: k_mm_gate<KT, 2><<<lg, MM_WARPS * 32, 0, st>>>(a); break;                                        \
    }
    if (kp_f32) {
        k_mm_grid<float><<<F, MM_GRID_T, smem, st>>>(a);
        if (a.lm_stride > 0) MM_GATE(float)
    } else {
        k_mm_grid<double><<<F, MM_GRID_T, smem, st>>>(a);
        if (a.lm_stride > 0) MM_GATE(double)
    }
#undef MM_GATE
    if (a.lm_stride > 0) k_mm_mutual<<<lm, MM_WARPS * 32, 0, st>>>(a);
    MCK(cudaGetLastError(), "mapmatch launch");
    return XCB_OK;
}

static size_t mm_al(size_t n) { return (n + 255) & ~(size_t)255; }

// scratch for N keypoints and L landmarks per frame (grown, never shrunk)
static int mm_reserve(xcb_mm* m, int N, int L)
{
    if (N <= m->cap_kp && L <= m->cap_lm) return XCB_OK;
    MCK(cudaStreamSynchronize(m->stream), "mapmatch: sync");
    return mm_alloc_scratch(m, std::max(N, m->cap_kp), std::max(L, m->cap_lm));
}

// page-locked staging blocks and their device twins for the host entries (grown, never shrunk); waits for `st`,
// whose previous call may still read them
static int mm_staging(xcb_mm* m, size_t in_bytes, size_t out_bytes, cudaStream_t st)
{
    MCK(cudaStreamSynchronize(st), "mapmatch: sync");
    if (in_bytes > m->in_cap) {
        MCK(cudaStreamSynchronize(m->stream), "mapmatch: sync");
        cudaFreeHost(m->h_in);
        cudaFree(m->d_in);
        m->h_in = m->d_in = nullptr;
        m->in_cap = 0;
        MCK(cudaMallocHost(&m->h_in, in_bytes * 2), "mapmatch: staging");
        MCK(cudaMalloc(&m->d_in, in_bytes * 2), "mapmatch: staging");
        m->in_cap = in_bytes * 2;
    }
    if (out_bytes > m->out_cap) {
        MCK(cudaStreamSynchronize(m->stream), "mapmatch: sync");
        cudaFreeHost(m->h_out);
        cudaFree(m->d_out);
        m->h_out = m->d_out = nullptr;
        m->out_cap = 0;
        MCK(cudaMallocHost(&m->h_out, out_bytes * 2), "mapmatch: staging");
        MCK(cudaMalloc(&m->d_out, out_bytes * 2), "mapmatch: staging");
        m->out_cap = out_bytes * 2;
    }
    return XCB_OK;
}

static int mm_check_match_args(xcb_mm* m, const double* kp, int N, const uint8_t* desc, const uint8_t* lm_desc, int D,
                               const int64_t* lm_ndesc, int L, int64_t* out_kp, int64_t* out_d, double* out_d2,
                               const char* who)
{
    if (N < 0 || L < 0 || D < 0) return mm_fail(m, XCB_ERR_ARG, std::string(who) + ": negative size");
    if (L > 0 && (!lm_ndesc || !out_kp || !out_d || !out_d2 || (D > 0 && !lm_desc)))
        return mm_fail(m, XCB_ERR_ARG, std::string(who) + ": null landmark argument");
    if (N > 0 && (!kp || !desc)) return mm_fail(m, XCB_ERR_ARG, std::string(who) + ": null keypoint argument");
    for (int l = 0; l < L; ++l)
        if (lm_ndesc[l] > D) return mm_fail(m, XCB_ERR_ARG, std::string(who) + ": lm_ndesc above the descriptor slots");
    for (int l = 0; l < L; ++l) {           // mapmatch.py:151-153 defaults; returned as they are when L or N is 0
        out_kp[l] = -1;
        out_d[l] = MM_NONE;
        out_d2[l] = INFINITY;
    }
    return XCB_OK;
}

extern "C" int xcb_mm_match_host(xcb_mm* m, const double* kp, int N, const uint8_t* desc, const double* uv,
                                 const double* S, const uint8_t* lm_desc, int D, const int64_t* lm_ndesc, int L,
                                 double chi2, int64_t* out_kp, int64_t* out_d, double* out_d2, void* stream)
{
    if (!m) return mm_fail(nullptr, XCB_ERR_ARG, "mm_match_host: null handle");
    if (L > 0 && (!uv || !S)) return mm_fail(m, XCB_ERR_ARG, "mm_match_host: null landmark argument");
    int rc = mm_check_match_args(m, kp, N, desc, lm_desc, D, lm_ndesc, L, out_kp, out_d, out_d2, "mm_match_host");
    if (rc || L == 0 || N == 0) return rc;
    if ((rc = mm_reserve(m, N, L))) return rc;
    const size_t o_desc = mm_al((size_t)N * 16), o_uv = o_desc + mm_al((size_t)N * 32), o_S = o_uv + mm_al((size_t)L * 16);
    const size_t o_lmd = o_S + mm_al((size_t)L * 32), o_lnd = o_lmd + mm_al((size_t)L * D * 32);
    const size_t in_bytes = o_lnd + mm_al((size_t)L * 8), out_bytes = (size_t)L * 24;
    cudaStream_t st = stream ? (cudaStream_t)stream : m->stream;
    if ((rc = mm_staging(m, in_bytes, out_bytes, st))) return rc;
    std::memcpy(m->h_in, kp, (size_t)N * 16);
    std::memcpy(m->h_in + o_desc, desc, (size_t)N * 32);
    std::memcpy(m->h_in + o_uv, uv, (size_t)L * 16);
    std::memcpy(m->h_in + o_S, S, (size_t)L * 32);
    if (D > 0) std::memcpy(m->h_in + o_lmd, lm_desc, (size_t)L * D * 32);
    std::memcpy(m->h_in + o_lnd, lm_ndesc, (size_t)L * 8);
    MCK(cudaMemcpyAsync(m->d_in, m->h_in, in_bytes, cudaMemcpyHostToDevice, st), "mm_match_host: H2D");
    MMArgs a = {};
    a.kp = m->d_in;
    a.nkp1 = N;
    a.kp_stride = N;
    a.desc = (const u8*)(m->d_in + o_desc);
    a.uv = (const double*)(m->d_in + o_uv);
    a.S = (const double*)(m->d_in + o_S);
    a.lmd = (const u8*)(m->d_in + o_lmd);
    a.lnd = (const i64*)(m->d_in + o_lnd);
    a.nlm1 = L;
    a.lm_stride = L;
    a.D = D;
    a.chi2 = chi2;
    a.out_kp = (i64*)m->d_out;
    a.out_d = (i64*)(m->d_out + (size_t)L * 8);
    a.out_d2 = (double*)(m->d_out + (size_t)L * 16);
    if ((rc = mm_launch(m, a, 1, false, st))) return rc;
    MCK(cudaMemcpyAsync(m->h_out, m->d_out, out_bytes, cudaMemcpyDeviceToHost, st), "mm_match_host: D2H");
    MCK(cudaStreamSynchronize(st), "mm_match_host: kernels");
    std::memcpy(out_kp, m->h_out, (size_t)L * 8);
    std::memcpy(out_d, m->h_out + (size_t)L * 8, (size_t)L * 8);
    std::memcpy(out_d2, m->h_out + (size_t)L * 16, (size_t)L * 8);
    return XCB_OK;
}

// ------------------------------------------------------------------------------------------------ gating prediction
// window.predict_projection (src/xclean/vio/window.py:1032-1144) on the device, one thread per landmark.  The file is
// built with --fmad=false, so every product and sum below is a separate IEEE round-to-nearest operation, evaluated
// left to right in the reference's order (numba contracts nothing either).
struct PredArgs {
    double Rwb[9], pwb[3], Rbc[9], pbc[3], Spose[36];   // predicted body pose, body-to-camera extrinsic, pose covariance
    const double* Rwc_h;      // [L][3][3] host camera rotations
    const double* pwc_h;      // [L][3] host camera centres
    const double* lmp;        // [L][3] (a, b, rho)
    const double* Sl;         // [L][3][3] landmark marginals
    double sig_px, fx, fy, cx, cy, W, H;
    int L;
    double* uv;               // [L][2] written where the point is in front, else NaN
    double* S;                // [L][2][2] written where it is also inside the image, else 0
    double* depth;            // [L] written where the point is in front, else 0
    u8* ok;                   // [L]
    u8* wr;                   // [L] 0: nothing written, 1: uv + depth, 2: uv + depth + S (the reference's writes)
    const i64* lnd_in;        // [L] descriptor counts, or NULL: no map matching follows
    i64* lnd_eff;             // [L] lnd_in where ok, else 0 (the landmarks the map matcher then sees)
};

__device__ __forceinline__ void pp_mm3(const double* A, const double* B, double* o)
{
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) o[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}

__global__ void __launch_bounds__(128) k_mm_predict(PredArgs a)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= a.L) return;
    double Rwc_t[9], pwc_t[3], Rcb[9], Px[9], Wt[9], Rct[9], RctWt[9];
    pp_mm3(a.Rwb, a.Rbc, Rwc_t);
#pragma unroll
    for (int i = 0; i < 3; ++i) pwc_t[i] = a.pwb[i] + a.Rwb[3 * i] * a.pbc[0] + a.Rwb[3 * i + 1] * a.pbc[1] + a.Rwb[3 * i + 2] * a.pbc[2];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            Rcb[3 * i + j] = a.Rbc[3 * j + i];
            Px[3 * i + j] = 0.0;
        }
    Px[1] = -a.pbc[2]; Px[2] = a.pbc[1]; Px[3] = a.pbc[2]; Px[5] = -a.pbc[0]; Px[6] = -a.pbc[1]; Px[7] = a.pbc[0];
    pp_mm3(a.Rwb, Px, Wt);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Rct[3 * i + j] = Rwc_t[3 * j + i];
    pp_mm3(Rct, Wt, RctWt);
    u8 wr = 0;
    double u = XCB_NAN, v = XCB_NAN, dep = 0.0, Sv[4] = {0.0, 0.0, 0.0, 0.0};
    const double* R = a.Rwc_h + 9 * (size_t)l;
    const double la = a.lmp[3 * l], lb = a.lmp[3 * l + 1], rho = a.lmp[3 * l + 2];
    const double d0 = a.pwc_h[3 * l] - pwc_t[0], d1 = a.pwc_h[3 * l + 1] - pwc_t[1], d2 = a.pwc_h[3 * l + 2] - pwc_t[2];
    const double Y0 = R[0] * la + R[1] * lb + R[2] + rho * d0;
    const double Y1 = R[3] * la + R[4] * lb + R[5] + rho * d1;
    const double Y2 = R[6] * la + R[7] * lb + R[8] + rho * d2;
    const double q0 = Rct[0] * Y0 + Rct[1] * Y1 + Rct[2] * Y2;
    const double q1 = Rct[3] * Y0 + Rct[4] * Y1 + Rct[5] * Y2;
    const double q2 = Rct[6] * Y0 + Rct[7] * Y1 + Rct[8] * Y2;
    if (!(q2 <= 1e-9 || rho <= 0.0)) {
        dep = q2 / rho;
        const double iq = 1.0 / q2;
        u = a.fx * q0 * iq + a.cx;
        v = a.fy * q1 * iq + a.cy;
        wr = 1;
        if (!(u < 0.0 || u >= a.W || v < 0.0 || v >= a.H)) {
            const double Dp[6] = {a.fx * iq, 0.0, -a.fx * q0 * iq * iq, 0.0, a.fy * iq, -a.fy * q1 * iq * iq};
            const double Qx[9] = {0.0, -q2, q1, q2, 0.0, -q0, -q1, q0, 0.0};
            double QR[9], Jp[12], Jl[6], RcR[9];
            pp_mm3(Qx, Rcb, QR);
#pragma unroll
            for (int r = 0; r < 2; ++r)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    Jp[6 * r + j] = Dp[3 * r] * (QR[j] + rho * RctWt[j]) + Dp[3 * r + 1] * (QR[3 + j] + rho * RctWt[3 + j])
                                    + Dp[3 * r + 2] * (QR[6 + j] + rho * RctWt[6 + j]);
                    Jp[6 * r + 3 + j] = -rho * (Dp[3 * r] * Rct[j] + Dp[3 * r + 1] * Rct[3 + j] + Dp[3 * r + 2] * Rct[6 + j]);
                }
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j)
                    RcR[3 * i + j] = Rct[3 * i] * R[j] + Rct[3 * i + 1] * R[3 + j] + Rct[3 * i + 2] * R[6 + j];
            const double e0 = Rct[0] * d0 + Rct[1] * d1 + Rct[2] * d2;
            const double e1 = Rct[3] * d0 + Rct[4] * d1 + Rct[5] * d2;
            const double e2 = Rct[6] * d0 + Rct[7] * d1 + Rct[8] * d2;
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                Jl[3 * r] = Dp[3 * r] * RcR[0] + Dp[3 * r + 1] * RcR[3] + Dp[3 * r + 2] * RcR[6];
                Jl[3 * r + 1] = Dp[3 * r] * RcR[1] + Dp[3 * r + 1] * RcR[4] + Dp[3 * r + 2] * RcR[7];
                Jl[3 * r + 2] = Dp[3 * r] * e0 + Dp[3 * r + 1] * e1 + Dp[3 * r + 2] * e2;
            }
            const double* sl = a.Sl + 9 * (size_t)l;
            double t6[12], t3[6];
#pragma unroll
            for (int r = 0; r < 2; ++r) {
#pragma unroll
                for (int j = 0; j < 6; ++j) {
                    double acc = 0.0;
#pragma unroll
                    for (int k = 0; k < 6; ++k) acc += Jp[6 * r + k] * a.Spose[6 * k + j];
                    t6[6 * r + j] = acc;
                }
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    double acc = 0.0;
#pragma unroll
                    for (int k = 0; k < 3; ++k) acc += Jl[3 * r + k] * sl[3 * k + j];
                    t3[3 * r + j] = acc;
                }
            }
#pragma unroll
            for (int r = 0; r < 2; ++r)
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    double acc = 0.0;
#pragma unroll
                    for (int k = 0; k < 6; ++k) acc += t6[6 * r + k] * Jp[6 * c + k];
#pragma unroll
                    for (int k = 0; k < 3; ++k) acc += t3[3 * r + k] * Jl[3 * c + k];
                    Sv[2 * r + c] = acc + (r == c ? a.sig_px * a.sig_px : 0.0);
                }
            wr = 2;
        }
    }
    a.uv[2 * l] = u;
    a.uv[2 * l + 1] = v;
#pragma unroll
    for (int i = 0; i < 4; ++i) a.S[4 * (size_t)l + i] = Sv[i];
    a.depth[l] = dep;
    a.ok[l] = wr == 2;
    a.wr[l] = wr;
    if (a.lnd_in) a.lnd_eff[l] = wr == 2 ? a.lnd_in[l] : 0;
}

// the reference's writes into the caller's arrays: ok everywhere, uv / depth / S only where it writes them
static void pp_scatter(int L, const char* ho, double* uv, double* S, uint8_t* ok, double* depth)
{
    const double* duv = (const double*)ho;
    const double* dS = (const double*)(ho + (size_t)L * 16);
    const double* ddep = (const double*)(ho + (size_t)L * 48);
    const u8* dok = (const u8*)(ho + (size_t)L * 56);
    const u8* dwr = dok + L;
    for (int l = 0; l < L; ++l) {
        ok[l] = dok[l];
        if (dwr[l] >= 1) {
            uv[2 * l] = duv[2 * l];
            uv[2 * l + 1] = duv[2 * l + 1];
            depth[l] = ddep[l];
        }
        if (dwr[l] == 2)
            for (int i = 0; i < 4; ++i) S[4 * (size_t)l + i] = dS[4 * (size_t)l + i];
    }
}

static int pp_setup(xcb_mm* m, PredArgs& p, const double* Rwb_t, const double* pwb_t, const double* Rbc,
                    const double* pbc, const double* Spose, double sig_px, double fx, double fy, double cx, double cy,
                    double W, double H, int L, const char* who)
{
    if (!Rwb_t || !pwb_t || !Rbc || !pbc || !Spose) return mm_fail(m, XCB_ERR_ARG, std::string(who) + ": null pose");
    if (L < 0) return mm_fail(m, XCB_ERR_ARG, std::string(who) + ": negative size");
    std::memcpy(p.Rwb, Rwb_t, sizeof(p.Rwb));
    std::memcpy(p.pwb, pwb_t, sizeof(p.pwb));
    std::memcpy(p.Rbc, Rbc, sizeof(p.Rbc));
    std::memcpy(p.pbc, pbc, sizeof(p.pbc));
    std::memcpy(p.Spose, Spose, sizeof(p.Spose));
    p.sig_px = sig_px;
    p.fx = fx;
    p.fy = fy;
    p.cx = cx;
    p.cy = cy;
    p.W = W;
    p.H = H;
    p.L = L;
    return XCB_OK;
}

// device layout of the prediction outputs (and the host copy): uv 16L, S 32L, depth 8L, ok L, wr L
static size_t pp_out_bytes(int L) { return mm_al((size_t)L * 58); }

static void pp_outputs(PredArgs& p, char* base, int L)
{
    p.uv = (double*)base;
    p.S = (double*)(base + (size_t)L * 16);
    p.depth = (double*)(base + (size_t)L * 48);
    p.ok = (u8*)(base + (size_t)L * 56);
    p.wr = p.ok + L;
}

extern "C" int xcb_mm_predict_host(xcb_mm* m, const double* Rwb_t, const double* pwb_t, const double* Rbc,
                                   const double* pbc, const double* Rwc_h, const double* pwc_h, const double* lmp,
                                   const double* Spose, const double* Sl, double sig_px, double fx, double fy,
                                   double cx, double cy, double W, double H, int L, double* uv, double* S, uint8_t* ok,
                                   double* depth, void* stream)
{
    if (!m) return mm_fail(nullptr, XCB_ERR_ARG, "mm_predict_host: null handle");
    PredArgs p = {};
    int rc = pp_setup(m, p, Rwb_t, pwb_t, Rbc, pbc, Spose, sig_px, fx, fy, cx, cy, W, H, L, "mm_predict_host");
    if (rc || L == 0) return rc;
    if (!Rwc_h || !pwc_h || !lmp || !Sl || !uv || !S || !ok || !depth)
        return mm_fail(m, XCB_ERR_ARG, "mm_predict_host: null landmark argument");
    const size_t o_p = mm_al((size_t)L * 72), o_l = o_p + mm_al((size_t)L * 24), o_s = o_l + mm_al((size_t)L * 24);
    const size_t in_bytes = o_s + mm_al((size_t)L * 72), out_bytes = pp_out_bytes(L);
    cudaStream_t st = stream ? (cudaStream_t)stream : m->stream;
    if ((rc = mm_staging(m, in_bytes, out_bytes, st))) return rc;
    std::memcpy(m->h_in, Rwc_h, (size_t)L * 72);
    std::memcpy(m->h_in + o_p, pwc_h, (size_t)L * 24);
    std::memcpy(m->h_in + o_l, lmp, (size_t)L * 24);
    std::memcpy(m->h_in + o_s, Sl, (size_t)L * 72);
    MCK(cudaMemcpyAsync(m->d_in, m->h_in, in_bytes, cudaMemcpyHostToDevice, st), "mm_predict_host: H2D");
    p.Rwc_h = (const double*)m->d_in;
    p.pwc_h = (const double*)(m->d_in + o_p);
    p.lmp = (const double*)(m->d_in + o_l);
    p.Sl = (const double*)(m->d_in + o_s);
    pp_outputs(p, m->d_out, L);
    k_mm_predict<<<(L + 127) / 128, 128, 0, st>>>(p);
    MCK(cudaGetLastError(), "mm_predict_host: launch");
    MCK(cudaMemcpyAsync(m->h_out, m->d_out, (size_t)L * 58, cudaMemcpyDeviceToHost, st), "mm_predict_host: D2H");
    MCK(cudaStreamSynchronize(st), "mm_predict_host: kernel");
    pp_scatter(L, m->h_out, uv, S, ok, depth);
    return XCB_OK;
}

extern "C" int xcb_mm_predict_match_host(xcb_mm* m, const double* Rwb_t, const double* pwb_t, const double* Rbc,
                                         const double* pbc, const double* Rwc_h, const double* pwc_h, const double* lmp,
                                         const double* Spose, const double* Sl, double sig_px, double fx, double fy,
                                         double cx, double cy, int L, const double* kp, int N, const uint8_t* desc,
                                         const uint8_t* lm_desc, int D, const int64_t* lm_ndesc, double chi2,
                                         double* uv, double* S, uint8_t* ok, double* depth, int64_t* out_kp,
                                         int64_t* out_d, double* out_d2, void* stream)
{
    if (!m) return mm_fail(nullptr, XCB_ERR_ARG, "mm_predict_match_host: null handle");
    PredArgs p = {};
    int rc = pp_setup(m, p, Rwb_t, pwb_t, Rbc, pbc, Spose, sig_px, fx, fy, cx, cy, (double)m->W, (double)m->H, L,
                      "mm_predict_match_host");
    if (rc) return rc;
    if (L > 0 && (!Rwc_h || !pwc_h || !lmp || !Sl || !uv || !S || !ok || !depth))
        return mm_fail(m, XCB_ERR_ARG, "mm_predict_match_host: null landmark argument");
    if ((rc = mm_check_match_args(m, kp, N, desc, lm_desc, D, lm_ndesc, L, out_kp, out_d, out_d2,
                                  "mm_predict_match_host")))
        return rc;
    if (L == 0) return XCB_OK;
    if ((rc = mm_reserve(m, N, L))) return rc;
    const size_t o_p = mm_al((size_t)L * 72), o_l = o_p + mm_al((size_t)L * 24), o_s = o_l + mm_al((size_t)L * 24);
    const size_t o_kp = o_s + mm_al((size_t)L * 72), o_desc = o_kp + mm_al((size_t)N * 16);
    const size_t o_lmd = o_desc + mm_al((size_t)N * 32), o_lnd = o_lmd + mm_al((size_t)L * D * 32);
    const size_t in_bytes = o_lnd + mm_al((size_t)L * 8);
    const size_t o_mo = pp_out_bytes(L), o_eff = o_mo + mm_al((size_t)L * 24), out_bytes = o_eff + mm_al((size_t)L * 8);
    cudaStream_t st = stream ? (cudaStream_t)stream : m->stream;
    if ((rc = mm_staging(m, in_bytes, out_bytes, st))) return rc;
    std::memcpy(m->h_in, Rwc_h, (size_t)L * 72);
    std::memcpy(m->h_in + o_p, pwc_h, (size_t)L * 24);
    std::memcpy(m->h_in + o_l, lmp, (size_t)L * 24);
    std::memcpy(m->h_in + o_s, Sl, (size_t)L * 72);
    if (N > 0) {
        std::memcpy(m->h_in + o_kp, kp, (size_t)N * 16);
        std::memcpy(m->h_in + o_desc, desc, (size_t)N * 32);
    }
    if (D > 0) std::memcpy(m->h_in + o_lmd, lm_desc, (size_t)L * D * 32);
    std::memcpy(m->h_in + o_lnd, lm_ndesc, (size_t)L * 8);
    MCK(cudaMemcpyAsync(m->d_in, m->h_in, in_bytes, cudaMemcpyHostToDevice, st), "mm_predict_match_host: H2D");
    p.Rwc_h = (const double*)m->d_in;
    p.pwc_h = (const double*)(m->d_in + o_p);
    p.lmp = (const double*)(m->d_in + o_l);
    p.Sl = (const double*)(m->d_in + o_s);
    p.lnd_in = (const i64*)(m->d_in + o_lnd);
    p.lnd_eff = (i64*)(m->d_out + o_eff);
    pp_outputs(p, m->d_out, L);
    k_mm_predict<<<(L + 127) / 128, 128, 0, st>>>(p);
    MCK(cudaGetLastError(), "mm_predict_match_host: launch");
    size_t d2h = o_mo;
    if (N > 0) {
        // the landmarks out of view carry no descriptors, so the gate skips them: the in-view ones are matched in
        // landmark order exactly as MapMatcher.match on the in-view subset matches them
        MMArgs a = {};
        a.kp = m->d_in + o_kp;
        a.nkp1 = N;
        a.kp_stride = N;
        a.desc = (const u8*)(m->d_in + o_desc);
        a.uv = p.uv;
        a.S = p.S;
        a.lmd = (const u8*)(m->d_in + o_lmd);
        a.lnd = p.lnd_eff;
        a.nlm1 = L;
        a.lm_stride = L;
        a.D = D;
        a.chi2 = chi2;
        a.out_kp = (i64*)(m->d_out + o_mo);
        a.out_d = a.out_kp + L;
        a.out_d2 = (double*)(a.out_d + L);
        if ((rc = mm_launch(m, a, 1, false, st))) return rc;
        d2h = o_mo + (size_t)L * 24;
    }
    MCK(cudaMemcpyAsync(m->h_out, m->d_out, d2h, cudaMemcpyDeviceToHost, st), "mm_predict_match_host: D2H");
    MCK(cudaStreamSynchronize(st), "mm_predict_match_host: kernels");
    pp_scatter(L, m->h_out, uv, S, ok, depth);
    if (N > 0) {
        std::memcpy(out_kp, m->h_out + o_mo, (size_t)L * 8);
        std::memcpy(out_d, m->h_out + o_mo + (size_t)L * 8, (size_t)L * 8);
        std::memcpy(out_d2, m->h_out + o_mo + (size_t)L * 16, (size_t)L * 8);
    }
    return XCB_OK;
}

extern "C" int xcb_mm_match_dev(xcb_mm* m, int F, const float* kp, const int32_t* nkp, int kp_stride,
                                const uint8_t* desc, const double* uv, const double* S, const uint8_t* lm_desc, int D,
                                const int64_t* lm_ndesc, const int32_t* nlm, int lm_stride, double chi2,
                                int64_t* out_kp, int64_t* out_d, double* out_d2, void* stream)
{
    if (!m) return mm_fail(nullptr, XCB_ERR_ARG, "mm_match_dev: null handle");
    if (F < 1 || kp_stride < 0 || lm_stride < 0 || D < 1) return mm_fail(m, XCB_ERR_ARG, "mm_match_dev: bad size");
    if (!kp || !nkp || !desc || !uv || !S || !lm_desc || !lm_ndesc || !nlm || !out_kp || !out_d || !out_d2)
        return mm_fail(m, XCB_ERR_ARG, "mm_match_dev: null argument");
    if (F > m->maxF || kp_stride > m->cap_kp || lm_stride > m->cap_lm)
        return mm_fail(m, XCB_ERR_CAPACITY, "mm_match_dev: more frames, keypoints or landmarks than the handle holds");
    MMArgs a = {};
    a.kp = kp;
    a.nkp = nkp;
    a.kp_stride = kp_stride;
    a.desc = desc;
    a.uv = uv;
    a.S = S;
    a.lmd = lm_desc;
    a.lnd = (const i64*)lm_ndesc;
    a.nlm = nlm;
    a.lm_stride = lm_stride;
    a.D = D;
    a.chi2 = chi2;
    a.out_kp = (i64*)out_kp;
    a.out_d = (i64*)out_d;
    a.out_d2 = out_d2;
    return mm_launch(m, a, F, true, stream ? (cudaStream_t)stream : m->stream);
}

extern "C" int xcb_mm_sync(xcb_mm* m, void* stream)
{
    if (!m) return mm_fail(nullptr, XCB_ERR_ARG, "mm_sync: null handle");
    MCK(cudaStreamSynchronize(stream ? (cudaStream_t)stream : m->stream), "mm_sync");
    return XCB_OK;
}
