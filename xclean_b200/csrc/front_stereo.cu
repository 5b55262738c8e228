// front_stereo.cu -- 1-D ZNCC epipolar stereo with the affine-LK sub-pixel step (sm_100a).
//
// Contract: front/stereo1d.stereo_points_band (src/xclean/front/stereo1d.py:335-472) bit for bit at HALF = 5 (the
// reference's patch, stereo/epipolar.py:35); the same arithmetic with HALF = 3 or 4 for the 7x7 / 9x9 windows.
// Every float64 sum whose rounding depends on order keeps the CPU's sequential order (the ZNCC cross term, the LK's
// ten sums); sums of integers (the u8 patch sums and sums of squares, exact in float64) are taken in any order.  The
// 3x3 solve / inverse replay OpenBLAS getf2 / getrs / trti2 + dgetri as numba's np.linalg.solve / inv run them on the
// reference's CPU (the reference's device form: gpu_front.py:607-922).
//
// B200 layout: ONE WARP PER POINT (the reference uses a 128-thread block and thread-0 serial sections).  The right
// image window of the point (all disparities, all band rows) is staged once in shared memory; each lane evaluates
// four disparities at a time, so four independent float64 dependency chains hide the DADD latency; argmax, second
// peak and left-right argmax are warp shuffles; the LK's ten sequential sums run on ten lanes that each resample the
// patch themselves (no shared-memory term table, no block barrier).  Points of many frames share one launch.
#include "common.cuh"
#include "front_kernels.h"

#define LK_ITERS 6
#define MAXD 128
#define ST_GROUP 32      // points per warp: searched one after another by the whole warp, then one LK per lane
#define BAND_MAX 16
#define LK_MG 4          // LK block columns: d within LK_MG of the integer peak (a sample beyond reads the image)

// warps per block: two blocks per SM at up to 128 registers (8 warps; 6 for the 11x11 window, whose LK blocks are
// larger)
static __host__ __device__ constexpr int st_warps(int half) { return half >= 5 ? 6 : 8; }

static __host__ __device__ __forceinline__ int win_w(int half) { return ((MAXD + 2 * half) + 3) & ~3; }

// LK block of one point: the right-image rows its samples can touch (PW + 2 rows from vi + js - HALF - 1) and the
// columns xr - HALF - LK_MG - 1 .. xr + HALF + LK_MG + 1 (u8 rows of lk_rs bytes), then the left image around the
// keypoint ((PW + 2) x (PW + 2) from row vi - HALF - 1, column ui - HALF - 1; rows of lk_ls bytes) for the template.
static __host__ __device__ __forceinline__ int lk_rw(int half) { return 2 * half + 1 + 2 * LK_MG + 2; }
static __host__ __device__ __forceinline__ int lk_rs(int half) { return (lk_rw(half) + 3) & ~3; }
static __host__ __device__ __forceinline__ int lk_ls(int half) { return (2 * half + 3 + 3) & ~3; }
static __host__ __device__ __forceinline__ int lk_job_bytes(int half)
{
    int words = ((2 * half + 3) * (lk_rs(half) + lk_ls(half)) + 3) / 4;
    if (!(words & 1)) ++words;       // odd word stride: lanes reading one offset of their own blocks hit distinct banks
    return 4 * words;
}

// a point that passed the searches, waiting for its LK
struct StJob {
    double u, v, seed, ts;
    long long oi;
    int ui, vi, xr, js, f, pad_;
};

// per-warp shared memory: jobs [ST_GROUP] | U.  U holds, while a point is searched: Td [NPIX] f64 | T2d [NPIX] f64 |
// sc [MAXD] f64 | jb [MAXD] i8 | the two templates' rows as words (PW x NTW each) | the exact-evaluation scratch |
// the image window | the exact evaluation's products (EXB x NPIX f64) (float32 rows of win_w, or u8 rows of U8Win::WWB); during the LKs:
// the group's LK blocks (ST_GROUP x lk_job_bytes); during the vertical scans: Td [NPIX] f64 | the scan block
// ((2 PW - 1) x PW float32).
static __host__ __device__ __forceinline__ size_t st_jobs_bytes() { return (ST_GROUP * sizeof(StJob) + 15) & ~(size_t)15; }

#define EXB 4          // patches evaluated exactly at once (their products staged in shared memory)
#define EZ 48          // exact-evaluation entries per pass (candidates x band rows)

// the search's exact-evaluation scratch: EZ entry offsets (i32), EZ results (f64), the candidate list (EZ i32), the
// exact flags of the disparities (MAXD u8)
static __host__ __device__ __forceinline__ size_t st_exact_bytes() { return (size_t)EZ * 16 + MAXD; }

static __host__ __device__ __forceinline__ size_t stereo_off_u(int half)
{
    int pw = 2 * half + 1, npix = pw * pw, ntw = (pw + 3) / 4;
    return ((size_t)npix * 16 + MAXD * 8 + MAXD + 2 * (size_t)pw * 4 * ntw + st_exact_bytes() + 15) & ~(size_t)15;
}

// the u8 window's row stride (U8Win<HALF>::WWB for a run-time half)
static __host__ __device__ __forceinline__ int u8_wwb(int half)
{
    const int pw = 2 * half + 1, nwd = (pw + 3 + 3) / 4, nsw = (pw + 3) / 4 + 1;
    return (MAXD + 4 * (nsw > nwd ? nsw : nwd) + 8 + 3) & ~3;
}

// per-warp shared memory of the search kernel: U (see below) with the window sized for its image type, then the
// exact evaluation's products
static __host__ __device__ __forceinline__ size_t st_win_bytes(int half, int band, bool flt)
{
    const int rows = 2 * half + 1 + 2 * band;
    const size_t b = flt ? (size_t)rows * win_w(half) * 4 : (size_t)rows * u8_wwb(half);
    return (b + 15) & ~(size_t)15;
}

static __host__ __device__ __forceinline__ size_t stereo_search_bytes(int half, int band, bool flt)
{
    const int pw = 2 * half + 1, npix = pw * pw;
    return (stereo_off_u(half) + st_win_bytes(half, band, flt) + (size_t)EXB * npix * 8 + 15) & ~(size_t)15;
}

// the vertical scan's staged block of a job (u8 images): the right image's 2 PW - 1 rows x PW columns around the
// match, then the template's PW x PW bytes; an odd word stride, so lanes reading their own jobs hit distinct banks
static __host__ __device__ __forceinline__ int st_vjob_bytes(int half)
{
    const int pw = 2 * half + 1;
    int words = ((2 * pw - 1) * pw + pw * pw + 3) / 4;
    if (!(words & 1)) ++words;
    return 4 * words;
}

// per-warp shared memory of the LK kernel: its jobs, then the LK blocks (later the vertical-scan blocks)
static __host__ __device__ __forceinline__ size_t stereo_lk_bytes(int half)
{
    const size_t lk = (size_t)ST_GROUP * lk_job_bytes(half), vs = (size_t)ST_GROUP * st_vjob_bytes(half);
    return (st_jobs_bytes() + (lk > vs ? lk : vs) + 15) & ~(size_t)15;
}

// the shared-memory opt-in limit of a block (227 KB); a launch whose warps would need more takes fewer warps
#define ST_SMEM_MAX ((size_t)227 * 1024)

// the dynamic shared memory the search kernel is enabled for: the widest band's block, at most the opt-in limit
static size_t st_smem_attr(int half, bool flt)
{
    const size_t pw = stereo_search_bytes(half, BAND_MAX, flt);
    size_t b = pw * st_warps(half);
    if (b > ST_SMEM_MAX) b = (ST_SMEM_MAX / pw) * pw;
    return b;
}

// ---------------------------------------------------------------- OpenBLAS 3x3 arithmetic (as the oracle restates it)
// Every loop has constant bounds and the pivot rows are applied by comparisons, so the matrix stays in registers (a
// pivot used as an index would put it in local memory); the arithmetic and its order are OpenBLAS getf2 / getrs /
// trti2 + getri's.
__device__ __forceinline__ void ob_getf2(double a[3][3], int piv[3])
{
#pragma unroll
    for (int j = 0; j < 3; ++j) {
#pragma unroll
        for (int i = 0; i < j; ++i)
#pragma unroll
            for (int r = i + 1; r < 3; ++r)
                if (piv[i] == r) { double t = a[i][j]; a[i][j] = a[r][j]; a[r][j] = t; }
#pragma unroll
        for (int i = 1; i < j; ++i) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < i; ++k) s = __fma_rn(a[i][k], a[k][j], s);
            a[i][j] = __dsub_rn(a[i][j], s);
        }
        if (j > 0)
#pragma unroll
            for (int i = j; i < 3; ++i) {
                double s = 0.0;
#pragma unroll
                for (int k = 0; k < j; ++k) s = __fma_rn(a[i][k], a[k][j], s);
                a[i][j] = __dsub_rn(a[i][j], s);
            }
        int jp = j;
        double mx = fabs(a[j][j]);
#pragma unroll
        for (int i = j + 1; i < 3; ++i)
            if (fabs(a[i][j]) > mx) { mx = fabs(a[i][j]); jp = i; }
        piv[j] = jp;
        double t = a[j][j];
#pragma unroll
        for (int r = j + 1; r < 3; ++r)
            if (jp == r) t = a[r][j];
        if (t != 0.0) {
            t = __ddiv_rn(1.0, t);
#pragma unroll
            for (int r = j + 1; r < 3; ++r)
                if (jp == r)
#pragma unroll
                    for (int k = 0; k <= j; ++k) { double u = a[j][k]; a[j][k] = a[r][k]; a[r][k] = u; }
#pragma unroll
            for (int i = j + 1; i < 3; ++i) a[i][j] = __dmul_rn(a[i][j], t);
        }
    }
}

__device__ __forceinline__ void ob_getrs(const double a[3][3], const int piv[3], double y[3])
{
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int r = j + 1; r < 3; ++r)
            if (piv[j] == r) { double t = y[j]; y[j] = y[r]; y[r] = t; }
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int i = j + 1; i < 3; ++i) y[i] = __fma_rn(-y[j], a[i][j], y[i]);
#pragma unroll
    for (int j = 2; j >= 0; --j) {
        y[j] = __ddiv_rn(y[j], a[j][j]);
#pragma unroll
        for (int i = 0; i < j; ++i) y[i] = __fma_rn(-y[j], a[i][j], y[i]);
    }
}

__device__ __forceinline__ void ob_getri(double a[3][3], const int piv[3])
{
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        double ajj = __ddiv_rn(1.0, a[j][j]);
        a[j][j] = ajj;
        double x[3];
#pragma unroll
        for (int i = 0; i < j; ++i) x[i] = a[i][j];
#pragma unroll
        for (int i = 0; i < j; ++i) {
#pragma unroll
            for (int q = 0; q < i; ++q) x[q] = __fma_rn(x[i], a[q][i], x[q]);
            x[i] = __dmul_rn(x[i], a[i][i]);
        }
#pragma unroll
        for (int i = 0; i < j; ++i) a[i][j] = __dmul_rn(x[i], -ajj);
    }
    double work[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int j = 2; j >= 0; --j) {
#pragma unroll
        for (int i = j + 1; i < 3; ++i) { work[i] = a[i][j]; a[i][j] = 0.0; }
        if (j < 2)
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                double s = 0.0;
#pragma unroll
                for (int k = j + 1; k < 3; ++k) s = __fma_rn(a[r][k], work[k], s);
                a[r][j] = __dsub_rn(a[r][j], s);
            }
    }
#pragma unroll
    for (int j = 1; j >= 0; --j)
#pragma unroll
        for (int c = j + 1; c < 3; ++c)
            if (piv[j] == c)
#pragma unroll
                for (int r = 0; r < 3; ++r) { double t = a[r][j]; a[r][j] = a[r][c]; a[r][c] = t; }
}

__global__ void k_lkcheck(const double* __restrict__ As, const double* __restrict__ gs, int n, double* __restrict__ X,
                          double* __restrict__ Inv)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double a[3][3], b[3][3];
    int piv[3], piv2[3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) a[i][j] = b[i][j] = As[9 * k + 3 * i + j];
    ob_getf2(a, piv);
    double y[3] = {gs[3 * k], gs[3 * k + 1], gs[3 * k + 2]};
    ob_getrs(a, piv, y);
    for (int i = 0; i < 3; ++i) X[3 * k + i] = y[i];
    ob_getf2(b, piv2);
    ob_getri(b, piv2);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Inv[9 * k + 3 * i + j] = b[i][j];
}

cudaError_t xcb_launch_lkcheck(const double* As, const double* gs, int n, double* X, double* Inv, cudaStream_t st)
{
    k_lkcheck<<<(n + 127) / 128, 128, 0, st>>>(As, gs, n, X, Inv);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- shift_rows (stereo1d.py:478-489), float32
__global__ void k_shift(const u8* __restrict__ R, int H, int W, double dy, float* __restrict__ Rs)
{
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y, f = blockIdx.z;
    if (x >= W) return;
    const u8* Rf = R + (size_t)f * H * W;
    double yy = __dadd_rn((double)y, dy);
    double y0d = floor(yy);
    float fr = __double2float_rn(__dsub_rn(yy, y0d));
    long long y0 = (long long)y0d;
    long long ya = y0 < 0 ? 0 : (y0 > H - 1 ? H - 1 : y0);
    long long yb = y0 + 1 < 0 ? 0 : (y0 + 1 > H - 1 ? H - 1 : y0 + 1);
    float a = (float)Rf[(size_t)ya * W + x], b = (float)Rf[(size_t)yb * W + x];
    Rs[(size_t)f * H * W + (size_t)y * W + x] = __fadd_rn(a, __fmul_rn(fr, __fsub_rn(b, a)));
}

cudaError_t xcb_launch_shift(const uint8_t* R, int F, int H, int W, double dy, float* Rs, cudaStream_t st)
{
    dim3 grid((W + 127) / 128, H, F);
    k_shift<<<grid, 128, 0, st>>>(R, H, W, dy, Rs);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- helpers
template <bool FLT>
struct RightImg {
    const u8* r8;
    const float* rf;
    __device__ __forceinline__ float at(size_t o) const { return FLT ? rf[o] : (float)r8[o]; }
};

// bilinear sample (stereo1d._bil) of float32-valued pixels: differences in float32 (exact for u8 data)
template <typename TP>
__device__ __forceinline__ void bil(const TP& img, int H, int W, double x, double y, double* val, double* gx)
{
    int x0 = (int)floor(x), y0 = (int)floor(y);
    double ax = __dsub_rn(x, (double)x0), ay = __dsub_rn(y, (double)y0);
    if (x0 < 0) x0 = 0;
    if (x0 > W - 2) x0 = W - 2;
    if (y0 < 0) y0 = 0;
    if (y0 > H - 2) y0 = H - 2;
    float fa = img.at((size_t)y0 * W + x0), fb = img.at((size_t)y0 * W + x0 + 1);
    float fc = img.at((size_t)(y0 + 1) * W + x0), fd = img.at((size_t)(y0 + 1) * W + x0 + 1);
    double a = (double)fa, c = (double)fc;
    double ba = (double)__fsub_rn(fb, fa), dc = (double)__fsub_rn(fd, fc);
    double top = __dadd_rn(a, __dmul_rn(ax, ba));
    double bot = __dadd_rn(c, __dmul_rn(ax, dc));
    *val = __dadd_rn(top, __dmul_rn(ay, __dsub_rn(bot, top)));
    *gx = __dadd_rn(__dmul_rn(ba, __dsub_rn(1.0, ay)), __dmul_rn(dc, ay));
}

struct LeftImg {
    const u8* p;
    __device__ __forceinline__ float at(size_t o) const { return (float)p[o]; }
};

__device__ __forceinline__ double zncc_finish(double s, double s2, double sx, double ts, int npix)
{
    double m = __ddiv_rn(s, (double)npix);
    double var = __dsub_rn(__ddiv_rn(s2, (double)npix), __dmul_rn(m, m));
    double sd = __dsqrt_rn(var > 0.0 ? var : 0.0);
    double den = __dmul_rn(__dmul_rn(ts, sd), (double)npix);
    return den > 1e-6 ? __ddiv_rn(sx, den) : -2.0;
}

// Q ZNCCs at once on a shared-memory window: patch q's top-left at (row0, col0[q]); T = template minus its mean.
// FLT: pixel sums in sequential float64 (shifted float32 image); else exact integer sums.
template <int HALF, bool FLT, int Q>
__device__ __forceinline__ void zncc_q(const float* win, int ww, int row0, const int* col0, const bool* valid,
                                       const double* T, double ts, double* out)
{
    constexpr int PW = 2 * HALF + 1, NPIX = PW * PW;
    double sx[Q], s[Q], s2[Q];
    int si[Q], s2i[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) { sx[q] = 0.0; s[q] = 0.0; s2[q] = 0.0; si[q] = 0; s2i[q] = 0; }
    int cb[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) cb[q] = valid[q] ? col0[q] : 0;
#pragma unroll 1
    for (int dy = 0; dy < PW; ++dy) {
        const float* row = win + (size_t)(row0 + dy) * ww;
#pragma unroll
        for (int dx = 0; dx < PW; ++dx) {
            const double tk = T[dy * PW + dx];
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const float v = row[cb[q] + dx];
                const double r = (double)v;
                if (FLT) {
                    s[q] = __dadd_rn(s[q], r);
                    s2[q] = __dadd_rn(s2[q], (double)__fmul_rn(v, v));
                } else {
                    const int iv = (int)v;
                    si[q] += iv;
                    s2i[q] += iv * iv;
                }
                sx[q] = __dadd_rn(sx[q], __dmul_rn(r, tk));
            }
        }
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        if (!FLT) { s[q] = (double)si[q]; s2[q] = (double)s2i[q]; }
        out[q] = valid[q] ? zncc_finish(s[q], s2[q], sx[q], ts, NPIX) : -2.0;
    }
}

// u8 image windows (the unshifted right image in the search, the left image in the left-right check): each lane scores
// four ADJACENT patches (top-left columns cb .. cb + 3), so one row of PW + 3 bytes, read as aligned 32-bit words,
// feeds 4 x PW products.  Pixel sums and sums of squares are exact integers (dp4a over whole words, then a sliding
// update per patch); the cross term keeps the CPU's sequential float64 order per patch.
template <int HALF>
struct U8Win {
    static constexpr int PW = 2 * HALF + 1;
    static constexpr int NV = PW + 3;                 // bytes a lane reads per row
    static constexpr int NWD = (NV + 3) / 4;          // ... as 32-bit words
    static constexpr int NTW = (PW + 3) / 4;          // a template row as zero-padded 32-bit words
    static constexpr int NSW = NTW + 1;               // window words a lane reads per row for the byte-shifted products
    static constexpr int PAD = 8;                     // left pad bytes: 4 + the alignment shift (0..3)
    static constexpr int WWB = (MAXD + 4 * (NSW > NWD ? NSW : NWD) + PAD + 3) & ~3;    // row stride in bytes
};

// z[k] = ZNCC of the patch whose top-left is byte `p` + k (rows WWB bytes apart); p is 4-byte aligned
template <int HALF>
__device__ __forceinline__ void zncc4_u8(const unsigned char* p, const double* T, double ts, double z[4])
{
    using G = U8Win<HALF>;
    constexpr int PW = G::PW, NPIX = PW * PW, NV = G::NV, NWD = G::NWD;
    double sx[4] = {0.0, 0.0, 0.0, 0.0};
    unsigned S[4] = {0u, 0u, 0u, 0u}, SQ[4] = {0u, 0u, 0u, 0u};
#pragma unroll 1
    for (int dy = 0; dy < PW; ++dy) {
        const unsigned* rp = (const unsigned*)(p + dy * G::WWB);
        unsigned w[NWD];
#pragma unroll
        for (int i = 0; i < NWD; ++i) w[i] = rp[i];
        unsigned b[NV];
#pragma unroll
        for (int i = 0; i < NV; ++i) b[i] = (w[i >> 2] >> (8 * (i & 3))) & 0xffu;
        unsigned s = 0u, sq = 0u;
#pragma unroll
        for (int i = 0; i < PW / 4; ++i) { s = __dp4a(w[i], 0x01010101u, s); sq = __dp4a(w[i], w[i], sq); }
#pragma unroll
        for (int i = (PW / 4) * 4; i < PW; ++i) { s += b[i]; sq += b[i] * b[i]; }
        S[0] += s; SQ[0] += sq;
#pragma unroll
        for (int k = 1; k < 4; ++k) {
            s += b[k - 1 + PW] - b[k - 1];
            sq += b[k - 1 + PW] * b[k - 1 + PW] - b[k - 1] * b[k - 1];
            S[k] += s; SQ[k] += sq;
        }
        double v[NV];
#pragma unroll
        for (int i = 0; i < NV; ++i) v[i] = (double)b[i];
        const double* Tr = T + dy * PW;
#pragma unroll
        for (int dx = 0; dx < PW; ++dx) {
            const double tk = Tr[dx];
#pragma unroll
            for (int k = 0; k < 4; ++k) sx[k] = __dadd_rn(sx[k], __dmul_rn(v[k + dx], tk));
        }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) z[k] = zncc_finish((double)S[k], (double)SQ[k], sx[k], ts, NPIX);
}

// The search filter (u8 images).  Every ZNCC the searches need is first bounded from exact integers: with the
// template bytes t, the patch bytes r, St = sum t, S = sum r, SQ = sum r^2, SI = sum r t (dp4a), N = NPIX SI - St S and
// V = NPIX SQ - S^2, the reference's float64 value is N / (NPIX ts sqrt(V)) up to its own roundings:
//   numerator   |sx - N / NPIX| <= E = gamma_NPIX 255 sum|T| + 510 u S  (the sequential sum of the rounded products,
//               and T = fl(t - fl(St / NPIX)) against t - St / NPIX), u = 2^-53
//   denominator the float64 variance's cancellation error is below 7e-7 relative for any V >= 1 (V is an integer)
// and the float32 evaluation (reciprocal square root, products) adds at most 4e-7 relative.  ea = 4e-6 |z| +
// 1.05 E / den + 1e-9 bounds |z_fp - za|.
// V = 0 (a flat patch) gives variance exactly 0 in float64 too, so z = -2 exactly (ea = 0); den within 1e-5 of the
// reference's 1e-6 cut is undecided (ea = inf).  A disparity whose interval lies strictly below another's cannot be
// the maximum (or the second peak, or the left-right maximum), so only the others are evaluated exactly, in the
// reference's sequential order (zexact_u8): the decisions and every value that leaves the search are bit for bit the
// reference's.
//
// za[k], ea[k] for the 4 adjacent patches whose top-left is byte p + k (p 4-byte aligned, rows WWB bytes apart);
// tw: the template's rows as NTW zero-padded words
template <int HALF>
__device__ __forceinline__ void zapprox4_u8(const unsigned char* p, const unsigned* tw, int st, float ts32, float at32,
                                            float za[4], float ea[4])
{
    using G = U8Win<HALF>;
    constexpr int PW = G::PW, NPIX = PW * PW, NV = G::NV, NTW = G::NTW, NSW = G::NSW;
    unsigned S[4] = {0u, 0u, 0u, 0u}, SQ[4] = {0u, 0u, 0u, 0u}, SI[4] = {0u, 0u, 0u, 0u};
#pragma unroll 1
    for (int dy = 0; dy < PW; ++dy) {
        const unsigned* rp = (const unsigned*)(p + dy * G::WWB);
        unsigned w[NSW];
#pragma unroll
        for (int i = 0; i < NSW; ++i) w[i] = rp[i];
        unsigned b[NV];
#pragma unroll
        for (int i = 0; i < NV; ++i) b[i] = (w[i >> 2] >> (8 * (i & 3))) & 0xffu;
        unsigned s = 0u, sq = 0u;
#pragma unroll
        for (int i = 0; i < PW / 4; ++i) { s = __dp4a(w[i], 0x01010101u, s); sq = __dp4a(w[i], w[i], sq); }
#pragma unroll
        for (int i = (PW / 4) * 4; i < PW; ++i) { s += b[i]; sq += b[i] * b[i]; }
        S[0] += s; SQ[0] += sq;
#pragma unroll
        for (int k = 1; k < 4; ++k) {
            s += b[k - 1 + PW] - b[k - 1];
            sq += b[k - 1 + PW] * b[k - 1 + PW] - b[k - 1] * b[k - 1];
            S[k] += s; SQ[k] += sq;
        }
        const unsigned* t = tw + dy * NTW;
#pragma unroll
        for (int i = 0; i < NTW; ++i) {
            const unsigned tt = t[i];
            SI[0] = __dp4a(w[i], tt, SI[0]);
            SI[1] = __dp4a(__byte_perm(w[i], w[i + 1], 0x4321), tt, SI[1]);
            SI[2] = __dp4a(__byte_perm(w[i], w[i + 1], 0x5432), tt, SI[2]);
            SI[3] = __dp4a(__byte_perm(w[i], w[i + 1], 0x6543), tt, SI[3]);
        }
    }
    const float c1 = 4.0f * 1.01f * (float)NPIX * 1.1102230246251565e-16f * 255.0f;
    const float c2 = 4.0f * 510.0f * 1.1102230246251565e-16f;
    // 1 / sqrt(V) by the hardware reciprocal square root (at most 2 ulp, 2.4e-7 relative) and multiplications by
    // 1 / ts: the approximation stays within 1e-6 relative of the exact quotient, inside the 4e-6 margin
    const float its = __fdividef(1.0f, ts32);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int N = NPIX * (int)SI[k] - st * (int)S[k];
        const int V = NPIX * (int)SQ[k] - (int)S[k] * (int)S[k];
        if (V <= 0) { za[k] = -2.0f; ea[k] = 0.0f; continue; }
        const float rs = rsqrtf((float)V);
        const float den = ts32 * ((float)V * rs);                   // ts sqrt(V): the reference's denominator
        if (den < 1e-6f * (1.0f - 1e-5f)) { za[k] = -2.0f; ea[k] = 0.0f; continue; }
        const float irden = rs * its;                               // 1 / den
        const float z = (float)N * irden * (1.0f / (float)NPIX);
        za[k] = z;
        ea[k] = den <= 1e-6f * (1.0f + 1e-5f) ? INFINITY
                                              : 4e-6f * fabsf(z) + 1.05f * (c1 * at32 + c2 * (float)S[k]) * irden + 1e-9f;
    }
}

// The reference's float64 ZNCC of n patches of a u8 window (entry i's top-left byte at winb + eoff[i], rows WWB bytes
// apart), EXB at a time: the whole warp forms the rounded products r x T into P, then lane i adds its patch's products in
// the reference's sequential order (with the exact integer sums) and finishes: zncc4_u8's arithmetic and order.  The
// lanes summing run the same instructions side by side.  Results in ez[i].
template <int HALF>
__device__ __noinline__ void zexact_list(const unsigned char* winb, const int* eoff, int n, const double* T, double ts,
                                         double* P, double* ez, int lane)
{
    using G = U8Win<HALF>;
    constexpr int PW = G::PW, NPIX = PW * PW;
    for (int b0 = 0; b0 < n; b0 += EXB) {
        const int m = n - b0 < EXB ? n - b0 : EXB;
        __syncwarp();
        for (int idx = lane; idx < m * NPIX; idx += 32) {
            const int e = idx / NPIX, k = idx - e * NPIX;
            const int r = winb[eoff[b0 + e] + (k / PW) * G::WWB + (k % PW)];
            P[e * NPIX + k] = __dmul_rn((double)r, T[k]);
        }
        __syncwarp();
        if (lane < m) {
            const unsigned char* pb = winb + eoff[b0 + lane];
            const double* Pe = P + lane * NPIX;
            double sx = 0.0;
            int S = 0, S2 = 0;
#pragma unroll 1
            for (int dy = 0; dy < PW; ++dy) {
#pragma unroll
                for (int dx = 0; dx < PW; ++dx) {
                    const int r = pb[dy * G::WWB + dx];
                    S += r;
                    S2 += r * r;
                    sx = __dadd_rn(sx, Pe[dy * PW + dx]);
                }
            }
            ez[b0 + lane] = zncc_finish((double)S, (double)S2, sx, ts, NPIX);
        }
    }
    __syncwarp();
}

__device__ __forceinline__ float warp_max_f(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ double warp_max_d(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// stage image rows r0 .. r0 + nrows - 1, columns c0 .. c0 + ncols - 1 of a u8 image into WWB-byte rows (column c at
// byte pad + c, zero bytes around it).  Each shared-memory word comes from two aligned 32-bit global words joined by a
// funnel shift, eight words per lane in flight.  The aligned words reach at most 6 bytes before column c0 and 7 bytes
// after the last column, i.e. into the rows just above and below the window: callers keep a row of the frame on either
// side of every window (and column c0 >= 2).
template <int HALF>
__device__ __forceinline__ void stage_u8(unsigned char* wb, const u8* __restrict__ img, int W, int r0, int nrows, int c0,
                                         int ncols, int pad, int lane)
{
    constexpr int NWW = U8Win<HALF>::WWB / 4;
    constexpr int UB = 8;
    unsigned* ws = (unsigned*)wb;
    const int total = nrows * NWW;
    for (int i0 = 0; i0 < total; i0 += 32 * UB) {
        unsigned lo[UB], hi[UB], msk[UB];
        int sh[UB];
#pragma unroll
        for (int u = 0; u < UB; ++u) {
            const int idx = i0 + 32 * u + lane;
            const int rr = idx / NWW, m = idx - rr * NWW;
            const int c = 4 * m - pad;                       // column of the word's first byte
            lo[u] = 0u; hi[u] = 0u; sh[u] = 0; msk[u] = 0u;
            if (idx < total && c + 3 >= 0 && c < ncols) {
                const size_t ga = (size_t)(img + (size_t)(r0 + rr) * W + c0) + (size_t)(ptrdiff_t)c;
                const unsigned* a4 = (const unsigned*)(ga & ~(size_t)3);
                sh[u] = (int)(ga & 3) * 8;
                lo[u] = __ldg(a4);
                hi[u] = __ldg(a4 + 1);
                msk[u] = (c >= 0 ? 0xffffffffu : (0xffffffffu << (8 * -c))) &
                         (c + 4 <= ncols ? 0xffffffffu : (0xffffffffu >> (8 * (c + 4 - ncols))));
            }
        }
#pragma unroll
        for (int u = 0; u < UB; ++u) {
            const int idx = i0 + 32 * u + lane;
            if (idx < total) ws[idx] = __funnelshift_r(lo[u], hi[u], sh[u]) & msk[u];
        }
    }
}

// warp argmax, first maximum in increasing index (strict '>' scan): ties keep the smaller index
__device__ __forceinline__ void warp_argmax(double& v, int& idx)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double v2 = __shfl_xor_sync(0xffffffffu, v, o);
        int i2 = __shfl_xor_sync(0xffffffffu, idx, o);
        if (v2 > v || (v2 == v && i2 < idx)) { v = v2; idx = i2; }
    }
}

// ---------------------------------------------------------------- the stereo kernel
// u8 -> float64 on the FP64 pipe: 2^52 + b carries b in its low mantissa bits, so the subtraction is exact
__device__ __forceinline__ double u8d(unsigned b)
{
    return __dsub_rn(__hiloint2double(0x43300000, (int)b), 4503599627370496.0);
}

// The search kernel: one warp per group of points (grp points, one after another).  The whole warp takes each point
// through the template statistics, the ZNCC search over the row band, the uniqueness test and the left-right check
// (lanes split the disparities); each point that passes is appended to the job list (gjobs, *gcount) for the LK kernel.
// Two blocks per SM of up to 128 registers (three blocks at 80 registers spilled and measured slower); the LK's registers
// and shared memory live in the other kernel.
#define ST_SEARCH_MINB 2
template <int HALF, bool FLT>
__global__ void __launch_bounds__(st_warps(HALF) * 32, ST_SEARCH_MINB) k_stereo_search(
    const u8* __restrict__ Lall, const u8* __restrict__ R8all, const float* __restrict__ Rsall, int H, int W,
    const double* __restrict__ kpd, const long long* __restrict__ dlo_a, const long long* __restrict__ dhi_a, int n,
    const float* __restrict__ kpf, const int* __restrict__ counts, int cap, int dlo_s, int dhi_s, int band,
    double* __restrict__ od, double* __restrict__ osig, u8* __restrict__ ook, double* __restrict__ ozn,
    double* __restrict__ ody, int grp, StJob* __restrict__ gjobs, int* __restrict__ gcount)
{
    constexpr int PW = 2 * HALF + 1, NPIX = PW * PW;
    const int NW = blockDim.x >> 5;                        // warps per block (at most st_warps(HALF))
    static_assert(U8Win<HALF>::WWB <= 4 * (((MAXD + 2 * HALF) + 3) & ~3), "u8 rows fit the float32 window rows");
    static_assert(sizeof(StJob) == 64, "job record");
    const double ZMIN = 0.5, UNIQ1 = 1.0 + 0.05, LRT = 1.0;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int ww = win_w(HALF);
    unsigned char* U = smem_raw + (size_t)wid * stereo_search_bytes(HALF, band, FLT);
    double* Td = (double*)U;
    double* T2d = Td + NPIX;
    double* sc = T2d + NPIX;
    signed char* jb = (signed char*)(sc + MAXD);
    float* win = (float*)(U + stereo_off_u(HALF));
    unsigned char* winb = U + stereo_off_u(HALF);          // the u8 windows (U8Win row stride)
    constexpr int KP = (NPIX + 31) / 32;                   // patch pixels per lane

    // ------------------------------------------------------------------------------------------- phase A: searches
    const long long g0 = ((long long)blockIdx.x * NW + wid) * grp;     // grp <= ST_GROUP points per warp
#pragma unroll 1
    for (int gi = 0; gi < grp; ++gi) {
        const long long p = g0 + gi;
        int f = 0;
        size_t oi;
        double u, v;
        long long lo, hi;
        if (kpd) {
            if (p >= n) break;
            oi = (size_t)p;
            u = kpd[2 * p]; v = kpd[2 * p + 1];
            lo = dlo_a[p]; hi = dhi_a[p];
        } else {
            f = (int)(p / cap);
            const int i = (int)(p % cap);
            if (f >= n) break;
            if (i >= counts[f]) continue;
            oi = (size_t)f * cap + i;
            u = (double)kpf[2 * oi]; v = (double)kpf[2 * oi + 1];
            lo = dlo_s; hi = dhi_s;
        }
        __syncwarp();                                      // the previous point's shared memory is free
        const u8* L = Lall + (size_t)f * H * W;
        RightImg<FLT> R;
        R.r8 = R8all ? R8all + (size_t)f * H * W : nullptr;
        R.rf = Rsall ? Rsall + (size_t)f * H * W : nullptr;
        if (lane == 0) { ook[oi] = 0; od[oi] = 0.0; osig[oi] = XCB_INF; ozn[oi] = -2.0; ody[oi] = XCB_NAN; }

        const int ui = (int)floor(__dadd_rn(u, 0.5)), vi = (int)floor(__dadd_rn(v, 0.5));
        if (ui - HALF - 2 < 0 || ui + HALF + 2 >= W || vi - HALF - 2 - band < 0 || vi + HALF + 2 + band >= H) continue;
        if (lo < 0) lo = 0;
        if (hi > MAXD - 1) hi = MAXD - 1;
        if (hi > ui - HALF - 2) hi = ui - HALF - 2;
        if (hi < lo) continue;

        // template statistics (_patch_stats on u8: integer sums, exact) and T - mean
        int tv[KP];
#pragma unroll
        for (int i = 0; i < KP; ++i) {
            const int k = lane + 32 * i;
            tv[i] = k < NPIX ? (int)L[(size_t)(vi + k / PW - HALF) * W + ui + k % PW - HALF] : 0;
        }
        // right-image window: rows vi-band-HALF .. vi+band+HALF, columns ui-hi-HALF .. ui-lo+HALF (window column =
        // hi - d); u8 images stage it now, its loads in flight with the template's
        const int wr0 = vi - band - HALF, wc0 = ui - (int)hi - HALF;
        const int nrows = PW + 2 * band, span = (int)(hi - lo), ncols = span + PW;
        const int pad = 4 + ((3 - span) & 3);
        if (!FLT) stage_u8<HALF>(winb, R.r8, W, wr0, nrows, wc0, ncols, pad, lane);
        int s = 0, s2 = 0;
#pragma unroll
        for (int i = 0; i < KP; ++i) { s += tv[i]; s2 += tv[i] * tv[i]; }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) { s += __shfl_xor_sync(0xffffffffu, s, o); s2 += __shfl_xor_sync(0xffffffffu, s2, o); }
        const double tm = __ddiv_rn((double)s, (double)NPIX);
        const double tvar = __dsub_rn(__ddiv_rn((double)s2, (double)NPIX), __dmul_rn(tm, tm));
        const double ts = __dsqrt_rn(tvar > 0.0 ? tvar : 0.0);
        if (ts <= 1e-6) continue;
#pragma unroll
        for (int i = 0; i < KP; ++i)
            if (lane + 32 * i < NPIX) Td[lane + 32 * i] = __dsub_rn((double)tv[i], tm);

        double bs, off = 0.0;
        int bestd, js, xr;
        if constexpr (FLT) {
            // shifted float32 right image: disparities lo + lane + 32 q, every ZNCC evaluated in the reference's order
            double lbest = -2.0;
            int lbd = -1;
            double best[4];
            int bj[4] = {0, 0, 0, 0}, dq[4], col[4];
            bool val[4];
            for (int idx = lane; idx < nrows * ncols; idx += 32) {
                int rr = idx / ncols, cc = idx % ncols;
                win[rr * ww + cc] = R.at((size_t)(wr0 + rr) * W + wc0 + cc);
            }
            __syncwarp();
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                dq[q] = (int)lo + lane + 32 * q;
                val[q] = dq[q] <= hi;
                col[q] = (int)hi - dq[q];
            }
            // rows in the CPU's order: vi, then vi - j, vi + j for j = 1..band; a later row wins only if strictly better
#pragma unroll 1
            for (int t = 0; t <= 2 * band; ++t) {
                const int j = t == 0 ? 0 : ((t & 1) ? -((t + 1) >> 1) : (t >> 1));
                double z[4];
                zncc_q<HALF, FLT, 4>(win, ww, band + j, col, val, Td, ts, z);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (t == 0 || z[q] > best[q]) { best[q] = z[q]; bj[q] = j; }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (val[q]) {
                    sc[dq[q]] = best[q];
                    jb[dq[q]] = (signed char)bj[q];
                    if (best[q] > lbest) { lbest = best[q]; lbd = dq[q]; }
                }
            }
            bs = lbest;
            bestd = lbd;
            warp_argmax(bs, bestd);
            if (lane == 0) ozn[oi] = bs;
            if (bestd < 0 || bs < ZMIN) continue;
            __syncwarp();
            double sec = -2.0;
            for (int d = (int)lo + lane; d <= hi; d += 32)
                if (abs(d - bestd) > 1 && sc[d] > sec) sec = sc[d];
            sec = warp_max_d(sec);
            if (!(__dsub_rn(1.0, sec) > __dmul_rn(__dsub_rn(1.0, bs), UNIQ1))) continue;

            // left-right check: the right patch at the peak searched back along the left row
            js = jb[bestd];
            xr = ui - bestd;
            float rv[KP];
#pragma unroll
            for (int i = 0; i < KP; ++i) {
                const int k = lane + 32 * i;
                rv[i] = k < NPIX ? R.at((size_t)(vi + js + k / PW - HALF) * W + xr + k % PW - HALF) : 0.f;
            }
            // float32 patch: the CPU's sequential float64 sums (x * x a float32 product)
            double a = 0.0, a2 = 0.0;
            if (lane == 0)
                for (int k = 0; k < NPIX; ++k) {
                    float x = R.at((size_t)(vi + js + k / PW - HALF) * W + xr + k % PW - HALF);
                    a = __dadd_rn(a, (double)x);
                    a2 = __dadd_rn(a2, (double)__fmul_rn(x, x));
                }
            a = __shfl_sync(0xffffffffu, a, 0);
            a2 = __shfl_sync(0xffffffffu, a2, 0);
            const double rm = __ddiv_rn(a, (double)NPIX);
            const double rvar = __dsub_rn(__ddiv_rn(a2, (double)NPIX), __dmul_rn(rm, rm));
            const double rsd = __dsqrt_rn(rvar > 0.0 ? rvar : 0.0);
            if (rsd <= 1e-6) continue;
#pragma unroll
            for (int i = 0; i < KP; ++i)
                if (lane + 32 * i < NPIX) T2d[lane + 32 * i] = __dsub_rn((double)rv[i], rm);
            int dmax = MAXD - 1;
            if (xr + dmax + HALF >= W) dmax = W - 1 - HALF - xr;
            const int lc0 = xr - HALF, lcols = dmax + PW;
            __syncwarp();
            // left-image window, candidate c at column c: lane scores c = 4 lane .. 4 lane + 3 (pad 4: word-aligned)
            stage_u8<HALF>(winb, L, W, vi - HALF, PW, lc0, lcols, 4, lane);
            __syncwarp();
            double lrb = -2.0;
            int lrd = -1;
            {
                double z[4];
                zncc4_u8<HALF>(winb + 4 + 4 * lane, T2d, rsd, z);
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (4 * lane + k <= dmax && z[k] > lrb) { lrb = z[k]; lrd = 4 * lane + k; }
            }
            warp_argmax(lrb, lrd);
            if (lrd < 0 || fabs((double)(lrd - bestd)) > LRT) continue;
        } else {
            // u8 right image, the search filter: lane's disparities lo + 4 lane + q (q = 0..3) are window columns
            // span - 4 lane - q, a block of four adjacent patches starting at column cb = span - 4 lane - 3.  The pad
            // makes every block start on a 32-bit word; a lane whose four disparities all exceed hi starts at the
            // lowest column >= -3 of the same residue mod 4 (pad bytes, results unused).
            using G = U8Win<HALF>;
            constexpr int RB = 4 * G::NTW;                       // template row bytes
            unsigned char* twb = (unsigned char*)(jb + MAXD);    // the search template's rows
            unsigned char* twb2 = twb + PW * RB;                 // the left-right template's rows
            int* eoff = (int*)(twb2 + PW * RB);                  // exact-evaluation entries
            double* ez = (double*)(eoff + EZ);                   // ... their values
            int* clist = (int*)(ez + EZ);                        // candidate disparities (or columns)
            unsigned char* exf = (unsigned char*)(clist + EZ);   // exact value known, per disparity
            double* P = (double*)(winb + st_win_bytes(HALF, band, FLT));   // products, after the window
            const int NR = 2 * band + 1;                         // band rows per disparity
            double at = 0.0;
#pragma unroll
            for (int i = 0; i < KP; ++i) {
                const int k = lane + 32 * i;
                if (k < NPIX) {
                    twb[(k / PW) * RB + k % PW] = (unsigned char)tv[i];
                    at = __dadd_rn(at, fabs(__dsub_rn((double)tv[i], tm)));
                }
            }
            for (int k = lane; k < PW * RB; k += 32)
                if (k % RB >= PW) twb[k] = 0;
            for (int k = lane; k < MAXD; k += 32) exf[k] = 0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) at = __dadd_rn(at, __shfl_xor_sync(0xffffffffu, at, o));
            __syncwarp();                                        // the window and the template rows
            int cb = span - 4 * lane - 3;
            if (cb < -3) cb += (-cb) & ~3;
            const unsigned char* pb = winb + pad + cb;
            int dq[4];
            bool val[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                dq[q] = (int)lo + 4 * lane + q;
                val[q] = dq[q] <= hi;
            }
            // bounds of every disparity's best row
            float za[4], ea[4];
            const float ts32 = (float)ts, at32 = (float)at;
#pragma unroll 1
            for (int t = 0; t < NR; ++t) {
                const int j = t == 0 ? 0 : ((t & 1) ? -((t + 1) >> 1) : (t >> 1));
                float z4[4], e4[4];
                zapprox4_u8<HALF>(pb + (band + j) * G::WWB, (const unsigned*)twb, s, ts32, at32, z4, e4);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    za[q] = t == 0 ? z4[3 - q] : fmaxf(za[q], z4[3 - q]);
                    ea[q] = t == 0 ? e4[3 - q] : fmaxf(ea[q], e4[3 - q]);
                }
            }
            // exact values of the flagged disparities: a disparity certainly -2 (flat patch or a denominator certainly
            // under the reference's cut in every row) is recorded directly; the others are listed, every band row of
            // each evaluated, and the best row taken in the reference's row order (a later row only if strictly better)
            auto exact_flagged = [&](const bool* want) {
                int nc = 0;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const bool cert = want[q] && !(ea[q] > 0.0f);
                    if (cert) { sc[dq[q]] = -2.0; jb[dq[q]] = 0; exf[dq[q]] = 1; }
                    const bool lst = want[q] && ea[q] > 0.0f;
                    const unsigned m = __ballot_sync(0xffffffffu, lst);
                    if (lst) {
                        const int pos = nc + __popc(m & ((1u << lane) - 1u));
                        if (pos < 32 * 4) clist[pos % EZ] = dq[q];    // (overflow handled below)
                    }
                    nc += __popc(m);
                }
                __syncwarp();
                if (nc > EZ) {
                    // more candidates than one list holds (a patch nearly flat everywhere): take them in passes
                    // straight from the flags, one disparity at a time
                    for (int d = (int)lo; d <= hi; ++d) {
                        bool w = false;
#pragma unroll
                        for (int q = 0; q < 4; ++q) w |= (dq[q] == d) && want[q] && ea[q] > 0.0f;
                        if (!__any_sync(0xffffffffu, w)) continue;
                        for (int t = lane; t < NR; t += 32) {
                            const int j = t == 0 ? 0 : ((t & 1) ? -((t + 1) >> 1) : (t >> 1));
                            eoff[t] = pad + ((int)hi - d) + (band + j) * G::WWB;
                        }
                        zexact_list<HALF>(winb, eoff, NR, Td, ts, P, ez, lane);
                        if (lane == 0) {
                            double bz = -2.0;
                            int bjr = 0;
                            for (int t = 0; t < NR; ++t)
                                if (t == 0 || ez[t] > bz) { bz = ez[t]; bjr = t == 0 ? 0 : ((t & 1) ? -((t + 1) >> 1) : (t >> 1)); }
                            sc[d] = bz; jb[d] = (signed char)bjr; exf[d] = 1;
                        }
                        __syncwarp();
                    }
                    return;
                }
                const int per = EZ / NR;                         // candidates per pass
                for (int c0 = 0; c0 < nc; c0 += per) {
                    const int m = nc - c0 < per ? nc - c0 : per;
                    for (int i = lane; i < m * NR; i += 32) {
                        const int c = i / NR, t = i - c * NR;
                        const int j = t == 0 ? 0 : ((t & 1) ? -((t + 1) >> 1) : (t >> 1));
                        eoff[i] = pad + ((int)hi - clist[c0 + c]) + (band + j) * G::WWB;
                    }
                    zexact_list<HALF>(winb, eoff, m * NR, Td, ts, P, ez, lane);
                    if (lane < m) {
                        double bz = -2.0;
                        int bjr = 0;
                        for (int t = 0; t < NR; ++t)
                            if (t == 0 || ez[lane * NR + t] > bz) {
                                bz = ez[lane * NR + t];
                                bjr = t == 0 ? 0 : ((t & 1) ? -((t + 1) >> 1) : (t >> 1));
                            }
                        const int d = clist[c0 + lane];
                        sc[d] = bz; jb[d] = (signed char)bjr; exf[d] = 1;
                    }
                    __syncwarp();
                }
            };
            // round A: the candidates for the maximum, the approximate peak's neighbours, the candidates for the second
            // peak away from it
            float lbq = -INFINITY, am = -INFINITY;
            int ad = 0x7fffffff;
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (val[q]) {
                    lbq = fmaxf(lbq, za[q] - ea[q]);
                    if (za[q] > am) { am = za[q]; ad = dq[q]; }
                }
            const float lb = warp_max_f(lbq);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const float a2 = __shfl_xor_sync(0xffffffffu, am, o);
                const int d2 = __shfl_xor_sync(0xffffffffu, ad, o);
                if (a2 > am || (a2 == am && d2 < ad)) { am = a2; ad = d2; }
            }
            float l2q = -INFINITY;
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (val[q] && abs(dq[q] - ad) > 1) l2q = fmaxf(l2q, za[q] - ea[q]);
            const float lb2 = warp_max_f(l2q);
            // round A, then (only when the exact peak is not the approximate one) round B: the second-peak candidates
            // and neighbours around the exact peak; one call site for both rounds
            bool want[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int dd = abs(dq[q] - ad);
                want[q] = val[q] && (za[q] + ea[q] >= lb || dd == 1 || (dd > 1 && za[q] + ea[q] >= lb2));
            }
            bool dead = false;
#pragma unroll 1
            for (int round = 0; round < 2; ++round) {
                exact_flagged(want);
                if (round == 1) break;
                double lbest = -2.0;
                int lbd = -1;
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (val[q] && exf[dq[q]] && sc[dq[q]] > lbest) { lbest = sc[dq[q]]; lbd = dq[q]; }
                bs = lbest;
                bestd = lbd;
                warp_argmax(bs, bestd);
                if (lane == 0) ozn[oi] = bs;
                if (bestd < 0 || bs < ZMIN) { dead = true; break; }
                if (bestd == ad) break;
                double l2d = -INFINITY;
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (val[q] && abs(dq[q] - bestd) > 1)
                        l2d = fmax(l2d, exf[dq[q]] ? sc[dq[q]] : (double)za[q] - (double)ea[q]);
                l2d = warp_max_d(l2d);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int dd = abs(dq[q] - bestd);
                    want[q] = val[q] && !exf[dq[q]] && (dd == 1 || (dd > 1 && (double)za[q] + (double)ea[q] >= l2d));
                }
            }
            if (dead) continue;
            double sec = -2.0;
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (val[q] && exf[dq[q]] && abs(dq[q] - bestd) > 1 && sc[dq[q]] > sec) sec = sc[dq[q]];
            sec = warp_max_d(sec);
            __syncwarp();
            if (!(__dsub_rn(1.0, sec) > __dmul_rn(__dsub_rn(1.0, bs), UNIQ1))) continue;

            // left-right check: the right patch at the peak searched back along the left row, through the same filter
            js = jb[bestd];
            xr = ui - bestd;
            int rvi[KP];
#pragma unroll
            for (int i = 0; i < KP; ++i) {
                const int k = lane + 32 * i;
                rvi[i] = k < NPIX ? (int)R.r8[(size_t)(vi + js + k / PW - HALF) * W + xr + k % PW - HALF] : 0;
            }
            // the left-image window, its loads in flight with the patch's (the right window is no longer read):
            // candidate c at column c, lane bounds c = 4 lane .. 4 lane + 3 (pad 4: word-aligned)
            int dmax = MAXD - 1;
            if (xr + dmax + HALF >= W) dmax = W - 1 - HALF - xr;
            const int lc0 = xr - HALF, lcols = dmax + PW;
            stage_u8<HALF>(winb, L, W, vi - HALF, PW, lc0, lcols, 4, lane);
            int a = 0, a2 = 0;
#pragma unroll
            for (int i = 0; i < KP; ++i) { a += rvi[i]; a2 += rvi[i] * rvi[i]; }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) { a += __shfl_xor_sync(0xffffffffu, a, o); a2 += __shfl_xor_sync(0xffffffffu, a2, o); }
            const double rm = __ddiv_rn((double)a, (double)NPIX);
            const double rvar = __dsub_rn(__ddiv_rn((double)a2, (double)NPIX), __dmul_rn(rm, rm));
            const double rsd = __dsqrt_rn(rvar > 0.0 ? rvar : 0.0);
            if (rsd <= 1e-6) continue;
            double at2 = 0.0;
#pragma unroll
            for (int i = 0; i < KP; ++i) {
                const int k = lane + 32 * i;
                if (k < NPIX) {
                    const double tk = __dsub_rn((double)rvi[i], rm);
                    T2d[k] = tk;
                    at2 = __dadd_rn(at2, fabs(tk));
                    twb2[(k / PW) * RB + k % PW] = (unsigned char)rvi[i];
                }
            }
            for (int k = lane; k < PW * RB; k += 32)
                if (k % RB >= PW) twb2[k] = 0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) at2 = __dadd_rn(at2, __shfl_xor_sync(0xffffffffu, at2, o));
            __syncwarp();                                        // the left window and the template rows
            float z4[4], e4[4];
            zapprox4_u8<HALF>(winb + 4 + 4 * lane, (const unsigned*)twb2, a, (float)rsd, (float)at2, z4, e4);
            float lq = -INFINITY;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (4 * lane + k <= dmax) lq = fmaxf(lq, z4[k] - e4[k]);
            const float llb = warp_max_f(lq);
            // Only the exact maximum's distance from the peak matters, and the maximum is one of the candidates (or
            // none exceeds -2).  Every candidate within LRT of the peak with a lower bound above -2: the check passes;
            // none within LRT: it fails; otherwise the candidates are evaluated exactly.
            bool cin = false, cout = false;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int c = 4 * lane + k;
                if (c <= dmax && z4[k] + e4[k] >= llb) {
                    if (fabs((double)(c - bestd)) > LRT) cout = true;
                    else cin = true;
                }
            }
            cin = __any_sync(0xffffffffu, cin);
            cout = __any_sync(0xffffffffu, cout);
            if (!cin) continue;
            if (cout || !(llb > -2.0f)) {
            // the candidates (a column certainly at -2 can never be the maximum, which must exceed -2)
            int nc = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const bool lst = 4 * lane + k <= dmax && z4[k] + e4[k] >= llb && e4[k] > 0.0f;
                const unsigned m = __ballot_sync(0xffffffffu, lst);
                if (lst) {
                    const int pos = nc + __popc(m & ((1u << lane) - 1u));
                    if (pos < EZ) { clist[pos] = 4 * lane + k; eoff[pos] = 4 + 4 * lane + k; }
                }
                nc += __popc(m);
            }
            double lrb = -2.0;
            int lrd = -1;
            for (int c0 = 0; c0 < nc; c0 += EZ) {
                const int m = nc - c0 < EZ ? nc - c0 : EZ;
                if (c0 > 0) {
                    // a further pass (more than EZ candidates): list them again from the bounds
                    int pos = 0;
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const bool lst = 4 * lane + k <= dmax && z4[k] + e4[k] >= llb && e4[k] > 0.0f;
                        const unsigned mk = __ballot_sync(0xffffffffu, lst);
                        if (lst) {
                            const int p2 = pos + __popc(mk & ((1u << lane) - 1u)) - c0;
                            if (p2 >= 0 && p2 < EZ) { clist[p2] = 4 * lane + k; eoff[p2] = 4 + 4 * lane + k; }
                        }
                        pos += __popc(mk);
                    }
                }
                __syncwarp();
                zexact_list<HALF>(winb, eoff, m, T2d, rsd, P, ez, lane);
                for (int i = lane; i < m; i += 32) {
                    const double z = ez[i];
                    const int c = clist[i];
                    if (z > lrb || (z == lrb && lrd >= 0 && c < lrd)) { lrb = z; lrd = c; }
                }
                __syncwarp();
            }
            warp_argmax(lrb, lrd);
            if (lrd < 0 || fabs((double)(lrd - bestd)) > LRT) continue;
            }
        }

        // parabola seed of the LK (from the sub-pixel keypoint position)
        if (bestd > lo && bestd < hi) {
            double y0 = sc[bestd - 1], y2 = sc[bestd + 1];
            double den = __dadd_rn(__dsub_rn(y0, __dmul_rn(2.0, bs)), y2);
            if (den < -1e-9) {
                off = __ddiv_rn(__dmul_rn(0.5, __dsub_rn(y0, y2)), den);
                if (off > 0.5) off = 0.5;
                if (off < -0.5) off = -0.5;
            }
        }
        if (lane == 0) {
            StJob J;
            J.u = u; J.v = v; J.ts = ts;
            J.seed = __dadd_rn(__dadd_rn((double)bestd, off), __dsub_rn(u, (double)ui));
            J.oi = (long long)oi;
            J.ui = ui; J.vi = vi; J.xr = xr; J.js = js; J.f = f; J.pad_ = 0;
            gjobs[atomicAdd(gcount, 1)] = J;
        }
    }
}

// The LK kernel: jpw jobs of the list per warp (up to 32).  The warp stages every job's right- and left-image
// neighbourhood, then each lane runs one job's affine LK (LK_ITERS steps and the covariance pass) with its ten sums in
// the CPU's sequential order and its own 3x3 OpenBLAS solve: the serial float64 chains of the jobs run side by side.
// Then each lane takes its accepted job through the vertical scan.  Outputs are written by point index, so the list's
// order (atomic appends) does not matter.
template <int HALF, bool FLT>
__global__ void __launch_bounds__(st_warps(HALF) * 32, 2) k_stereo_lk(
    const u8* __restrict__ Lall, const u8* __restrict__ R8all, const float* __restrict__ Rsall, int H, int W,
    const StJob* __restrict__ gjobs, const int* __restrict__ gcount, int jpw, double* __restrict__ od,
    double* __restrict__ osig, u8* __restrict__ ook, double* __restrict__ ody)
{
    constexpr int PW = 2 * HALF + 1, NPIX = PW * PW;
    const int NW = blockDim.x >> 5;
    constexpr int LKR = PW + 2, LKW = PW + 2 * LK_MG + 2;
    const int RS = lk_rs(HALF), LS = lk_ls(HALF), JB = lk_job_bytes(HALF);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned char* base = smem_raw + (size_t)wid * stereo_lk_bytes(HALF);
    StJob* jobs = (StJob*)base;
    unsigned char* U = base + st_jobs_bytes();
    const long long j0 = ((long long)blockIdx.x * NW + wid) * jpw;
    const int total = *gcount;
    if (j0 >= total) return;
    const int njobs = (int)(total - j0 < jpw ? total - j0 : jpw);
    if (lane < njobs) jobs[lane] = gjobs[j0 + lane];

    // ----------------------------------------------------------------------------------------------- phase B: LKs
    __syncwarp();
    // every job's blocks (right image, then left image), staged by the whole warp over all jobs at once with eight
    // loads in flight per lane
    {
        const int RB = LKR * RS, PJ = RB + LKR * LS;           // bytes per job
        constexpr int UB = 8;
        const int total = njobs * PJ;
        for (int t0 = lane; t0 < total; t0 += 32 * UB) {
            u8 v[UB];
#pragma unroll
            for (int u = 0; u < UB; ++u) {
                const int t = t0 + 32 * u;
                v[u] = 0;
                if (t < total) {
                    const int j = t / PJ, q = t - j * PJ;
                    const StJob& J = jobs[j];
                    const size_t fo = (size_t)J.f * H * W;
                    if (q < RB) {
                        if (!FLT) {
                            const int rr = q / RS, cc = q - rr * RS, col = J.xr - HALF - LK_MG - 1 + cc;
                            if (cc < LKW && col >= 0 && col < W)
                                v[u] = R8all[fo + (size_t)(J.vi + J.js - HALF - 1 + rr) * W + col];
                        }
                    } else {
                        const int q2 = q - RB, rr = q2 / LS, cc = q2 - rr * LS;
                        if (cc < PW + 2) v[u] = Lall[fo + (size_t)(J.vi - HALF - 1 + rr) * W + J.ui - HALF - 1 + cc];
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < UB; ++u) {
                const int t = t0 + 32 * u;
                if (t < total) {
                    const int j = t / PJ, q = t - j * PJ;
                    U[(size_t)j * JB + q] = v[u];
                }
            }
        }
    }
    __syncwarp();
    bool okl = false;
    if (lane < njobs) {
        const StJob J = jobs[lane];
        const unsigned char* rb = U + (size_t)lane * JB;
        const unsigned char* lb = rb + LKR * RS;
        RightImg<FLT> R;
        R.r8 = R8all ? R8all + (size_t)J.f * H * W : nullptr;
        R.rf = Rsall ? Rsall + (size_t)J.f * H * W : nullptr;
        const int ys0 = J.vi + J.js - HALF - 1, xs0 = J.xr - HALF - LK_MG - 1;
        const int xa = xs0 > 0 ? xs0 : 0, xb = xs0 + LKW - 1 < W - 1 ? xs0 + LKW - 1 : W - 1;
        const int ly0 = J.vi - HALF - 1, lx0 = J.ui - HALF - 1;
        const double u = J.u, v = J.v, voff = (double)J.js, seed = J.seed;
        double d = seed, a = 1.0, b = 0.0, sig = 0.0;
#pragma unroll 1
        for (int it = 0; it <= LK_ITERS; ++it) {
            double S[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) S[q] = 0.0;
#pragma unroll 1
            for (int dy = 0; dy < PW; ++dy) {
                const double py = __dadd_rn(v, (double)(dy - HALF));
                // the right samples' row: y = v + dy - HALF + js, its floor and fraction, for every pixel of the row
                const double y = __dadd_rn(py, voff);
                int y0 = (int)floor(y);
                const double ay = __dsub_rn(y, (double)y0);
                if (y0 < 0) y0 = 0;
                if (y0 > H - 2) y0 = H - 2;
                const double omay = __dsub_rn(1.0, ay);
                const bool rin = y0 >= ys0 && y0 + 1 < ys0 + LKR;
                // the template's row (the keypoint's neighbourhood keeps every sample off the image border: no clamp)
                const int ty0 = (int)floor(py);
                const double tay = __dsub_rn(py, (double)ty0);
                int tr = ty0 - ly0;
                tr = tr < 0 ? 0 : (tr > PW ? PW : tr);
                const unsigned char* lrow = lb + tr * LS;
                // three pixels per unrolled step: a full unroll of the row spills at the 128-register budget
#pragma unroll 3
                for (int dx = 0; dx < PW; ++dx) {
                    const double px = __dadd_rn(u, (double)(dx - HALF));
                    // template sample: bilinear left at (px, py) (stereo1d._bil); u8 differences are exact
                    const int tx0 = (int)floor(px);
                    const double tax = __dsub_rn(px, (double)tx0);
                    int tc = tx0 - lx0;
                    tc = tc < 0 ? 0 : (tc > PW ? PW : tc);
                    const unsigned char* lp = lrow + tc;
                    const double tfa = u8d(lp[0]), tfb = u8d(lp[1]), tfc = u8d(lp[LS]), tfd = u8d(lp[LS + 1]);
                    const double tba = __dsub_rn(tfb, tfa), tdc = __dsub_rn(tfd, tfc);
                    const double ttop = __dadd_rn(tfa, __dmul_rn(tax, tba));
                    const double tbot = __dadd_rn(tfc, __dmul_rn(tax, tdc));
                    const double Tl = __dadd_rn(ttop, __dmul_rn(tay, __dsub_rn(tbot, ttop)));
                    // right sample at (px - d, y)
                    double rv, rg;
                    if (FLT) {
                        bil(R, H, W, __dsub_rn(px, d), y, &rv, &rg);
                    } else {
                        const double x = __dsub_rn(px, d);
                        int x0 = (int)floor(x);
                        const double ax = __dsub_rn(x, (double)x0);
                        if (x0 < 0) x0 = 0;
                        if (x0 > W - 2) x0 = W - 2;
                        double fa, fb, fc, fd;
                        if (rin && x0 >= xa && x0 + 1 <= xb) {
                            const unsigned char* sp = rb + (y0 - ys0) * RS + (x0 - xs0);
                            fa = u8d(sp[0]); fb = u8d(sp[1]); fc = u8d(sp[RS]); fd = u8d(sp[RS + 1]);
                        } else {
                            const u8* gp = R.r8 + (size_t)y0 * W + x0;
                            fa = u8d(gp[0]); fb = u8d(gp[1]); fc = u8d(gp[W]); fd = u8d(gp[W + 1]);
                        }
                        const double ba = __dsub_rn(fb, fa), dc = __dsub_rn(fd, fc);
                        const double top = __dadd_rn(fa, __dmul_rn(ax, ba));
                        const double bot = __dadd_rn(fc, __dmul_rn(ax, dc));
                        rv = __dadd_rn(top, __dmul_rn(ay, __dsub_rn(bot, top)));
                        rg = __dadd_rn(__dmul_rn(ba, omay), __dmul_rn(dc, ay));
                    }
                    const double r = __dsub_rn(Tl, __dadd_rn(__dmul_rn(a, rv), b));
                    const double J0 = __dmul_rn(-a, rg), J1 = rv;
                    S[0] = __dadd_rn(S[0], __dmul_rn(J0, r));
                    S[1] = __dadd_rn(S[1], __dmul_rn(J1, r));
                    S[2] = __dadd_rn(S[2], r);
                    S[3] = __dadd_rn(S[3], __dmul_rn(J0, J0));
                    S[4] = __dadd_rn(S[4], __dmul_rn(J0, J1));
                    S[5] = __dadd_rn(S[5], J0);
                    S[6] = __dadd_rn(S[6], __dmul_rn(J1, J1));
                    S[7] = __dadd_rn(S[7], J1);
                    if (it == LK_ITERS) S[8] = __dadd_rn(S[8], __dmul_rn(r, r));
                }
            }
            double A[3][3] = {{S[3], S[4], S[5]}, {S[4], S[6], S[7]}, {S[5], S[7], (double)NPIX}};
#pragma unroll
            for (int i = 0; i < 3; ++i) A[i][i] = __dadd_rn(A[i][i], 1e-9);
            int piv[3];
            ob_getf2(A, piv);
            if (it < LK_ITERS) {
                double dl[3] = {S[0], S[1], S[2]};
                ob_getrs(A, piv, dl);
                d = __dadd_rn(d, dl[0]);
                a = __dadd_rn(a, dl[1]);
                b = __dadd_rn(b, dl[2]);
                if (!(isfinite(d) && isfinite(a))) break;
            } else {
                const double s2v = __ddiv_rn(S[8], (double)(NPIX - 3));
                ob_getri(A, piv);
                const double var = __dmul_rn(s2v, A[0][0]);
                sig = var > 0.0 ? __dsqrt_rn(var) : 0.0;
                const bool conv = isfinite(d) && fabs(__dsub_rn(d, seed)) <= 1.0 && a > 0.5 && a < 2.0;
                okl = conv && !(d < 0.5);
            }
        }
        if (okl) { od[J.oi] = d; osig[J.oi] = sig; ook[J.oi] = 1; }
    }

    // --------------------------------------------------------------------------------------- phase C: vertical scans
    // one lane per accepted job: the ZNCC of the matched right patch's column neighbourhood (scan offsets -HALF ..
    // HALF), its PW patches summed side by side, each in the reference's pixel order; then the first maximum and the
    // parabola.  u8 images: every accepted job's right-image block (2 PW - 1 rows x PW columns) and template are first
    // staged in shared memory over the LK blocks; the shifted float32 image is read from global memory (L1).
    const unsigned okm = __ballot_sync(0xffffffffu, okl);
    constexpr int VR = (2 * PW - 1) * PW;
    const int VJ = st_vjob_bytes(HALF);
    if (!FLT) {
        __syncwarp();
        constexpr int UB = 8;
        const int total = njobs * (VR + NPIX);
        for (int t0 = lane; t0 < total; t0 += 32 * UB) {
            u8 v[UB];
            bool w[UB];
#pragma unroll
            for (int u = 0; u < UB; ++u) {
                const int t = t0 + 32 * u;
                v[u] = 0;
                w[u] = false;
                if (t < total) {
                    const int j = t / (VR + NPIX), q = t - j * (VR + NPIX);
                    const StJob& J = jobs[j];
                    if (((okm >> j) & 1u) && J.vi - 2 * HALF - 1 >= 0 && J.vi + 2 * HALF + 1 < H) {
                        const size_t fo = (size_t)J.f * H * W;
                        w[u] = true;
                        if (q < VR) {
                            const int rr = q / PW, cc = q - rr * PW;
                            v[u] = R8all[fo + (size_t)(J.vi - 2 * HALF + rr) * W + J.xr - HALF + cc];
                        } else {
                            const int p2 = q - VR;
                            v[u] = Lall[fo + (size_t)(J.vi + p2 / PW - HALF) * W + J.ui + p2 % PW - HALF];
                        }
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < UB; ++u) {
                const int t = t0 + 32 * u;
                if (w[u]) {
                    const int j = t / (VR + NPIX), q = t - j * (VR + NPIX);
                    U[(size_t)j * VJ + q] = v[u];
                }
            }
        }
        __syncwarp();
    }
    if (okl) {
        const StJob J = jobs[lane];
        const int vi = J.vi, xr = J.xr, ui = J.ui;
        if (vi - 2 * HALF - 1 >= 0 && vi + 2 * HALF + 1 < H) {
            const u8* L = Lall + (size_t)J.f * H * W;
            RightImg<FLT> R;
            R.r8 = R8all ? R8all + (size_t)J.f * H * W : nullptr;
            R.rf = Rsall ? Rsall + (size_t)J.f * H * W : nullptr;
            const unsigned char* blk = U + (size_t)lane * VJ;
            auto tpl = [&](int q) -> int {
                return FLT ? (int)L[(size_t)(vi + q / PW - HALF) * W + ui + q % PW - HALF] : (int)blk[VR + q];
            };
            int st = 0;
#pragma unroll 1
            for (int q = 0; q < NPIX; ++q) st += tpl(q);
            const double tm = __ddiv_rn((double)st, (double)NPIX);
            double sx[PW], zs[PW], zs2[PW];
            int is[PW], is2[PW];
#pragma unroll
            for (int j = 0; j < PW; ++j) { sx[j] = 0.0; zs[j] = 0.0; zs2[j] = 0.0; is[j] = 0; is2[j] = 0; }
            const size_t r0 = (size_t)(vi - 2 * HALF) * W + (xr - HALF);
#pragma unroll 1
            for (int dy = 0; dy < PW; ++dy) {
#pragma unroll 1
                for (int dx = 0; dx < PW; ++dx) {
                    const double T = __dsub_rn((double)tpl(dy * PW + dx), tm);
#pragma unroll
                    for (int j = 0; j < PW; ++j) {
                        const float rf = FLT ? R.at(r0 + (size_t)(dy + j) * W + dx) : (float)blk[(dy + j) * PW + dx];
                        const double r = (double)rf;
                        if (FLT) {
                            zs[j] = __dadd_rn(zs[j], r);
                            zs2[j] = __dadd_rn(zs2[j], (double)__fmul_rn(rf, rf));
                        } else {
                            const int iv = (int)rf;
                            is[j] += iv;
                            is2[j] += iv * iv;
                        }
                        sx[j] = __dadd_rn(sx[j], __dmul_rn(r, T));
                    }
                }
            }
            double z[PW];
#pragma unroll
            for (int j = 0; j < PW; ++j) {
                if (!FLT) { zs[j] = (double)is[j]; zs2[j] = (double)is2[j]; }
                z[j] = zncc_finish(zs[j], zs2[j], sx[j], J.ts, NPIX);
            }
            // the first maximum above -2 (row 0 when none), then the parabola from its neighbours
            int jp = 0;
            double cs = -2.0;
#pragma unroll
            for (int j = 0; j < PW; ++j)
                if (z[j] > cs) { cs = z[j]; jp = j - HALF; }
            double y0 = 0.0, y2 = 0.0;
#pragma unroll
            for (int j = 0; j < PW; ++j) {
                if (j == jp - 1 + HALF) y0 = z[j];
                if (j == jp + 1 + HALF) y2 = z[j];
            }
            double offy = 0.0;
            if (jp > -HALF && jp < HALF) {
                const double den = __dadd_rn(__dsub_rn(y0, __dmul_rn(2.0, cs)), y2);
                if (den < -1e-9) {
                    offy = __ddiv_rn(__dmul_rn(0.5, __dsub_rn(y0, y2)), den);
                    if (offy > 0.5) offy = 0.5;
                    if (offy < -0.5) offy = -0.5;
                }
            }
            ody[J.oi] = __dadd_rn((double)jp, offy);
        }
    }
}

static int st_sm_count()
{
    static int sms[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (!sms[dev]) {
        int v = 0;
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        sms[dev] = v > 0 ? v : 148;
    }
    return sms[dev];
}

// units per warp that fill `per_sm` blocks of nw warps on every SM once, at most ST_GROUP
static int st_per_warp(long long units, int nw, int per_sm)
{
    const long long slots = (long long)st_sm_count() * per_sm * nw;
    const long long g = (units + slots - 1) / slots;
    return g < 1 ? 1 : (g > ST_GROUP ? ST_GROUP : (int)g);
}

template <int HALF, bool FLT>
static cudaError_t launch_stereo_t(const uint8_t* L, const uint8_t* R8, const float* Rs, int H, int W,
                                   const double* kpd, const long long* dlo_a, const long long* dhi_a, int n,
                                   const float* kpf, const int* counts, int cap, int dlo, int dhi, int band,
                                   double* od, double* osig, uint8_t* ook, double* ozn, double* ody, long long npts,
                                   int warps, int grp, void* jobs, cudaStream_t st)
{
    if (npts <= 0) return cudaSuccess;
    int* gcount = (int*)jobs;
    StJob* gjobs = (StJob*)((char*)jobs + 256);
    cudaError_t e = cudaMemsetAsync(gcount, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    // the search: the knobs, else st_warps warps and as many points per warp as fill ST_SEARCH_MINB blocks per SM
    int NW = warps >= 1 && warps <= st_warps(HALF) ? warps : st_warps(HALF);
    const size_t pw = stereo_search_bytes(HALF, band, FLT);
    if ((size_t)NW * pw > ST_SMEM_MAX) NW = (int)(ST_SMEM_MAX / pw);    // the widest bands: fewer warps per block
    const int G = grp >= 1 && grp <= ST_GROUP ? grp : st_per_warp(npts, NW, ST_SEARCH_MINB);
    const long long nb = (npts + (long long)NW * G - 1) / ((long long)NW * G);
    k_stereo_search<HALF, FLT><<<(unsigned)nb, NW * 32, pw * NW, st>>>(L, R8, Rs, H, W, kpd, dlo_a, dhi_a, n, kpf,
                                                                         counts, cap, dlo, dhi, band, od, osig, ook,
                                                                         ozn, ody, G, gjobs, gcount);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // the LKs and vertical scans of the jobs (at most npts), as many per warp as fill two blocks per SM once
    const int NW2 = st_warps(HALF);
    const int JP = st_per_warp(npts, NW2, 2);
    const long long nb2 = (npts + (long long)NW2 * JP - 1) / ((long long)NW2 * JP);
    k_stereo_lk<HALF, FLT><<<(unsigned)nb2, NW2 * 32, stereo_lk_bytes(HALF) * NW2, st>>>(L, R8, Rs, H, W, gjobs,
                                                                                      gcount, JP, od, osig, ook, ody);
    return cudaGetLastError();
}

// the largest window (band BAND_MAX) of every instantiation, set once before any launch or graph capture
// bytes of the job list a launch over npts points needs (a counter, then a 64-byte record per point that passes)
size_t xcb_stereo_jobs_bytes(long long npts) { return 256 + (size_t)(npts > 0 ? npts : 0) * sizeof(StJob); }

cudaError_t xcb_stereo_init_attrs()
{
    cudaError_t e = cudaSuccess;
#define XCB_SA(HH, FF)                                                                                            \
    if (e == cudaSuccess)                                                                                         \
        e = cudaFuncSetAttribute(k_stereo_search<HH, FF>, cudaFuncAttributeMaxDynamicSharedMemorySize,            \
                                 (int)st_smem_attr(HH, FF));                                                     \
    if (e == cudaSuccess)                                                                                         \
        e = cudaFuncSetAttribute(k_stereo_lk<HH, FF>, cudaFuncAttributeMaxDynamicSharedMemorySize,                \
                                 (int)(stereo_lk_bytes(HH) * st_warps(HH)));
    XCB_SA(3, false) XCB_SA(3, true) XCB_SA(4, false) XCB_SA(4, true) XCB_SA(5, false) XCB_SA(5, true)
#undef XCB_SA
    return e;
}

cudaError_t xcb_launch_stereo(const uint8_t* L, const uint8_t* R8, const float* Rs, int F, int H, int W,
                              const double* kpd, const long long* dlo_a, const long long* dhi_a, int n,
                              const float* kpf, const int* counts, int cap, int dlo, int dhi, int band, int half,
                              double* od, double* osig, uint8_t* ook, double* ozn, double* ody, unsigned int* err,
                              void* jobs, int warps, int grp, cudaStream_t st)
{
    if (band < 0 || band > BAND_MAX) return cudaErrorInvalidValue;
    long long npts = kpd ? (long long)n : (long long)F * cap;
    int nn = kpd ? n : F;
    bool flt = Rs != nullptr;
#define XCB_ST(HH)                                                                                                  \
    return flt ? launch_stereo_t<HH, true>(L, nullptr, Rs, H, W, kpd, dlo_a, dhi_a, nn, kpf, counts, cap, dlo, dhi,  \
                                           band, od, osig, ook, ozn, ody, npts, warps, grp, jobs, st)               \
               : launch_stereo_t<HH, false>(L, R8, nullptr, H, W, kpd, dlo_a, dhi_a, nn, kpf, counts, cap, dlo, dhi, \
                                            band, od, osig, ook, ozn, ody, npts, warps, grp, jobs, st);
    switch (half) {
        case 3: XCB_ST(3)
        case 4: XCB_ST(4)
        case 5: XCB_ST(5)
        default: return cudaErrorInvalidValue;
    }
#undef XCB_ST
}
