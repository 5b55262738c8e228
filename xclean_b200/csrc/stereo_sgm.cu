// stereo_sgm.cu -- dense 32-direction SGM on B200 (the reference's src/xclean/stereo/sgm32.py, bit for bit).
//
// The algorithm is the reference's: census 9x9 (80 comparisons in two words, the centre takes no bit, a neighbour
// outside the image reads as the centre), Hamming cost over d = 0..127 (80 where x - d < 0), Hirschmueller's
// recursion along 32 directed paths with the family-scaled penalties, one uint16 sum volume, the left winner with the
// uniqueness test and the parabola, the right winner off the same volume's diagonal, the left-right check.
//
// B200 layout:
//   k_sgm_cost   CTA per image row: the nine rows around it (both images) staged in shared memory, the row's census
//                words computed there for both images, then the row's 128 costs per pixel written as 32-bit words of
//                four disparities (consecutive threads, consecutive words): no census arrays in HBM
//   k_sgm_agg    warp per path, lane = four disparities (the recursion's neighbours d - 1 / d + 1 by shuffles), the
//                next pixel's costs loaded one step ahead; the path starts are computed from the path index, not
//                read from a table; the 32 directions' paths all in one launch, their terms added into the uint16
//                volume as pairs by 32-bit atomic adds (integer: the sum does not depend on the order)
//   k_sgm_select CTA per row: the row's right winners into shared memory, then the left winner, uniqueness, parabola,
//                confidence and the left-right check per pixel, one pass over the row's volume
#include <string>
#include <vector>

#include "common.cuh"

extern void xcb_set_last_error(const std::string& m);

#define SGM_D 128
#define SGM_BITS 80
#define SGM_MAXW 2048
#define SGM_INF (1 << 28)

struct xcb_sgm {
    int W, H, p1, p2;
    float uniq, lr, dmin;
    int npaths;
    int dir_dx[32], dir_dy[32], dir_p1[32], dir_p2[32];
    long long dir_off[33];       // first path index of each direction
    unsigned char* C;            // [H][W][128]
    unsigned short* S;           // [H][W][128]
    float *disp, *conf;          // host entry's device outputs
    unsigned char *in_l, *in_r;  // host entry's device inputs
    cudaStream_t stream;
    std::string err;
    // stage timing (xcb_sgm_set_stage_timing): per timed call four events (cost | aggregation incl. the zeroing of the
    // sum volume | selection), in a ring of SGM_TRING sets; xcb_sgm_stage_times sums the sets recorded since its last
    // call
    bool timing;
    int tn;
    std::vector<cudaEvent_t> tev;
};

#define SGM_TRING 256

struct SgmDirs {
    int dx[32], dy[32], p1[32], p2[32];
    long long off[33];
};

static int sgm_fail(xcb_sgm* s, int code, const std::string& m)
{
    if (s) s->err = m;
    xcb_set_last_error(m);
    return code;
}

// ----------------------------------------------------------------------------------------------------------- cost
__device__ __forceinline__ void census_at(const unsigned char* rows, int W, int x, int rvalid, uint64_t& a,
                                          unsigned& b)
{
    // rows: 9 staged rows (row 4 = the centre row); rvalid: bit r set when staged row r lies inside the image
    const unsigned char c = rows[4 * W + x];
    a = 0;
    b = 0;
    int bit = 0;
#pragma unroll
    for (int dy = 0; dy < 9; ++dy)
#pragma unroll
        for (int dx = -4; dx <= 4; ++dx) {
            if (dy == 4 && dx == 0) continue;
            const int nx = x + dx;
            const unsigned char v = ((rvalid >> dy) & 1) && nx >= 0 && nx < W ? rows[dy * W + nx] : c;
            const unsigned s = v < c;
            if (bit < 64) a |= (uint64_t)s << bit;
            else b |= s << (bit - 64);
            ++bit;
        }
}

__global__ void __launch_bounds__(256) k_sgm_cost(const unsigned char* __restrict__ L, const unsigned char* __restrict__ R,
                                                  int H, int W, unsigned char* __restrict__ C)
{
    extern __shared__ __align__(16) unsigned char sm[];
    unsigned char* rl = sm;                         // [9][W]
    unsigned char* rr = rl + 9 * W;                 // [9][W]
    uint64_t* l0 = (uint64_t*)(sm + ((18 * (size_t)W + 15) & ~(size_t)15));
    uint64_t* r0 = l0 + W;
    unsigned short* l1 = (unsigned short*)(r0 + W);
    unsigned short* r1 = l1 + W;
    const int y = blockIdx.x;
    int rvalid = 0;
    for (int r = 0; r < 9; ++r)
        if (y + r - 4 >= 0 && y + r - 4 < H) rvalid |= 1 << r;
    for (int i = threadIdx.x; i < 9 * W; i += blockDim.x) {
        const int r = i / W, x = i - r * W, yy = y + r - 4;
        const bool in = yy >= 0 && yy < H;
        rl[i] = in ? L[(size_t)yy * W + x] : 0;
        rr[i] = in ? R[(size_t)yy * W + x] : 0;
    }
    __syncthreads();
    for (int x = threadIdx.x; x < W; x += blockDim.x) {
        uint64_t a;
        unsigned b;
        census_at(rl, W, x, rvalid, a, b);
        l0[x] = a;
        l1[x] = (unsigned short)b;
        census_at(rr, W, x, rvalid, a, b);
        r0[x] = a;
        r1[x] = (unsigned short)b;
    }
    __syncthreads();
    unsigned* out = (unsigned*)(C + (size_t)y * W * SGM_D);
    for (int i = threadIdx.x; i < W * (SGM_D / 4); i += blockDim.x) {
        const int x = i >> 5, d0 = (i & 31) * 4;
        const uint64_t la = l0[x];
        const unsigned lb = l1[x];
        unsigned w = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int xr = x - d0 - k;
            const unsigned c = xr < 0 ? SGM_BITS : (unsigned)(__popcll(la ^ r0[xr]) + __popc(lb ^ (unsigned)r1[xr]));
            w |= c << (8 * k);
        }
        out[i] = w;
    }
}

// ---------------------------------------------------------------------------------------------------- aggregation
__device__ __forceinline__ int wmin32(int v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// path p of direction k starts at the p-th pixel whose predecessor lies outside the image: first the |dx| border
// columns (all rows), then the |dy| border rows (the other columns)
__device__ __forceinline__ void sgm_start(int dx, int dy, int W, int H, long long p, int& x, int& y)
{
    const int adx = abs(dx), ady = abs(dy);
    const long long ncol = (long long)adx * H;
    if (p < ncol) {
        const int c = (int)(p / H), r = (int)(p % H);
        x = dx > 0 ? c : W - 1 - c;
        y = r;
    } else {
        const long long q = p - ncol;
        const int wr = W - adx;                       // columns outside the border band
        const int r = (int)(q / wr), c = (int)(q % wr);
        y = dy > 0 ? r : H - 1 - r;
        x = dx > 0 ? adx + c : c;                     // dx < 0: the band is on the right, columns 0 .. W - adx - 1
    }
}

__global__ void __launch_bounds__(256) k_sgm_agg(const unsigned char* __restrict__ C, unsigned* __restrict__ S2, int H,
                                                 int W, SgmDirs dirs, long long npaths)
{
    const long long wp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (wp >= npaths) return;
    int k = 0;
    while (k < 31 && dirs.off[k + 1] <= wp) ++k;
    const int dx = dirs.dx[k], dy = dirs.dy[k], p1 = dirs.p1[k], p2 = dirs.p2[k];
    int x, y;
    sgm_start(dx, dy, W, H, wp - dirs.off[k], x, y);
    size_t base = ((size_t)y * W + x) * SGM_D + 4 * lane;
    uchar4 c4 = *reinterpret_cast<const uchar4*>(C + base);
    int L0 = c4.x, L1 = c4.y, L2 = c4.z, L3 = c4.w;
    atomicAdd(S2 + (base >> 1), (unsigned)L0 | ((unsigned)L1 << 16));
    atomicAdd(S2 + (base >> 1) + 1, (unsigned)L2 | ((unsigned)L3 << 16));
    int mprev = wmin32(min(min(L0, L1), min(L2, L3)));
    x += dx;
    y += dy;
    bool in = x >= 0 && x < W && y >= 0 && y < H;
    uchar4 nx4 = make_uchar4(0, 0, 0, 0);
    if (in) nx4 = *reinterpret_cast<const uchar4*>(C + ((size_t)y * W + x) * SGM_D + 4 * lane);
    while (in) {
        base = ((size_t)y * W + x) * SGM_D + 4 * lane;
        c4 = nx4;
        const int xn = x + dx, yn = y + dy;
        const bool in_n = xn >= 0 && xn < W && yn >= 0 && yn < H;
        if (in_n) nx4 = *reinterpret_cast<const uchar4*>(C + ((size_t)yn * W + xn) * SGM_D + 4 * lane);   // ahead
        int left = __shfl_up_sync(0xffffffffu, L3, 1);
        int right = __shfl_down_sync(0xffffffffu, L0, 1);
        if (lane == 0) left = SGM_INF;
        if (lane == 31) right = SGM_INF;
        const int mp2 = mprev + p2;
        const int n0 = (int)c4.x + min(min(L0, mp2), min(left, L1) + p1) - mprev;
        const int n1 = (int)c4.y + min(min(L1, mp2), min(L0, L2) + p1) - mprev;
        const int n2 = (int)c4.z + min(min(L2, mp2), min(L1, L3) + p1) - mprev;
        const int n3 = (int)c4.w + min(min(L3, mp2), min(L2, right) + p1) - mprev;
        L0 = n0; L1 = n1; L2 = n2; L3 = n3;
        atomicAdd(S2 + (base >> 1), (unsigned)L0 | ((unsigned)L1 << 16));
        atomicAdd(S2 + (base >> 1) + 1, (unsigned)L2 | ((unsigned)L3 << 16));
        mprev = wmin32(min(min(L0, L1), min(L2, L3)));
        x = xn;
        y = yn;
        in = in_n;
    }
}

// ------------------------------------------------------------------------------------------------------ selection
// CTA per row.  One pass over the row's sum vectors, a warp per pixel (four disparities per lane, 8-byte coalesced
// loads): the left winner (first minimum), the second best more than one disparity away and the parabola by shuffles;
// each S[x][d] is also a candidate of the right pixel x - d, whose winner (first minimum over d, as the reference scans
// it) is a shared-memory atomicMin of (sum << 8 | d).  Then the right winners' parabolas and the left-right check.
__device__ __forceinline__ unsigned sgm_pick(unsigned c0, unsigned c1, unsigned c2, unsigned c3, int k)
{
    return k == 0 ? c0 : (k == 1 ? c1 : (k == 2 ? c2 : c3));
}

__global__ void __launch_bounds__(256) k_sgm_select(const unsigned short* __restrict__ S, int H, int W, float uniq,
                                                    float dmin, float lr_thr, float* __restrict__ disp,
                                                    float* __restrict__ conf)
{
    extern __shared__ unsigned char sraw[];
    unsigned* rkey = (unsigned*)sraw;              // [W] right winner keys, then the right disparities (float bits)
    float* ld = (float*)(rkey + W);                // [W] left disparity (0 = invalid)
    float* lc = ld + W;                            // [W] its confidence
    const int y = blockIdx.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const unsigned short* Sy = S + (size_t)y * W * SGM_D;
    for (int x = threadIdx.x; x < W; x += blockDim.x) rkey[x] = 0xFFFFFFFFu;
    __syncthreads();
    for (int x = wid; x < W; x += nw) {
        const uint2 v = *reinterpret_cast<const uint2*>(Sy + (size_t)x * SGM_D + 4 * lane);
        const unsigned c0 = v.x & 0xffffu, c1 = v.x >> 16, c2 = v.y & 0xffffu, c3 = v.y >> 16;
        const int nd = min(SGM_D, x + 1);
        // right-winner candidates: right pixel x - d, d <= x
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int d = 4 * lane + k;
            if (d <= x) atomicMin(&rkey[x - d], (sgm_pick(c0, c1, c2, c3, k) << 8) | (unsigned)d);
        }
        // left winner: the first minimum over d < nd
        unsigned best = 0xFFFFFFFFu;
        int bd = 0x7fffffff;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int d = 4 * lane + k;
            const unsigned c = sgm_pick(c0, c1, c2, c3, k);
            if (d < nd && c < best) { best = c; bd = d; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned b2 = __shfl_xor_sync(0xffffffffu, best, o);
            const int d2 = __shfl_xor_sync(0xffffffffu, bd, o);
            if (b2 < best || (b2 == best && d2 < bd)) { best = b2; bd = d2; }
        }
        // the best more than one disparity away
        unsigned sec = 0xFFFFFFFFu;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int d = 4 * lane + k;
            const unsigned c = sgm_pick(c0, c1, c2, c3, k);
            if (d < nd && abs(d - bd) > 1 && c < sec) sec = c;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sec = min(sec, __shfl_xor_sync(0xffffffffu, sec, o));
        // the neighbours of the winner (for the parabola)
        const int dm = bd > 0 ? bd - 1 : 0, dp = bd + 1 < SGM_D ? bd + 1 : SGM_D - 1;
        const unsigned cvl = sgm_pick(c0, c1, c2, c3, dm & 3), cnl = sgm_pick(c0, c1, c2, c3, dp & 3);
        const int cv = (int)__shfl_sync(0xffffffffu, cvl, dm >> 2);
        const int cn = (int)__shfl_sync(0xffffffffu, cnl, dp >> 2);
        if (lane == 0) {
            float o_d = 0.0f, o_c = 0.0f;
            if (!(sec != 0xFFFFFFFFu && (float)sec <= __fmul_rn((float)best, __fadd_rn(1.0f, uniq)))) {
                float sd = (float)bd;
                if (bd > 0 && bd < nd - 1) {
                    const int den = cv - 2 * (int)best + cn;
                    if (den > 0) {
                        const float off = __fdiv_rn((float)(cv - cn), (float)(2 * den));
                        sd = __fadd_rn((float)bd, fmaxf(-1.0f, fminf(1.0f, off)));
                    }
                }
                const float cval = (sec != 0xFFFFFFFFu && sec > 0) ? __fsub_rn(1.0f, __fdiv_rn((float)best, (float)sec))
                                                                   : 0.5f;
                o_d = sd >= dmin ? sd : 0.0f;
                o_c = sd >= dmin ? fmaxf(0.0f, fminf(1.0f, cval)) : 0.0f;
            }
            ld[x] = o_d;
            lc[x] = o_c;
        }
    }
    __syncthreads();
    // the right winners' parabolas (their neighbours read from the volume), in place of the keys
    for (int x = threadIdx.x; x < W; x += blockDim.x) {
        const unsigned key = rkey[x];
        const int bd = (int)(key & 0xffu), best = (int)(key >> 8);
        const int nd = min(SGM_D, W - x);
        float sd = (float)bd;
        if (bd > 0 && bd < nd - 1) {
            const int cv = (int)Sy[(size_t)(x + bd - 1) * SGM_D + bd - 1];
            const int cn = (int)Sy[(size_t)(x + bd + 1) * SGM_D + bd + 1];
            const int den = cv - 2 * best + cn;
            if (den > 0) {
                const float off = __fdiv_rn((float)(cv - cn), (float)(2 * den));
                sd = __fadd_rn((float)bd, fmaxf(-1.0f, fminf(1.0f, off)));
            }
        }
        rkey[x] = __float_as_uint(sd);
    }
    __syncthreads();
    // the left-right check against the row's right winners
    for (int x = threadIdx.x; x < W; x += blockDim.x) {
        float o_d = ld[x], o_c = lc[x];
        if (o_d > 0.0f) {
            const int xr = x - (int)__fadd_rn(o_d, 0.5f);
            if (xr < 0 || xr >= W || fabsf(__fsub_rn(o_d, __uint_as_float(rkey[xr]))) > lr_thr) { o_d = 0.0f; o_c = 0.0f; }
        }
        const size_t p = (size_t)y * W + x;
        disp[p] = o_d;
        conf[p] = o_c;
    }
}

// ---------------------------------------------------------------------------------------------------------- C ABI
static const int kFam[7][4] = {{1, 1, 1, 1}, {1, 2, 9, 4}, {2, 1, 9, 4}, {1, 3, 19, 6},
                               {3, 1, 19, 6}, {2, 3, 18, 5}, {3, 2, 18, 5}};

extern "C" int xcb_sgm_create(int width, int height, int p1, int p2, float uniq, float lr_thr, float dmin,
                              xcb_sgm** out)
{
    if (!out) return sgm_fail(nullptr, XCB_ERR_ARG, "sgm_create: null output");
    *out = nullptr;
    if (width < 4 || width > SGM_MAXW || height < 1 || height > 16384 || p1 < 0 || p2 < 0)
        return sgm_fail(nullptr, XCB_ERR_ARG, "sgm_create: 4 <= width <= 2048, 1 <= height <= 16384, p1 / p2 >= 0");
    xcb_sgm* s = new xcb_sgm();
    s->W = width; s->H = height; s->p1 = p1; s->p2 = p2; s->uniq = uniq; s->lr = lr_thr; s->dmin = dmin;
    int k = 0;
    const int ax[4][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}};
    for (auto& a : ax) { s->dir_dx[k] = a[0]; s->dir_dy[k] = a[1]; s->dir_p1[k] = p1; s->dir_p2[k] = p2; ++k; }
    for (auto& f : kFam)
        for (int sx = 1; sx >= -1; sx -= 2)
            for (int sy = 1; sy >= -1; sy -= 2) {
                s->dir_dx[k] = sx * f[0]; s->dir_dy[k] = sy * f[1];
                s->dir_p1[k] = p1 * f[2] / f[3]; s->dir_p2[k] = p2 * f[2] / f[3];
                ++k;
            }
    // the uint16 sum is exact only while 32 x (80 + the largest P2) fits
    int p2max = 0;
    for (int i = 0; i < 32; ++i) p2max = p2max > s->dir_p2[i] ? p2max : s->dir_p2[i];
    if (32 * (SGM_BITS + p2max) >= 65536) {
        delete s;
        return sgm_fail(nullptr, XCB_ERR_ARG, "sgm_create: p2 too large for an exact uint16 sum volume");
    }
    long long off = 0;
    for (int i = 0; i < 32; ++i) {
        s->dir_off[i] = off;
        const int adx = abs(s->dir_dx[i]), ady = abs(s->dir_dy[i]);
        const int bx = adx < width ? adx : width, by = ady < height ? ady : height;
        off += (long long)bx * height + (long long)by * (width - bx);
    }
    s->dir_off[32] = off;
    s->npaths = (int)off;
    const size_t n = (size_t)width * height;
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&s->C, n * SGM_D);
    if (e == cudaSuccess) e = cudaMalloc(&s->S, n * SGM_D * 2);
    if (e == cudaSuccess) e = cudaMalloc(&s->disp, n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&s->conf, n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&s->in_l, n);
    if (e == cudaSuccess) e = cudaMalloc(&s->in_r, n);
    static XcbAttrOnce a_cost;
    const int sm_cost = (int)(((18 * (size_t)SGM_MAXW + 15) & ~(size_t)15) + (size_t)SGM_MAXW * 20);
    if (e == cudaSuccess) e = xcb_smem_attr_once(a_cost, (const void*)k_sgm_cost, sm_cost);
    if (e != cudaSuccess) {
        const std::string m = std::string("sgm_create: ") + cudaGetErrorString(e);
        cudaFree(s->C); cudaFree(s->S); cudaFree(s->disp); cudaFree(s->conf); cudaFree(s->in_l); cudaFree(s->in_r);
        if (s->stream) cudaStreamDestroy(s->stream);
        delete s;
        return sgm_fail(nullptr, XCB_ERR_CUDA, m);
    }
    *out = s;
    return XCB_OK;
}

extern "C" void xcb_sgm_destroy(xcb_sgm* s)
{
    if (!s) return;
    cudaStreamSynchronize(s->stream);
    for (cudaEvent_t e : s->tev) cudaEventDestroy(e);
    cudaFree(s->C); cudaFree(s->S); cudaFree(s->disp); cudaFree(s->conf); cudaFree(s->in_l); cudaFree(s->in_r);
    cudaStreamDestroy(s->stream);
    delete s;
}

extern "C" const char* xcb_sgm_last_error(const xcb_sgm* s) { return s ? s->err.c_str() : xcb_last_error(); }

extern "C" int xcb_sgm_set_stage_timing(xcb_sgm* s, int on)
{
    if (!s) return sgm_fail(nullptr, XCB_ERR_ARG, "sgm_set_stage_timing: null handle");
    if (on && s->tev.empty()) {
        s->tev.assign(4 * SGM_TRING, nullptr);
        for (auto& e : s->tev) {
            const cudaError_t r = cudaEventCreate(&e);
            if (r != cudaSuccess) {
                for (auto& q : s->tev)
                    if (q) cudaEventDestroy(q);
                s->tev.clear();
                return sgm_fail(s, XCB_ERR_CUDA, std::string("sgm_set_stage_timing: ") + cudaGetErrorString(r));
            }
        }
    }
    s->timing = on != 0;
    s->tn = 0;
    return XCB_OK;
}

// ms[3]: cost, aggregation (with the zeroing of the sum volume), selection, summed over the timed calls since the last
// read (at most the last SGM_TRING); *ncalls: how many.  Waits for those calls.
extern "C" int xcb_sgm_stage_times(xcb_sgm* s, float* ms, int* ncalls)
{
    if (!s || !ms) return sgm_fail(s, XCB_ERR_ARG, "sgm_stage_times: null argument");
    ms[0] = ms[1] = ms[2] = 0.0f;
    const int n = s->tn < SGM_TRING ? s->tn : SGM_TRING;
    for (int c = 0; c < n; ++c) {
        cudaEvent_t* ev = &s->tev[4 * c];
        for (int i = 0; i < 3; ++i) {
            float t = 0.0f;
            cudaError_t e = cudaEventSynchronize(ev[i + 1]);
            if (e == cudaSuccess) e = cudaEventElapsedTime(&t, ev[i], ev[i + 1]);
            if (e != cudaSuccess) return sgm_fail(s, XCB_ERR_CUDA, std::string("sgm_stage_times: ") + cudaGetErrorString(e));
            ms[i] += t;
        }
    }
    if (ncalls) *ncalls = n;
    s->tn = 0;
    return XCB_OK;
}

extern "C" int xcb_sgm_compute_dev(xcb_sgm* s, const uint8_t* left, const uint8_t* right, float* disp, float* conf,
                                   void* stream)
{
    if (!s || !left || !right || !disp || !conf) return sgm_fail(s, XCB_ERR_ARG, "sgm_compute: null argument");
    cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
    const int W = s->W, H = s->H;
    const size_t n = (size_t)W * H;
    SgmDirs dirs;
    for (int i = 0; i < 32; ++i) {
        dirs.dx[i] = s->dir_dx[i]; dirs.dy[i] = s->dir_dy[i]; dirs.p1[i] = s->dir_p1[i]; dirs.p2[i] = s->dir_p2[i];
        dirs.off[i] = s->dir_off[i];
    }
    dirs.off[32] = s->dir_off[32];
    cudaEvent_t* ev = s->timing ? &s->tev[4 * (s->tn % SGM_TRING)] : nullptr;
    if (ev) ++s->tn;
    const size_t sm_cost = ((18 * (size_t)W + 15) & ~(size_t)15) + (size_t)W * 20;
    if (ev) cudaEventRecord(ev[0], st);
    k_sgm_cost<<<H, 256, sm_cost, st>>>(left, right, H, W, s->C);
    if (ev) cudaEventRecord(ev[1], st);
    cudaError_t e = cudaMemsetAsync(s->S, 0, n * SGM_D * 2, st);
    if (e != cudaSuccess) return sgm_fail(s, XCB_ERR_CUDA, std::string("sgm_compute: ") + cudaGetErrorString(e));
    const long long threads = (long long)s->npaths * 32;
    k_sgm_agg<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(s->C, (unsigned*)s->S, H, W, dirs, s->npaths);
    if (ev) cudaEventRecord(ev[2], st);
    k_sgm_select<<<H, 256, (size_t)W * 12, st>>>(s->S, H, W, s->uniq, s->dmin, s->lr, disp, conf);
    if (ev) cudaEventRecord(ev[3], st);
    e = cudaGetLastError();
    if (e != cudaSuccess) return sgm_fail(s, XCB_ERR_CUDA, std::string("sgm_compute: ") + cudaGetErrorString(e));
    return XCB_OK;
}

extern "C" int xcb_sgm_compute_host(xcb_sgm* s, const uint8_t* left, const uint8_t* right, float* disp, float* conf)
{
    if (!s || !left || !right || !disp || !conf) return sgm_fail(s, XCB_ERR_ARG, "sgm_compute_host: null argument");
    const size_t n = (size_t)s->W * s->H;
    cudaError_t e = cudaMemcpyAsync(s->in_l, left, n, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->in_r, right, n, cudaMemcpyHostToDevice, s->stream);
    if (e != cudaSuccess) return sgm_fail(s, XCB_ERR_CUDA, std::string("sgm_compute_host: ") + cudaGetErrorString(e));
    int rc = xcb_sgm_compute_dev(s, s->in_l, s->in_r, s->disp, s->conf, s->stream);
    if (rc) return rc;
    e = cudaMemcpyAsync(disp, s->disp, n * 4, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(conf, s->conf, n * 4, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return sgm_fail(s, XCB_ERR_CUDA, std::string("sgm_compute_host: ") + cudaGetErrorString(e));
    return XCB_OK;
}

extern "C" int xcb_sgm_buffers(xcb_sgm* s, void** cost, void** sum, int* npaths)
{
    if (!s) return sgm_fail(nullptr, XCB_ERR_ARG, "sgm_buffers: null handle");
    if (cost) *cost = s->C;
    if (sum) *sum = s->S;
    if (npaths) *npaths = s->npaths;
    return XCB_OK;
}

extern "C" int xcb_sgm_read_volumes(xcb_sgm* s, uint8_t* cost, uint16_t* sum)
{
    if (!s) return sgm_fail(nullptr, XCB_ERR_ARG, "sgm_read_volumes: null handle");
    const size_t n = (size_t)s->W * s->H * SGM_D;
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e == cudaSuccess && cost) e = cudaMemcpy(cost, s->C, n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && sum) e = cudaMemcpy(sum, s->S, n * 2, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return sgm_fail(s, XCB_ERR_CUDA, std::string("sgm_read_volumes: ") + cudaGetErrorString(e));
    return XCB_OK;
}
