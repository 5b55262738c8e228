// ba_assemble.cu -- the window Problem assembled on the device from the engine's state (P1Engine._problem,
// src/xclean/vio/engine_live.py:407-530, visual part), straight into the batched solve's window layout, so that a
// keyframe's BA needs no host round trip between the engine state and the solve.
//
// Steps (each a launch on the caller's stream, no host synchronisation):
//   k_asm_alive   one CTA: the alive (and selected) landmarks in id order -> their local index (block scan),
//                 the alive list, L; the slots' observation offsets
//   k_asm_count   thread per observation: its landmark's local index, per-landmark counts
//   k_asm_scan    one CTA: the per-landmark observation ranges (lm_ob), M
//   k_asm_place   thread per kept observation: a slot in its landmark's range
//   k_asm_order   thread per landmark: the range sorted by observation index (the reference's stable sort)
//   k_asm_rows    thread per row: pose slot, camera, pixel, validity, whitening, (slot, index) source
//   k_asm_lms     thread per landmark: position, host slot, inverse-depth prior
#include <string>

#include "common.cuh"

extern void xcb_set_last_error(const std::string& m);

#define ASM_T 1024

struct AsmWork {
    int* loc;        // [n_lm] local index or -1
    int* local;      // [M] local index of each observation or -1
    int* cnt;        // [n_lm] observations per landmark, then the placement cursors
    int* tmp;        // [M] observation indices in landmark order
    long long* soff; // [P + 1] slot observation offsets
};

// exclusive block scan of one int per thread (ASM_T threads); returns the total through *total
__device__ int asm_block_scan(int v, int* total)
{
    __shared__ int ws[ASM_T / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int w = lane < ASM_T / 32 ? ws[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < ASM_T / 32) ws[lane] = w;
    }
    __syncthreads();
    const int before = (wid > 0 ? ws[wid - 1] : 0) + x - v;
    *total = ws[ASM_T / 32 - 1];
    __syncthreads();
    return before;
}

__global__ void __launch_bounds__(ASM_T) k_asm_alive(xcb_ba_engine e, xcb_ba_assembled o, AsmWork w)
{
    const int tid = threadIdx.x;
    if (tid == 0) {
        long long s = 0;
        for (int i = 0; i < e.P; ++i) { w.soff[i] = s; s += e.slot_n[i]; }
        w.soff[e.P] = s;
    }
    const int per = (e.n_lm + ASM_T - 1) / ASM_T;
    const int b = tid * per, end = min(e.n_lm, b + per);
    int c = 0;
    for (int i = b; i < end; ++i) c += (e.lm_alive[i] && (!e.select || e.select[i])) ? 1 : 0;
    int total = 0;
    int r = asm_block_scan(c, &total);
    for (int i = b; i < end; ++i) {
        const bool a = e.lm_alive[i] && (!e.select || e.select[i]);
        w.loc[i] = a ? r : -1;
        if (a) o.alive[r++] = i;
        w.cnt[i] = 0;
    }
    if (tid == 0) o.counts[0] = total;
}

__device__ __forceinline__ int asm_slot_of(const long long* soff, int P, long long j)
{
    int s = 0;
    while (s + 1 < P && soff[s + 1] <= j) ++s;
    return s;
}

__global__ void k_asm_count(xcb_ba_engine e, AsmWork w)
{
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= e.M) return;
    const long long id = e.lid[j];
    const int l = (id >= 0 && id < e.n_lm) ? w.loc[id] : -1;
    w.local[j] = l;
    if (l >= 0) atomicAdd(&w.cnt[l], 1);
}

__global__ void __launch_bounds__(ASM_T) k_asm_scan(xcb_ba_engine e, xcb_ba_assembled o, AsmWork w)
{
    const int L = o.counts[0];
    const int per = (L + ASM_T - 1) / ASM_T;
    const int b = threadIdx.x * per, end = min(L, b + per);
    int c = 0;
    for (int i = b; i < end; ++i) c += w.cnt[i];
    int total = 0;
    int r = asm_block_scan(c, &total);
    for (int i = b; i < end; ++i) {
        o.lm_ob[i] = r;
        r += w.cnt[i];
        w.cnt[i] = 0;                        // the placement cursors
    }
    if (threadIdx.x == 0) {
        o.lm_ob[L] = total;
        o.counts[1] = total;
    }
}

__global__ void k_asm_place(xcb_ba_engine e, xcb_ba_assembled o, AsmWork w)
{
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= e.M) return;
    const int l = w.local[j];
    if (l < 0) return;
    w.tmp[o.lm_ob[l] + atomicAdd(&w.cnt[l], 1)] = (int)j;
}

// a landmark's rows in increasing observation index (insertion sort: a landmark has tens of rows at most)
__global__ void k_asm_order(xcb_ba_assembled o, AsmWork w)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= o.counts[0]) return;
    int* a = w.tmp + o.lm_ob[l];
    const int n = o.lm_ob[l + 1] - o.lm_ob[l];
    for (int i = 1; i < n; ++i) {
        const int v = a[i];
        int k = i - 1;
        while (k >= 0 && a[k] > v) { a[k + 1] = a[k]; --k; }
        a[k + 1] = v;
    }
}

// numpy's maximum: NaN wins
__device__ __forceinline__ double asm_maximum(double a, double b)
{
    if (a != a || b != b) return __longlong_as_double(0x7ff8000000000000LL);
    return a >= b ? a : b;
}

__global__ void k_asm_rows(xcb_ba_engine e, xcb_ba_assembled o, AsmWork w)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= o.counts[1]) return;
    const long long j = w.tmp[r];
    const int s = asm_slot_of(w.soff, e.P, j);
    const long long cam = e.cam[j];
    o.ob_pose[r] = s;
    o.ob_cam[r] = (uint8_t)cam;
    o.ob_z[2 * r] = e.uv[2 * j];
    o.ob_z[2 * r + 1] = e.uv[2 * j + 1];
    o.ob_valid[r] = e.valid[j] ? 1 : 0;
    o.ob_isig[r] = cam == 0 ? 1.0 / e.sig_px : 1.0 / asm_maximum(e.kappa_d * e.sig[j], 1e-9);
    o.src[2 * r] = s;
    o.src[2 * r + 1] = (int)(j - w.soff[s]);
}

__global__ void k_asm_lms(xcb_ba_engine e, xcb_ba_assembled o)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= o.counts[0]) return;
    const long long g = o.alive[l];
    for (int k = 0; k < 3; ++k) o.lmp[3 * l + k] = e.lm_p[3 * g + k];
    int hs = -1;
    for (int s = 0; s < e.P; ++s)
        if (e.sids[s] == e.lm_host[g]) { hs = s; break; }
    if (hs < 0) atomicExch(&o.counts[2], 1);       // a host that left the window (the reference raises)
    o.lm_host[l] = hs < 0 ? 0 : hs;
    o.lm_mask[l] = 1;
    double rm = 0.0, ris = 0.0;
    if (e.prior_mode) {
        rm = e.lm_rho_meas[g];
        const double sg = asm_maximum(e.kappa_d * e.lm_sig_lk[g], e.lm_span[g]) / e.fB;
        const bool fin = sg == sg && fabs(sg) != __longlong_as_double(0x7ff0000000000000LL);
        ris = (fin && sg > 0.0 && rm > 0.0) ? 1.0 / sg : 0.0;
    }
    o.rho_meas[l] = rm;
    o.rho_isig[l] = ris;
}

extern "C" size_t xcb_ba_assemble_scratch_bytes(int n_lm, int M, int P)
{
    const size_t a = ((size_t)(n_lm > 0 ? n_lm : 1) * 4 + 255) / 256 * 256;
    const size_t b = ((size_t)(M > 0 ? M : 1) * 4 + 255) / 256 * 256;
    const size_t c = ((size_t)(P + 1) * 8 + 255) / 256 * 256;
    return 2 * a + 2 * b + c;
}

extern "C" int xcb_ba_assemble_dev(const xcb_ba_engine* e, xcb_ba_assembled* o, void* scratch, size_t scratch_bytes,
                                   void* stream)
{
    if (!e || !o || !scratch) {
        xcb_set_last_error("ba_assemble: null argument");
        return XCB_ERR_ARG;
    }
    if (e->P < 1 || e->P > 64 || e->M < 0 || e->n_lm < 0 || e->fB == 0.0) {
        xcb_set_last_error("ba_assemble: P in 1..64, M and n_lm non-negative, fB non-zero");
        return XCB_ERR_ARG;
    }
    if (scratch_bytes < xcb_ba_assemble_scratch_bytes(e->n_lm, e->M, e->P)) {
        xcb_set_last_error("ba_assemble: scratch smaller than xcb_ba_assemble_scratch_bytes");
        return XCB_ERR_CAPACITY;
    }
    char* p = (char*)scratch;
    const size_t a = ((size_t)(e->n_lm > 0 ? e->n_lm : 1) * 4 + 255) / 256 * 256;
    const size_t b = ((size_t)(e->M > 0 ? e->M : 1) * 4 + 255) / 256 * 256;
    AsmWork w;
    w.loc = (int*)p; p += a;
    w.cnt = (int*)p; p += a;
    w.local = (int*)p; p += b;
    w.tmp = (int*)p; p += b;
    w.soff = (long long*)p;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t err = cudaMemsetAsync(o->counts, 0, 3 * sizeof(int), st);
    if (err == cudaSuccess) {
        const unsigned gm = (unsigned)((e->M + 255) / 256 > 0 ? (e->M + 255) / 256 : 1);
        const unsigned gl = (unsigned)((e->n_lm + 255) / 256 > 0 ? (e->n_lm + 255) / 256 : 1);
        k_asm_alive<<<1, ASM_T, 0, st>>>(*e, *o, w);
        k_asm_count<<<gm, 256, 0, st>>>(*e, w);
        k_asm_scan<<<1, ASM_T, 0, st>>>(*e, *o, w);
        k_asm_place<<<gm, 256, 0, st>>>(*e, *o, w);
        k_asm_order<<<gl, 256, 0, st>>>(*o, w);
        k_asm_rows<<<gm, 256, 0, st>>>(*e, *o, w);
        k_asm_lms<<<gl, 256, 0, st>>>(*e, *o);
        err = cudaGetLastError();
    }
    if (err != cudaSuccess) {
        xcb_set_last_error(std::string("ba_assemble: ") + cudaGetErrorString(err));
        return XCB_ERR_CUDA;
    }
    return XCB_OK;
}
