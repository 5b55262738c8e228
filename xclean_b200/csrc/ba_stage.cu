// ba_stage.cu -- the local-BA stage kernels behind the drop-in of src/xclean/backend/kernels.py (sm_100a).
//
// Same entry points, argument order, layouts (float32 / int32, row-major) and arithmetic as the reference's kernels;
// the differences are in how the work is mapped onto the GPU:
//   * build_blocks[_id]: one thread per observation; the per-landmark sums (Hll, bl) are first reduced across each
//     warp's runs of equal landmark index with a segmented shuffle scan (observations arrive sorted by landmark from
//     the solver, so a warp usually holds a handful of landmarks) and added once per run instead of once per
//     observation;
//   * schur_pairs[_id], schur_grad[_id], pose_blocks[_id]: one thread per (item, row) computes the row's 3-vector
//     Hpl Hlli once and loops over the columns, instead of one thread per (item, row, column) recomputing it;
//   * chol_solve: one CTA; the matrix is staged in shared memory when it fits (n <= 150), so the n column steps
//     and their barriers run against shared memory rather than L2.
// Sums into Hll, bl, Hred and g use float atomics, as in the reference: their order is unspecified, and results are
// compared with a tolerance.
#include <string>

#include "common.cuh"

extern void xcb_set_last_error(const std::string& m);

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int TPB = 256;

inline unsigned nblk(long long total, int tpb = TPB) { return (unsigned)((total + tpb - 1) / tpb); }

// Segmented sum over runs of equal `key` in the warp: -> this lane's inclusive run sum; *tail = last lane of its run.
__device__ __forceinline__ float seg_sum(float v, int key, int lane, bool* tail)
{
    const int kprev = __shfl_up_sync(FULL, key, 1);
    const int knext = __shfl_down_sync(FULL, key, 1);
    bool f = lane == 0 || kprev != key;
    *tail = lane == 31 || knext != key;
    float s = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const float so = __shfl_up_sync(FULL, s, d);
        const bool fo = __shfl_up_sync(FULL, (int)f, d) != 0;
        if (lane >= d) {
            if (!f) s += so;
            f = f || fo;
        }
    }
    return s;
}

// Hll (9) and bl (3) of one observation into the landmark's sums, aggregated per warp run of equal landmark.
// `l` < 0 for lanes without an observation (their values are zero and never written).
__device__ __forceinline__ void add_landmark_sums(const float hv[9], const float bv[3], int l, float* Hll, float* bl)
{
    const int lane = threadIdx.x & 31;
    const int key = l >= 0 ? l : -1 - lane;          // lanes without an observation form runs of their own
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        bool tail;
        const float s = seg_sum(i < 9 ? hv[i] : bv[i - 9], key, lane, &tail);
        if (tail && l >= 0) {
            if (i < 9) atomicAdd(&Hll[(long long)l * 9 + i], s);
            else atomicAdd(&bl[(long long)l * 3 + i - 9], s);
        }
    }
}

__device__ __forceinline__ float huber_sw(float e, float k)
{
    const float w = e <= k ? 1.f : k / fmaxf(e, 1e-9f);
    return sqrtf(w);
}

// ------------------------------------------------------------------------------------------------ Euclidean build
__global__ void __launch_bounds__(TPB) k_build_blocks(const float* __restrict__ Tcw, const float* __restrict__ pts,
                                                      const int* __restrict__ okf, const int* __restrict__ olm,
                                                      const float* __restrict__ ouv, float* __restrict__ Jpose,
                                                      float* __restrict__ Jlm, float* __restrict__ resw,
                                                      float* __restrict__ Hll, float* __restrict__ bl,
                                                      float* __restrict__ Hpl, int N, float fx, float cx, float cy,
                                                      float huber)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    float hv[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, bv[3] = {0.f, 0.f, 0.f};
    int l = -1;
    if (o < N) {
        const int k = okf[o];
        l = olm[o];
        const float* T = Tcw + (long long)k * 12;
        const float* P = pts + (long long)l * 3;
        const float x = T[0] * P[0] + T[1] * P[1] + T[2] * P[2] + T[3];
        const float y = T[4] * P[0] + T[5] * P[1] + T[6] * P[2] + T[7];
        const float z = fmaxf(T[8] * P[0] + T[9] * P[1] + T[10] * P[2] + T[11], 1e-6f);
        const float iz = 1.f / z;
        const float ru = fx * x * iz + cx - ouv[2 * (long long)o];
        const float rv = fx * y * iz + cy - ouv[2 * (long long)o + 1];
        const float sw = huber_sw(sqrtf(ru * ru + rv * rv), huber);
        // d(u, v)/d(Pc), scaled by sqrt(w)
        const float a0 = fx * iz * sw, a2u = -fx * x * iz * iz * sw, a2v = -fx * y * iz * iz * sw;
        // pose block: A [I | -hat(Pc)]
        float jp[2][6];
        jp[0][0] = a0; jp[0][1] = 0.f; jp[0][2] = a2u;
        jp[0][3] = a2u * y; jp[0][4] = a0 * z - a2u * x; jp[0][5] = -a0 * y;
        jp[1][0] = 0.f; jp[1][1] = a0; jp[1][2] = a2v;
        jp[1][3] = -a0 * z + a2v * y; jp[1][4] = -a2v * x; jp[1][5] = a0 * x;
        // landmark block: A R_cw
        float jl[2][3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            jl[0][c] = a0 * T[c] + a2u * T[8 + c];
            jl[1][c] = a0 * T[4 + c] + a2v * T[8 + c];
        }
        const float rwu = ru * sw, rwv = rv * sw;
        float* jo = Jpose + (long long)o * 12;
#pragma unroll
        for (int c = 0; c < 6; ++c) { jo[c] = jp[0][c]; jo[6 + c] = jp[1][c]; }
        float* lo = Jlm + (long long)o * 6;
#pragma unroll
        for (int c = 0; c < 3; ++c) { lo[c] = jl[0][c]; lo[3 + c] = jl[1][c]; }
        resw[2 * (long long)o] = rwu;
        resw[2 * (long long)o + 1] = rwv;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
#pragma unroll
            for (int b = 0; b < 3; ++b) hv[a * 3 + b] = jl[0][a] * jl[0][b] + jl[1][a] * jl[1][b];
            bv[a] = -(jl[0][a] * rwu + jl[1][a] * rwv);
        }
        float* ho = Hpl + (long long)o * 18;
#pragma unroll
        for (int a = 0; a < 6; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) ho[a * 3 + b] = jp[0][a] * jl[0][b] + jp[1][a] * jl[1][b];
    }
    add_landmark_sums(hv, bv, l, Hll, bl);
}

__global__ void k_depth_prior(const float* __restrict__ pts, const float* __restrict__ chost,
                              const float* __restrict__ rho0, const float* __restrict__ invsig,
                              const float* __restrict__ valid, float* __restrict__ Hll, float* __restrict__ bl, int nl,
                              float huber)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nl || valid[l] < 0.5f) return;
    const float dx = pts[3 * l] - chost[3 * l], dy = pts[3 * l + 1] - chost[3 * l + 1],
                dz = pts[3 * l + 2] - chost[3 * l + 2];
    const float d2 = dx * dx + dy * dy + dz * dz;
    if (d2 < 1e-12f) return;
    const float dist = sqrtf(d2), rho = 1.f / dist, is = invsig[l];
    const float r = (rho - rho0[l]) * is;
    const float sw = huber_sw(fabsf(r), huber);
    const float g = -rho * rho / dist * is * sw;       // d rho / dP = -(P - c) / dist^3
    const float J[3] = {g * dx, g * dy, g * dz};
    const float rw = r * sw;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int b = 0; b < 3; ++b) atomicAdd(&Hll[(long long)l * 9 + a * 3 + b], J[a] * J[b]);
        atomicAdd(&bl[(long long)l * 3 + a], -J[a] * rw);
    }
}

__global__ void k_inv3_damped(const float* __restrict__ Hll, float* __restrict__ Hlli, int nl, float lam)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nl) return;
    const float* H = Hll + (long long)l * 9;
    const float dmp = lam * fmaxf((H[0] + H[4] + H[8]) / 3.f, 1e-9f);
    const float a = H[0] + dmp, b = H[1], c = H[2], d = H[3], e = H[4] + dmp, f = H[5], g = H[6], h = H[7],
                i = H[8] + dmp;
    // cofactors of the first row, the determinant, then the adjugate
    const float C0 = e * i - f * h, C1 = -(d * i - f * g), C2 = d * h - e * g;
    float det = a * C0 + b * C1 + c * C2;
    if (fabsf(det) < 1e-30f) det = det < 0.f ? -1e-30f : 1e-30f;
    const float id = 1.f / det;
    float* O = Hlli + (long long)l * 9;
    O[0] = C0 * id;                 O[1] = -(b * i - c * h) * id;   O[2] = (b * f - c * e) * id;
    O[3] = C1 * id;                 O[4] = (a * i - c * g) * id;    O[5] = -(a * f - c * d) * id;
    O[6] = C2 * id;                 O[7] = -(a * h - b * g) * id;   O[8] = (a * e - b * d) * id;
}

// row a of (Hpl_block Hlli): t[k] = sum_q h[a][q] Hlli[q][k]
__device__ __forceinline__ void row_times_inv(const float* h3, const float* hl, float t[3])
{
#pragma unroll
    for (int k = 0; k < 3; ++k) t[k] = h3[0] * hl[k] + h3[1] * hl[3 + k] + h3[2] * hl[6 + k];
}

__global__ void k_schur_pairs(const float* __restrict__ Hpl, const float* __restrict__ Hlli,
                              const int* __restrict__ okf, const int* __restrict__ olm, const int* __restrict__ pa,
                              const int* __restrict__ pb, float* __restrict__ Hred, long long npair, int d, int n)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= npair * d) return;
    const int a = (int)(idx % d);
    const long long p = idx / d;
    const int oi = pa[p], oj = pb[p];
    const int ki = okf[oi], kj = okf[oj];
    float t[3];
    row_times_inv(Hpl + (long long)oi * d * 3 + a * 3, Hlli + (long long)olm[oi] * 9, t);
    const float* hj = Hpl + (long long)oj * d * 3;
    float* row = Hred + (long long)(ki * d + a) * n + (long long)kj * d;
    for (int b = 0; b < d; ++b) atomicAdd(&row[b], -(t[0] * hj[b * 3] + t[1] * hj[b * 3 + 1] + t[2] * hj[b * 3 + 2]));
}

__global__ void k_schur_grad(const float* __restrict__ Hpl, const float* __restrict__ Hlli,
                             const float* __restrict__ bl, const int* __restrict__ okf, const int* __restrict__ olm,
                             float* __restrict__ g, int N, int d)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)N * d) return;
    const int a = (int)(idx % d);
    const int o = (int)(idx / d);
    const int l = olm[o];
    float t[3];
    row_times_inv(Hpl + (long long)o * d * 3 + a * 3, Hlli + (long long)l * 9, t);
    const float* bb = bl + (long long)l * 3;
    atomicAdd(&g[okf[o] * d + a], -(t[0] * bb[0] + t[1] * bb[1] + t[2] * bb[2]));
}

__global__ void k_pose_blocks(const float* __restrict__ Jp, const float* __restrict__ res,
                              const int* __restrict__ kf, float* __restrict__ Hred, float* __restrict__ g, int N,
                              int r, int d, int n)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)N * d) return;
    const int a = (int)(idx % d);
    const int o = (int)(idx / d);
    const int k = kf[o];
    if (k < 0) return;
    const float* J = Jp + (long long)o * r * d;
    float* row = Hred + (long long)(k * d + a) * n + (long long)k * d;
    for (int b = 0; b < d; ++b) {
        float acc = 0.f;
        for (int q = 0; q < r; ++q) acc += J[q * d + a] * J[q * d + b];
        atomicAdd(&row[b], acc);
    }
    float gg = 0.f;
    for (int q = 0; q < r; ++q) gg += J[q * d + a] * res[(long long)o * r + q];
    atomicAdd(&g[k * d + a], -gg);
}

// One CTA: in-place lower Cholesky (column by column) and the two triangular solves, column-oriented.
template <bool SMEM>
__global__ void k_chol_solve(float* __restrict__ Hg, const float* __restrict__ b, float* __restrict__ x, int n,
                             int* __restrict__ status)
{
    extern __shared__ float sH[];
    float* H = SMEM ? sH : Hg;
    const int tid = threadIdx.x, nt = blockDim.x;
    if (SMEM)
        for (long long q = tid; q < (long long)n * n; q += nt) sH[q] = Hg[q];
    if (tid == 0) *status = 0;
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        if (tid == 0) {
            float dkk = H[(long long)k * n + k];
            if (!(dkk > 0.f)) { *status = k + 1; dkk = 1e-8f; }
            H[(long long)k * n + k] = sqrtf(dkk);
        }
        __syncthreads();
        const float inv = 1.f / H[(long long)k * n + k];
        for (int i = k + 1 + tid; i < n; i += nt) H[(long long)i * n + k] *= inv;
        __syncthreads();
        // trailing update of the lower triangle: one warp per row
        for (int i = k + 1 + tid / 32; i < n; i += nt / 32) {
            const float lik = H[(long long)i * n + k];
            for (int j = k + 1 + (tid & 31); j <= i; j += 32) H[(long long)i * n + j] -= lik * H[(long long)j * n + k];
        }
        __syncthreads();
    }
    for (int i = tid; i < n; i += nt) x[i] = b[i];
    __syncthreads();
    for (int j = 0; j < n; ++j) {
        if (tid == 0) x[j] /= H[(long long)j * n + j];
        __syncthreads();
        const float xj = x[j];
        for (int i = j + 1 + tid; i < n; i += nt) x[i] -= H[(long long)i * n + j] * xj;
        __syncthreads();
    }
    for (int j = n - 1; j >= 0; --j) {
        if (tid == 0) x[j] /= H[(long long)j * n + j];
        __syncthreads();
        const float xj = x[j];
        for (int i = tid; i < j; i += nt) x[i] -= H[(long long)j * n + i] * xj;
        __syncthreads();
    }
    if (SMEM)
        for (long long q = tid; q < (long long)n * n; q += nt) Hg[q] = sH[q];
}

__global__ void k_backsub(const float* __restrict__ Hpl, const float* __restrict__ Hlli, const float* __restrict__ bl,
                          const float* __restrict__ dxp, const int* __restrict__ okf, const int* __restrict__ offs,
                          float* __restrict__ dxl, int nl, int d)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nl) return;
    float rhs[3] = {bl[3 * l], bl[3 * l + 1], bl[3 * l + 2]};
    for (int s = offs[l]; s < offs[l + 1]; ++s) {
        const float* h = Hpl + (long long)s * d * 3;
        const float* x = dxp + (long long)okf[s] * d;
        for (int a = 0; a < d; ++a)
#pragma unroll
            for (int c = 0; c < 3; ++c) rhs[c] -= h[a * 3 + c] * x[a];
    }
    const float* hl = Hlli + (long long)l * 9;
#pragma unroll
    for (int c = 0; c < 3; ++c) dxl[3 * l + c] = hl[c * 3] * rhs[0] + hl[c * 3 + 1] * rhs[1] + hl[c * 3 + 2] * rhs[2];
}

// -------------------------------------------------------------------------------------------- inverse-depth build
__global__ void __launch_bounds__(TPB) k_build_blocks_id(
    const float* __restrict__ Tcw, const float* __restrict__ hpose, const int* __restrict__ hidx,
    const float* __restrict__ mbear, const float* __restrict__ rhov, const int* __restrict__ okf,
    const int* __restrict__ olm, const float* __restrict__ ouv, float* __restrict__ Jp, float* __restrict__ resw,
    int* __restrict__ kslot, float* __restrict__ Hll, float* __restrict__ bl, float* __restrict__ Hpl, int N, float fx,
    float cx, float cy, float huber)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    float hv[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, bv[3] = {0.f, 0.f, 0.f};
    int l = -1;
    if (o < N) {
        const int k = okf[o];
        l = olm[o];
        const int hk = hidx[l];
        const float* T = Tcw + (long long)k * 12;
        // T_wc of the host: the in-window host inverted from its T_cw, else the carried constant
        float Hw[12];
        if (hk >= 0) {
            const float* C = Tcw + (long long)hk * 12;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
#pragma unroll
                for (int b = 0; b < 3; ++b) Hw[a * 4 + b] = C[b * 4 + a];
                Hw[a * 4 + 3] = -(C[a] * C[3] + C[4 + a] * C[7] + C[8 + a] * C[11]);
            }
        } else {
#pragma unroll
            for (int a = 0; a < 12; ++a) Hw[a] = hpose[(long long)l * 12 + a];
        }
        const float rho = rhov[l], irho = 1.f / rho;
        const float Ph[3] = {mbear[3 * (long long)l] * irho, mbear[3 * (long long)l + 1] * irho,
                             mbear[3 * (long long)l + 2] * irho};
        float Pw[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) Pw[a] = Hw[a * 4] * Ph[0] + Hw[a * 4 + 1] * Ph[1] + Hw[a * 4 + 2] * Ph[2] + Hw[a * 4 + 3];
        const float x = T[0] * Pw[0] + T[1] * Pw[1] + T[2] * Pw[2] + T[3];
        const float y = T[4] * Pw[0] + T[5] * Pw[1] + T[6] * Pw[2] + T[7];
        const float z = fmaxf(T[8] * Pw[0] + T[9] * Pw[1] + T[10] * Pw[2] + T[11], 1e-6f);
        const float iz = 1.f / z;
        const float ru = fx * x * iz + cx - ouv[2 * (long long)o];
        const float rv = fx * y * iz + cy - ouv[2 * (long long)o + 1];
        const float sw = huber_sw(sqrtf(ru * ru + rv * rv), huber);
        const float A[2][3] = {{fx * iz, 0.f, -fx * x * iz * iz}, {0.f, fx * iz, -fx * y * iz * iz}};
        float* jo = Jp + (long long)o * 24;
        // observer block: A [I | -hat(Pc)]
        float J[2][2][6];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            J[0][q][0] = A[q][0]; J[0][q][1] = A[q][1]; J[0][q][2] = A[q][2];
            J[0][q][3] = A[q][1] * (-z) + A[q][2] * y;
            J[0][q][4] = A[q][0] * z - A[q][2] * x;
            J[0][q][5] = -A[q][0] * y + A[q][1] * x;
        }
        // A R_cw_obs R_wc_host
        float ARch[2][3];
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                float v = 0.f;
#pragma unroll
                for (int m = 0; m < 3; ++m) {
                    const float rch = T[m * 4] * Hw[b] + T[m * 4 + 1] * Hw[4 + b] + T[m * 4 + 2] * Hw[8 + b];
                    v += A[q][m] * rch;
                }
                ARch[q][b] = v;
            }
        // host block: A R_ch [-I | +hat(Ph)]  (T_cw_host <- exp(d) T_cw_host)
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            if (hk >= 0) {
                J[1][q][0] = -ARch[q][0]; J[1][q][1] = -ARch[q][1]; J[1][q][2] = -ARch[q][2];
                J[1][q][3] = ARch[q][1] * Ph[2] - ARch[q][2] * Ph[1];
                J[1][q][4] = -ARch[q][0] * Ph[2] + ARch[q][2] * Ph[0];
                J[1][q][5] = ARch[q][0] * Ph[1] - ARch[q][1] * Ph[0];
            } else {
#pragma unroll
                for (int c = 0; c < 6; ++c) J[1][q][c] = 0.f;
            }
        }
#pragma unroll
        for (int s = 0; s < 2; ++s)
#pragma unroll
            for (int q = 0; q < 2; ++q)
#pragma unroll
                for (int c = 0; c < 6; ++c) {
                    J[s][q][c] *= sw;
                    jo[s * 12 + q * 6 + c] = J[s][q][c];
                }
        kslot[2 * (long long)o] = k;
        kslot[2 * (long long)o + 1] = hk;
        // landmark block (x_n, y_n, rho): d Ph / d(x_n, y_n) = e1, e2 / rho, d Ph / d rho = -Ph / rho
        float jl[2][3];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const float dr = ARch[q][0] * Ph[0] + ARch[q][1] * Ph[1] + ARch[q][2] * Ph[2];
            jl[q][0] = ARch[q][0] * irho * sw;
            jl[q][1] = ARch[q][1] * irho * sw;
            jl[q][2] = -dr * irho * sw;
        }
        const float rwu = ru * sw, rwv = rv * sw;
        resw[2 * (long long)o] = rwu;
        resw[2 * (long long)o + 1] = rwv;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
#pragma unroll
            for (int b = 0; b < 3; ++b) hv[a * 3 + b] = jl[0][a] * jl[0][b] + jl[1][a] * jl[1][b];
            bv[a] = -(jl[0][a] * rwu + jl[1][a] * rwv);
        }
        float* ho = Hpl + (long long)o * 36;
#pragma unroll
        for (int s = 0; s < 2; ++s)
#pragma unroll
            for (int a = 0; a < 6; ++a)
#pragma unroll
                for (int c = 0; c < 3; ++c) ho[s * 18 + a * 3 + c] = J[s][0][a] * jl[0][c] + J[s][1][a] * jl[1][c];
    }
    add_landmark_sums(hv, bv, l, Hll, bl);
}

__global__ void k_landmark_prior_id(const float* __restrict__ mb, const float* __restrict__ rhov,
                                    const float* __restrict__ m0, const float* __restrict__ rho0,
                                    const float* __restrict__ invsig, const float* __restrict__ wbear,
                                    const float* __restrict__ valid, float* __restrict__ Hll, float* __restrict__ bl,
                                    int nl, float huber)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nl || valid[l] < 0.5f) return;
    const float wb = wbear[l], is = invsig[l];
    const float r[3] = {(mb[3 * l] - m0[2 * l]) * wb, (mb[3 * l + 1] - m0[2 * l + 1]) * wb, (rhov[l] - rho0[l]) * is};
    const float J0[3] = {wb, wb, is};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        // the bearing rows are not robustified; the inverse-depth row is
        const float sw = a == 2 ? huber_sw(fabsf(r[a]), huber) : 1.f;
        const float J = J0[a] * sw;
        atomicAdd(&Hll[(long long)l * 9 + a * 4], J * J);
        atomicAdd(&bl[(long long)l * 3 + a], -J * r[a] * sw);
    }
}

__global__ void k_pose_blocks_id(const float* __restrict__ Jp, const float* __restrict__ res,
                                 const int* __restrict__ kslot, float* __restrict__ Hred, float* __restrict__ g,
                                 int N, int d, int n)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)N * d) return;
    const int a = (int)(idx % d);
    const int o = (int)(idx / d);
    const float r0 = res[2 * (long long)o], r1 = res[2 * (long long)o + 1];
    for (int sa = 0; sa < 2; ++sa) {
        const int ka = kslot[2 * (long long)o + sa];
        if (ka < 0) continue;
        const float* Ja = Jp + (long long)o * 4 * d + sa * 2 * d;
        for (int sb = 0; sb < 2; ++sb) {
            const int kb = kslot[2 * (long long)o + sb];
            if (kb < 0) continue;
            const float* Jb = Jp + (long long)o * 4 * d + sb * 2 * d;
            float* row = Hred + (long long)(ka * d + a) * n + (long long)kb * d;
            for (int b = 0; b < d; ++b) atomicAdd(&row[b], Ja[a] * Jb[b] + Ja[d + a] * Jb[d + b]);
        }
        atomicAdd(&g[ka * d + a], -(Ja[a] * r0 + Ja[d + a] * r1));
    }
}

__global__ void k_schur_pairs_id(const float* __restrict__ Hpl, const float* __restrict__ Hlli,
                                 const int* __restrict__ kslot, const int* __restrict__ olm,
                                 const int* __restrict__ pa, const int* __restrict__ pb, float* __restrict__ Hred,
                                 long long npair, int d, int n)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= npair * d) return;
    const int a = (int)(idx % d);
    const long long p = idx / d;
    const int oi = pa[p], oj = pb[p];
    const float* hl = Hlli + (long long)olm[oi] * 9;
    for (int si = 0; si < 2; ++si) {
        const int ki = kslot[2 * (long long)oi + si];
        if (ki < 0) continue;
        float t[3];
        row_times_inv(Hpl + (long long)oi * 6 * d + si * 3 * d + a * 3, hl, t);
        for (int sj = 0; sj < 2; ++sj) {
            const int kj = kslot[2 * (long long)oj + sj];
            if (kj < 0) continue;
            const float* hj = Hpl + (long long)oj * 6 * d + sj * 3 * d;
            float* row = Hred + (long long)(ki * d + a) * n + (long long)kj * d;
            for (int b = 0; b < d; ++b)
                atomicAdd(&row[b], -(t[0] * hj[b * 3] + t[1] * hj[b * 3 + 1] + t[2] * hj[b * 3 + 2]));
        }
    }
}

__global__ void k_schur_grad_id(const float* __restrict__ Hpl, const float* __restrict__ Hlli,
                                const float* __restrict__ bl, const int* __restrict__ kslot,
                                const int* __restrict__ olm, float* __restrict__ g, int N, int d)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)N * 2 * d) return;
    const int a = (int)(idx % d);
    const long long t2 = idx / d;
    const int s = (int)(t2 % 2);
    const int o = (int)(t2 / 2);
    const int k = kslot[2 * (long long)o + s];
    if (k < 0) return;
    const int l = olm[o];
    float t[3];
    row_times_inv(Hpl + (long long)o * 6 * d + s * 3 * d + a * 3, Hlli + (long long)l * 9, t);
    const float* bb = bl + (long long)l * 3;
    atomicAdd(&g[k * d + a], -(t[0] * bb[0] + t[1] * bb[1] + t[2] * bb[2]));
}

__global__ void k_backsub_id(const float* __restrict__ Hpl, const float* __restrict__ Hlli,
                             const float* __restrict__ bl, const float* __restrict__ dxp, const int* __restrict__ kslot,
                             const int* __restrict__ offs, float* __restrict__ dxl, int nl, int d)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nl) return;
    float rhs[3] = {bl[3 * l], bl[3 * l + 1], bl[3 * l + 2]};
    for (int s = offs[l]; s < offs[l + 1]; ++s)
        for (int sl = 0; sl < 2; ++sl) {
            const int k = kslot[2 * (long long)s + sl];
            if (k < 0) continue;
            const float* h = Hpl + (long long)s * 6 * d + sl * 3 * d;
            const float* x = dxp + (long long)k * d;
            for (int a = 0; a < d; ++a)
#pragma unroll
                for (int c = 0; c < 3; ++c) rhs[c] -= h[a * 3 + c] * x[a];
        }
    const float* hl = Hlli + (long long)l * 9;
#pragma unroll
    for (int c = 0; c < 3; ++c) dxl[3 * l + c] = hl[c * 3] * rhs[0] + hl[c * 3 + 1] * rhs[1] + hl[c * 3 + 2] * rhs[2];
}

int fail(int code, const std::string& m)
{
    xcb_set_last_error(m);
    return code;
}

int launched(const char* what)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(XCB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return XCB_OK;
}

#define BK_REQUIRE(cond, what)                                                                                        \
    do {                                                                                                              \
        if (!(cond)) return fail(XCB_ERR_ARG, std::string(what));                                                     \
    } while (0)

constexpr int CHOL_SMEM_MAX_N = 150;

}  // namespace

// -------------------------------------------------------------------------------------------------------- C ABI
extern "C" int xcb_bk_build_blocks(const float* Tcw, const float* pts, const int* okf, const int* olm,
                                   const float* ouv, float* Jpose, float* Jlm, float* resw, float* Hll, float* bl,
                                   float* Hpl, int N, float fx, float cx, float cy, float huber, void* stream)
{
    BK_REQUIRE(N >= 0, "build_blocks: N < 0");
    if (N == 0) return XCB_OK;
    BK_REQUIRE(Tcw && pts && okf && olm && ouv && Jpose && Jlm && resw && Hll && bl && Hpl, "build_blocks: null pointer");
    k_build_blocks<<<nblk(N), TPB, 0, (cudaStream_t)stream>>>(Tcw, pts, okf, olm, ouv, Jpose, Jlm, resw, Hll, bl, Hpl,
                                                               N, fx, cx, cy, huber);
    return launched("build_blocks");
}

extern "C" int xcb_bk_depth_prior(const float* pts, const float* chost, const float* rho0, const float* invsig,
                                  const float* valid, float* Hll, float* bl, int nl, float huber, void* stream)
{
    BK_REQUIRE(nl >= 0, "depth_prior: nl < 0");
    if (nl == 0) return XCB_OK;
    BK_REQUIRE(pts && chost && rho0 && invsig && valid && Hll && bl, "depth_prior: null pointer");
    k_depth_prior<<<nblk(nl), TPB, 0, (cudaStream_t)stream>>>(pts, chost, rho0, invsig, valid, Hll, bl, nl, huber);
    return launched("depth_prior");
}

extern "C" int xcb_bk_inv3_damped(const float* Hll, float* Hlli, int nl, float lam, void* stream)
{
    BK_REQUIRE(nl >= 0, "inv3_damped: nl < 0");
    if (nl == 0) return XCB_OK;
    BK_REQUIRE(Hll && Hlli, "inv3_damped: null pointer");
    k_inv3_damped<<<nblk(nl), TPB, 0, (cudaStream_t)stream>>>(Hll, Hlli, nl, lam);
    return launched("inv3_damped");
}

extern "C" int xcb_bk_schur_pairs(const float* Hpl, const float* Hlli, const int* okf, const int* olm, const int* pa,
                                  const int* pb, float* Hred, long long npair, int d, int n, void* stream)
{
    BK_REQUIRE(npair >= 0 && d > 0 && n > 0, "schur_pairs: bad size");
    if (npair == 0) return XCB_OK;
    BK_REQUIRE(Hpl && Hlli && okf && olm && pa && pb && Hred, "schur_pairs: null pointer");
    k_schur_pairs<<<nblk(npair * d), TPB, 0, (cudaStream_t)stream>>>(Hpl, Hlli, okf, olm, pa, pb, Hred, npair, d, n);
    return launched("schur_pairs");
}

extern "C" int xcb_bk_schur_grad(const float* Hpl, const float* Hlli, const float* bl, const int* okf, const int* olm,
                                 float* g, int N, int d, void* stream)
{
    BK_REQUIRE(N >= 0 && d > 0, "schur_grad: bad size");
    if (N == 0) return XCB_OK;
    BK_REQUIRE(Hpl && Hlli && bl && okf && olm && g, "schur_grad: null pointer");
    k_schur_grad<<<nblk((long long)N * d), TPB, 0, (cudaStream_t)stream>>>(Hpl, Hlli, bl, okf, olm, g, N, d);
    return launched("schur_grad");
}

extern "C" int xcb_bk_pose_blocks(const float* Jp, const float* res, const int* kf, float* Hred, float* g, int N,
                                  int r, int d, int n, void* stream)
{
    BK_REQUIRE(N >= 0 && r > 0 && d > 0 && n > 0, "pose_blocks: bad size");
    if (N == 0) return XCB_OK;
    BK_REQUIRE(Jp && res && kf && Hred && g, "pose_blocks: null pointer");
    k_pose_blocks<<<nblk((long long)N * d), TPB, 0, (cudaStream_t)stream>>>(Jp, res, kf, Hred, g, N, r, d, n);
    return launched("pose_blocks");
}

extern "C" int xcb_bk_chol_solve(float* H, const float* b, float* x, int n, int* status, int nthreads, void* stream)
{
    BK_REQUIRE(n > 0 && n <= 1024, "chol_solve: n out of range (1..1024)");
    BK_REQUIRE(H && b && x && status, "chol_solve: null pointer");
    if (nthreads <= 0) nthreads = 256;
    nthreads = ((nthreads + 31) / 32) * 32;
    if (nthreads > 1024) nthreads = 1024;
    if (n <= CHOL_SMEM_MAX_N) {
        const size_t sm = (size_t)n * n * sizeof(float);
        static XcbAttrOnce attr;
        const cudaError_t e = xcb_smem_attr_once(attr, (const void*)k_chol_solve<true>,
                                                 (int)(CHOL_SMEM_MAX_N * CHOL_SMEM_MAX_N * sizeof(float)));
        if (e != cudaSuccess) return fail(XCB_ERR_CUDA, std::string("chol_solve: ") + cudaGetErrorString(e));
        k_chol_solve<true><<<1, nthreads, sm, (cudaStream_t)stream>>>(H, b, x, n, status);
    } else {
        k_chol_solve<false><<<1, nthreads, 0, (cudaStream_t)stream>>>(H, b, x, n, status);
    }
    return launched("chol_solve");
}

extern "C" int xcb_bk_backsub(const float* Hpl, const float* Hlli, const float* bl, const float* dxp, const int* okf,
                              const int* offs, float* dxl, int nl, int d, void* stream)
{
    BK_REQUIRE(nl >= 0 && d > 0, "backsub: bad size");
    if (nl == 0) return XCB_OK;
    BK_REQUIRE(Hpl && Hlli && bl && dxp && okf && offs && dxl, "backsub: null pointer");
    k_backsub<<<nblk(nl), TPB, 0, (cudaStream_t)stream>>>(Hpl, Hlli, bl, dxp, okf, offs, dxl, nl, d);
    return launched("backsub");
}

extern "C" int xcb_bk_build_blocks_id(const float* Tcw, const float* hpose, const int* hidx, const float* mbear,
                                      const float* rhov, const int* okf, const int* olm, const float* ouv, float* Jp,
                                      float* resw, int* kslot, float* Hll, float* bl, float* Hpl, int N, float fx,
                                      float cx, float cy, float huber, void* stream)
{
    BK_REQUIRE(N >= 0, "build_blocks_id: N < 0");
    if (N == 0) return XCB_OK;
    BK_REQUIRE(Tcw && hpose && hidx && mbear && rhov && okf && olm && ouv && Jp && resw && kslot && Hll && bl && Hpl,
               "build_blocks_id: null pointer");
    k_build_blocks_id<<<nblk(N), TPB, 0, (cudaStream_t)stream>>>(Tcw, hpose, hidx, mbear, rhov, okf, olm, ouv, Jp,
                                                                  resw, kslot, Hll, bl, Hpl, N, fx, cx, cy, huber);
    return launched("build_blocks_id");
}

extern "C" int xcb_bk_landmark_prior_id(const float* mb, const float* rhov, const float* m0, const float* rho0,
                                        const float* invsig, const float* wbear, const float* valid, float* Hll,
                                        float* bl, int nl, float huber, void* stream)
{
    BK_REQUIRE(nl >= 0, "landmark_prior_id: nl < 0");
    if (nl == 0) return XCB_OK;
    BK_REQUIRE(mb && rhov && m0 && rho0 && invsig && wbear && valid && Hll && bl, "landmark_prior_id: null pointer");
    k_landmark_prior_id<<<nblk(nl), TPB, 0, (cudaStream_t)stream>>>(mb, rhov, m0, rho0, invsig, wbear, valid, Hll, bl,
                                                                     nl, huber);
    return launched("landmark_prior_id");
}

extern "C" int xcb_bk_pose_blocks_id(const float* Jp, const float* res, const int* kslot, float* Hred, float* g,
                                     int N, int d, int n, void* stream)
{
    BK_REQUIRE(N >= 0 && d > 0 && n > 0, "pose_blocks_id: bad size");
    if (N == 0) return XCB_OK;
    BK_REQUIRE(Jp && res && kslot && Hred && g, "pose_blocks_id: null pointer");
    k_pose_blocks_id<<<nblk((long long)N * d), TPB, 0, (cudaStream_t)stream>>>(Jp, res, kslot, Hred, g, N, d, n);
    return launched("pose_blocks_id");
}

extern "C" int xcb_bk_schur_pairs_id(const float* Hpl, const float* Hlli, const int* kslot, const int* olm,
                                     const int* pa, const int* pb, float* Hred, long long npair, int d, int n,
                                     void* stream)
{
    BK_REQUIRE(npair >= 0 && d > 0 && n > 0, "schur_pairs_id: bad size");
    if (npair == 0) return XCB_OK;
    BK_REQUIRE(Hpl && Hlli && kslot && olm && pa && pb && Hred, "schur_pairs_id: null pointer");
    k_schur_pairs_id<<<nblk(npair * d), TPB, 0, (cudaStream_t)stream>>>(Hpl, Hlli, kslot, olm, pa, pb, Hred, npair, d,
                                                                         n);
    return launched("schur_pairs_id");
}

extern "C" int xcb_bk_schur_grad_id(const float* Hpl, const float* Hlli, const float* bl, const int* kslot,
                                    const int* olm, float* g, int N, int d, void* stream)
{
    BK_REQUIRE(N >= 0 && d > 0, "schur_grad_id: bad size");
    if (N == 0) return XCB_OK;
    BK_REQUIRE(Hpl && Hlli && bl && kslot && olm && g, "schur_grad_id: null pointer");
    k_schur_grad_id<<<nblk((long long)N * 2 * d), TPB, 0, (cudaStream_t)stream>>>(Hpl, Hlli, bl, kslot, olm, g, N, d);
    return launched("schur_grad_id");
}

extern "C" int xcb_bk_backsub_id(const float* Hpl, const float* Hlli, const float* bl, const float* dxp,
                                 const int* kslot, const int* offs, float* dxl, int nl, int d, void* stream)
{
    BK_REQUIRE(nl >= 0 && d > 0, "backsub_id: bad size");
    if (nl == 0) return XCB_OK;
    BK_REQUIRE(Hpl && Hlli && bl && dxp && kslot && offs && dxl, "backsub_id: null pointer");
    k_backsub_id<<<nblk(nl), TPB, 0, (cudaStream_t)stream>>>(Hpl, Hlli, bl, dxp, kslot, offs, dxl, nl, d);
    return launched("backsub_id");
}
