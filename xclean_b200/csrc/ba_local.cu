// ba_local.cu -- the local-BA LM loop of src/xclean/backend/ba.py (_solve_gpu, ba.py:930-1089; _solve_gpu_id,
// ba.py:1345-1497) with every decision on the device (sm_100a).
//
// The reference runs each LM iteration as ~10 launches plus three host round trips (chi, the step and the landmark
// step are copied back; the accept test and the SE(3) update run in numpy).  Here the host only enqueues: a control
// kernel takes the accept / reject decision from the device-side chi and restores or saves the float64 state, the
// later kernels of a rejected iteration see the flag and return at once, and the pose update (exp(xi) T) and the
// non-finite guard run on the device.  One wait at the end.
//
// Per iteration (one stream):
//   prep      float64 state -> the float32 inputs of the build; clear the accumulators
//   build     xcb_bk_build_blocks[_id] (+ the prior kernel): float32 Jacobians, Hll, bl, Hpl (the reference's stage)
//   ctl       chi = sum resw^2 (float64, fixed order); LM accept / reject; state save / restore
//   schur     one warp per landmark: damped 3x3 inverse (float64), the landmark's distinct keyframes, their summed Hpl
//             blocks U, then the pose-pose blocks, -U Hll^-1 U^T and the gradient added once per entry of the lower
//             triangle (float64 atomics) instead of once per ordered observation pair
//   rot       gyro relative-rotation factors (ba.py _rot_factor_blocks), float64
//   solve     one CTA: held keyframes, damping, Cholesky of the reduced system in shared memory (packed lower, float64)
//   backsub   one thread per landmark, float64; the non-finite guard
//   apply     T_cw <- exp(xi) T_cw for free keyframes, landmark update, lam
// After the loop: rotation projection onto SO(3) (polar iteration), one more build, final chi.
#include <algorithm>
#include <string>

#include "common.cuh"

extern void xcb_set_last_error(const std::string& m);

namespace {

constexpr int SCHUR_WARPS = 4;
constexpr int MAXT = XCB_LBA_MAX_TOUCHED;
constexpr int SOLVE_THREADS = 1024;
constexpr int SOLVE_SMEM_MAX_N = 216;          // packed lower float64: 216 * 217 / 2 * 8 = 187,488 bytes

struct LbaCtl {
    double lam, chi_prev, chi_best, rms0;
    int have_prev, have_best, have_rms0, skip, nonfinite, accepted, rejected, nonfin_steps, overflow;
};

struct LbaK {
    int model, so, nk, nl, N, n, nrot;
    double fx, cx, cy, huber, rho_floor;
    double* Tcw;
    double* lm;
    double* rho;
    const int* okf;
    const int* olm;
    const int* offs;
    const unsigned char* freem;
    const int* rot_a;
    const int* rot_b;
    const double* rot_M;
    const double* rot_sig;
    // workspace
    float* Tcw32;
    float* lm32;
    float* rho32;
    float* Jp;
    float* resw;
    float* Hll;
    float* bl;
    float* Hpl;
    const int* slot;      // (N, so): okf (Euclidean) or kslot (inverse depth)
    double* S;
    double* g;
    double* dxp;
    double* dxl;
    double* Hi;
    double* bestT;
    double* bestL;
    double* bestR;
    LbaCtl* ctl;
};

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// block-wide float64 sum, fixed order (every thread gets the result)
__device__ double block_sum(double v)
{
    __shared__ double red[32];
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
    return s;
}

// ------------------------------------------------------------------------------------------------- SO(3) / SE(3)
// Rodrigues coefficients with their Taylor series near zero (sin t / t, (1 - cos t) / t^2, (t - sin t) / t^3)
__device__ __forceinline__ void so3_coeffs(double t2, double* a, double* b, double* c)
{
    if (t2 < 0.0158) {        // t < 0.126: the 4-term series is at rounding level there
        *a = 1.0 - t2 / 6.0 + t2 * t2 / 120.0 - t2 * t2 * t2 / 5040.0;
        *b = 0.5 - t2 / 24.0 + t2 * t2 / 720.0 - t2 * t2 * t2 / 40320.0;
        *c = 1.0 / 6.0 - t2 / 120.0 + t2 * t2 / 5040.0 - t2 * t2 * t2 / 362880.0;
    } else {
        const double t = sqrt(t2), s = sin(t), co = cos(t);
        *a = s / t;
        *b = (1.0 - co) / t2;
        *c = (t - s) / (t2 * t);
    }
}

__device__ __forceinline__ void hat3(const double* v, double* K)
{
    K[0] = 0.0;   K[1] = -v[2]; K[2] = v[1];
    K[3] = v[2];  K[4] = 0.0;   K[5] = -v[0];
    K[6] = -v[1]; K[7] = v[0];  K[8] = 0.0;
}

__device__ __forceinline__ void mm3(const double* A, const double* B, double* C)
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C[i * 3 + j] = A[i * 3] * B[j] + A[i * 3 + 1] * B[3 + j] + A[i * 3 + 2] * B[6 + j];
}

// T (3x4 rows) <- exp(xi) T, xi = [rho (translation), phi (rotation)]
__device__ void se3_left_update(const double* xi, double* T)
{
    const double* r = xi;
    const double* p = xi + 3;
    const double t2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
    double a, b, c, K[9], KK[9], R[9], V[9];
    so3_coeffs(t2, &a, &b, &c);
    hat3(p, K);
    mm3(K, K, KK);
    for (int i = 0; i < 9; ++i) {
        const double I = (i % 4 == 0) ? 1.0 : 0.0;
        R[i] = I + a * K[i] + b * KK[i];
        V[i] = I + b * K[i] + c * KK[i];
    }
    double t[3];
    for (int i = 0; i < 3; ++i) t[i] = V[i * 3] * r[0] + V[i * 3 + 1] * r[1] + V[i * 3 + 2] * r[2];
    double out[12];
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 4; ++j) out[i * 4 + j] = R[i * 3] * T[j] + R[i * 3 + 1] * T[4 + j] + R[i * 3 + 2] * T[8 + j];
        out[i * 4 + 3] += t[i];
    }
    for (int i = 0; i < 12; ++i) T[i] = out[i];
}

// log of a rotation through its unit quaternion (Shepperd's branch on the largest of trace and the diagonal;
// w >= 0), so that angles near pi keep their digits
__device__ void so3_log(const double* R, double* w)
{
    const double m00 = R[0], m11 = R[4], m22 = R[8], tr = m00 + m11 + m22;
    double q[4];
    if (tr > 0.0) {
        const double t = sqrt(fmax(tr + 1.0, 0.0)) * 2.0;
        q[0] = 0.25 * t;
        q[1] = (R[7] - R[5]) / t;
        q[2] = (R[2] - R[6]) / t;
        q[3] = (R[3] - R[1]) / t;
    } else {
        int a = 0;
        if (m11 > m00 && m11 >= m22) a = 1;
        else if (m22 > m00 && m22 > m11) a = 2;
        const int c = (a + 1) % 3, d = (a + 2) % 3;
        const double t = sqrt(fmax(1.0 + R[a * 4] - R[c * 4] - R[d * 4], 0.0)) * 2.0;
        q[0] = (R[d * 3 + c] - R[c * 3 + d]) / t;
        q[1 + a] = 0.25 * t;
        q[1 + c] = (R[c * 3 + a] + R[a * 3 + c]) / t;
        q[1 + d] = (R[d * 3 + a] + R[a * 3 + d]) / t;
    }
    if (q[0] < 0.0)
        for (int i = 0; i < 4; ++i) q[i] = -q[i];
    const double nv = sqrt(q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    const double th = 2.0 * atan2(nv, q[0]);
    const double s = nv < 3.65e-8 ? 2.0 : th / nv;
    for (int i = 0; i < 3; ++i) w[i] = q[1 + i] * s;
}

// inverse right Jacobian of SO(3) at e: I + 1/2 hat(e) + k hat(e)^2, k = (1 - t sin t / (2 (1 - cos t))) / t^2
__device__ void so3_jr_inv(const double* e, double* J)
{
    const double t2 = e[0] * e[0] + e[1] * e[1] + e[2] * e[2];
    double k;
    if (t2 < 0.0158) k = 1.0 / 12.0 + t2 / 720.0 + t2 * t2 / 30240.0 + t2 * t2 * t2 / 1209600.0;
    else {
        const double t = sqrt(t2);
        k = (1.0 - t * sin(t) / (2.0 * (1.0 - cos(t)))) / t2;
    }
    double K[9], KK[9];
    hat3(e, K);
    mm3(K, K, KK);
    for (int i = 0; i < 9; ++i) J[i] = ((i % 4 == 0) ? 1.0 : 0.0) + 0.5 * K[i] + k * KK[i];
}

// ---------------------------------------------------------------------------------------------------- kernels
__global__ void k_lba_init(LbaK P, double lam0)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    LbaCtl& c = *P.ctl;
    c.lam = lam0;
    c.chi_prev = c.chi_best = c.rms0 = 0.0;
    c.have_prev = c.have_best = c.have_rms0 = c.skip = c.nonfinite = 0;
    c.accepted = c.rejected = c.nonfin_steps = c.overflow = 0;
}

__global__ void k_lba_prep(LbaK P)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (long long i = t0; i < (long long)P.nk * 12; i += stride) P.Tcw32[i] = (float)P.Tcw[i];
    for (long long i = t0; i < (long long)P.nl * 3; i += stride) {
        P.lm32[i] = (float)P.lm[i];
        P.bl[i] = 0.f;
    }
    if (P.model == XCB_LBA_INVDEPTH)
        for (long long i = t0; i < P.nl; i += stride) P.rho32[i] = (float)P.rho[i];
    for (long long i = t0; i < (long long)P.nl * 9; i += stride) P.Hll[i] = 0.f;
    for (long long i = t0; i < (long long)P.n * P.n; i += stride) P.S[i] = 0.0;
    for (long long i = t0; i < P.n; i += stride) P.g[i] = 0.0;
}

// chi and the LM decision of the reference's loop head: a chi above the previous accepted one restores the best
// state and multiplies lam by 4 (the rest of the iteration is skipped); otherwise the state becomes the best one.
__global__ void k_lba_ctl(LbaK P)
{
    __shared__ int s_rej;
    LbaCtl& c = *P.ctl;
    double acc = 0.0;
    for (long long i = threadIdx.x; i < 2LL * P.N; i += blockDim.x) acc += (double)P.resw[i] * (double)P.resw[i];
    const double chi = block_sum(acc);
    if (threadIdx.x == 0) {
        c.nonfinite = 0;
        if (!c.have_rms0) {
            c.rms0 = sqrt(chi / (double)(P.N > 0 ? P.N : 1));
            c.have_rms0 = 1;
        }
        const int rej = c.have_prev && chi > c.chi_prev;
        if (rej) {
            c.lam = fmin(c.lam * 4.0, 1e2);
            c.rejected += 1;
        } else {
            c.chi_prev = chi;
            c.have_prev = 1;
            c.chi_best = chi;
            c.have_best = 1;
        }
        c.skip = rej;
        s_rej = rej;
    }
    __syncthreads();
    const int rej = s_rej;
    double* a = rej ? P.Tcw : P.bestT;
    const double* b = rej ? P.bestT : P.Tcw;
    for (int i = threadIdx.x; i < P.nk * 12; i += blockDim.x) a[i] = b[i];
    double* la = rej ? P.lm : P.bestL;
    const double* lb = rej ? P.bestL : P.lm;
    for (long long i = threadIdx.x; i < 3LL * P.nl; i += blockDim.x) la[i] = lb[i];
    if (P.model == XCB_LBA_INVDEPTH) {
        double* ra = rej ? P.rho : P.bestR;
        const double* rb = rej ? P.bestR : P.rho;
        for (long long i = threadIdx.x; i < P.nl; i += blockDim.x) ra[i] = rb[i];
    }
}

struct SchurWarp {
    int ts[MAXT];
    double U[MAXT][18];     // summed Hpl blocks per distinct keyframe (6 x 3)
    double T[MAXT][18];     // Hll^-1 U^T (3 x 6)
};

__device__ __forceinline__ int tri_root(int pr)
{
    int a = (int)((sqrtf(8.0f * pr + 1.0f) - 1.0f) * 0.5f);
    while (a * (a + 1) / 2 > pr) --a;
    while ((a + 1) * (a + 2) / 2 <= pr) ++a;
    return a;
}

template <int SO>
__global__ void __launch_bounds__(SCHUR_WARPS * 32) k_lba_schur(LbaK P)
{
    __shared__ SchurWarp sw[SCHUR_WARPS];
    if (P.ctl->skip) return;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    SchurWarp& W = sw[wid];
    const double lam = P.ctl->lam;
    const int n = P.n;
    for (int l = blockIdx.x * SCHUR_WARPS + wid; l < P.nl; l += gridDim.x * SCHUR_WARPS) {
        const int o0 = P.offs[l], nobs = P.offs[l + 1] - o0;
        const int e0 = o0 * SO, nE = nobs * SO;
        // distinct keyframes of the landmark
        unsigned long long m = 0;
        for (int e = lane; e < nE; e += 32) {
            const int s = P.slot[e0 + e];
            if (s >= 0) m |= 1ull << s;
        }
        const unsigned lo = __reduce_or_sync(0xffffffffu, (unsigned)m);
        const unsigned hi = __reduce_or_sync(0xffffffffu, (unsigned)(m >> 32));
        m = ((unsigned long long)hi << 32) | lo;
        int nt = __popcll(m);
        if (nt > MAXT) {
            if (lane == 0) atomicAdd(&P.ctl->overflow, 1);
            nt = MAXT;
        }
        for (int a = lane; a < 64; a += 32)
            if ((m >> a) & 1ull) {
                const int r = __popcll(m & ((1ull << a) - 1ull));
                if (r < MAXT) W.ts[r] = a;
            }
        // damped landmark block and its inverse, float64 (the damping of kernels.inv3_damped)
        double H[9];
        for (int i = 0; i < 9; ++i) H[i] = (double)P.Hll[(long long)l * 9 + i];
        const double dmp = lam * fmax((H[0] + H[4] + H[8]) / 3.0, 1e-9);
        H[0] += dmp; H[4] += dmp; H[8] += dmp;
        const double C0 = H[4] * H[8] - H[5] * H[7], C1 = -(H[3] * H[8] - H[5] * H[6]), C2 = H[3] * H[7] - H[4] * H[6];
        double det = H[0] * C0 + H[1] * C1 + H[2] * C2;
        if (fabs(det) < 1e-30) det = det < 0.0 ? -1e-30 : 1e-30;
        const double id = 1.0 / det;
        const double Hi[9] = {C0 * id, -(H[1] * H[8] - H[2] * H[7]) * id, (H[1] * H[5] - H[2] * H[4]) * id,
                              C1 * id, (H[0] * H[8] - H[2] * H[6]) * id, -(H[0] * H[5] - H[2] * H[3]) * id,
                              C2 * id, -(H[0] * H[7] - H[1] * H[6]) * id, (H[0] * H[4] - H[1] * H[3]) * id};
        if (lane < 9) P.Hi[(long long)l * 9 + lane] = Hi[lane];
        const double b0 = P.bl[3 * (long long)l], b1 = P.bl[3 * (long long)l + 1], b2 = P.bl[3 * (long long)l + 2];
        const double HiB[3] = {Hi[0] * b0 + Hi[1] * b1 + Hi[2] * b2, Hi[3] * b0 + Hi[4] * b1 + Hi[5] * b2,
                               Hi[6] * b0 + Hi[7] * b1 + Hi[8] * b2};
        __syncwarp();
        // U[a] = sum of the Hpl blocks of the entries on keyframe ts[a]
        for (int it = lane; it < nt * 18; it += 32) {
            const int a = it / 18, q = it % 18, s = W.ts[a];
            double acc = 0.0;
            for (int e = 0; e < nE; ++e)
                if (P.slot[e0 + e] == s) acc += (double)P.Hpl[(long long)(e0 + e) * 18 + q];
            W.U[a][q] = acc;
        }
        __syncwarp();
        for (int it = lane; it < nt * 18; it += 32) {
            const int a = it / 18, r = it % 18, k = r / 6, j = r % 6;
            W.T[a][r] = Hi[k * 3] * W.U[a][j * 3] + Hi[k * 3 + 1] * W.U[a][j * 3 + 1] + Hi[k * 3 + 2] * W.U[a][j * 3 + 2];
        }
        __syncwarp();
        // gradient: -sum J^T rw - U Hll^-1 bl
        for (int it = lane; it < nt * 6; it += 32) {
            const int a = it / 6, i = it % 6, s = W.ts[a];
            double acc = 0.0;
            for (int e = 0; e < nE; ++e)
                if (P.slot[e0 + e] == s) {
                    const float* J = P.Jp + (long long)(e0 + e) * 12;
                    const long long o = o0 + e / SO;
                    acc -= (double)J[i] * (double)P.resw[2 * o] + (double)J[6 + i] * (double)P.resw[2 * o + 1];
                }
            acc -= W.U[a][i * 3] * HiB[0] + W.U[a][i * 3 + 1] * HiB[1] + W.U[a][i * 3 + 2] * HiB[2];
            atomicAdd(&P.g[s * 6 + i], acc);
        }
        // reduced system, lower triangle: keyframe pairs (ts[a], ts[b]), a >= b
        const int npair = nt * (nt + 1) / 2;
        for (int it = lane; it < npair * 36; it += 32) {
            const int pr = it / 36, r = it % 36, i = r / 6, j = r % 6;
            const int a = tri_root(pr), b = pr - a * (a + 1) / 2;
            if (a == b && j > i) continue;
            const int sa = W.ts[a], sb = W.ts[b];
            double acc = 0.0;
            for (int o = 0; o < nobs; ++o)
#pragma unroll
                for (int s1 = 0; s1 < SO; ++s1) {
                    if (P.slot[e0 + o * SO + s1] != sa) continue;
                    const float* Ja = P.Jp + (long long)(e0 + o * SO + s1) * 12;
#pragma unroll
                    for (int s2 = 0; s2 < SO; ++s2) {
                        if (P.slot[e0 + o * SO + s2] != sb) continue;
                        const float* Jb = P.Jp + (long long)(e0 + o * SO + s2) * 12;
                        acc += (double)Ja[i] * (double)Jb[j] + (double)Ja[6 + i] * (double)Jb[6 + j];
                    }
                }
            acc -= W.U[a][i * 3] * W.T[b][j] + W.U[a][i * 3 + 1] * W.T[b][6 + j] + W.U[a][i * 3 + 2] * W.T[b][12 + j];
            atomicAdd(&P.S[(long long)(sa * 6 + i) * n + sb * 6 + j], acc);
        }
        __syncwarp();
    }
}

// gyro relative-rotation factors: e = log(M^T R_a R_b^T), Jacobians Jr^-1(e) R_a R_b^T and -Jr^-1(e), weight 1/sigma
__global__ void k_lba_rot(LbaK P)
{
    if (P.ctl->skip) return;
    for (int f = threadIdx.x; f < P.nrot; f += blockDim.x) {
        const int a = P.rot_a[f], b = P.rot_b[f];
        if (a < 0 || b < 0 || a >= P.nk || b >= P.nk) continue;
        const double w = 1.0 / fmax(P.rot_sig[f], 1e-9);
        double Ra[9], Rb[9], A[9], E[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                Ra[i * 3 + j] = P.Tcw[a * 12 + i * 4 + j];
                Rb[i * 3 + j] = P.Tcw[b * 12 + i * 4 + j];
            }
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                A[i * 3 + j] = Ra[i * 3] * Rb[j * 3] + Ra[i * 3 + 1] * Rb[j * 3 + 1] + Ra[i * 3 + 2] * Rb[j * 3 + 2];
        const double* M = P.rot_M + (long long)f * 9;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) E[i * 3 + j] = M[i] * A[j] + M[3 + i] * A[3 + j] + M[6 + i] * A[6 + j];
        double e[3], Jr[9], Ja[9], Jb[9];
        so3_log(E, e);
        so3_jr_inv(e, Jr);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                Ja[i * 3 + j] = w * (Jr[i * 3] * A[j * 3] + Jr[i * 3 + 1] * A[j * 3 + 1] + Jr[i * 3 + 2] * A[j * 3 + 2]);
                Jb[i * 3 + j] = -w * Jr[i * 3 + j];
            }
        const double r[3] = {w * e[0], w * e[1], w * e[2]};
        const int base[2] = {a * 6 + 3, b * 6 + 3};
        const double* Jx[2] = {Ja, Jb};
        for (int p = 0; p < 2; ++p) {
            for (int i = 0; i < 3; ++i) {
                double gg = 0.0;
                for (int k = 0; k < 3; ++k) gg += Jx[p][k * 3 + i] * r[k];
                atomicAdd(&P.g[base[p] + i], -gg);
            }
            for (int q = 0; q < 2; ++q)
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) {
                        const int row = base[p] + i, col = base[q] + j;
                        if (row < col) continue;         // the lower triangle carries the symmetric sum
                        double h = 0.0;
                        for (int k = 0; k < 3; ++k) h += Jx[p][k * 3 + i] * Jx[q][k * 3 + j];
                        atomicAdd(&P.S[(long long)row * P.n + col], h);
                    }
        }
    }
}

template <bool SMEM>
__device__ __forceinline__ double& Sel(double* L, int n, int i, int j)
{
    return SMEM ? L[(long long)i * (i + 1) / 2 + j] : L[(long long)i * n + j];
}

// one CTA: held keyframes, damping, Cholesky (float64; a non-positive pivot is replaced by 1e-8 as the reference
// does), the two triangular solves -> dxp, and the finite check of the step
template <bool SMEM>
__global__ void __launch_bounds__(SOLVE_THREADS) k_lba_solve(LbaK P)
{
    extern __shared__ double sL[];
    if (P.ctl->skip) return;
    const int n = P.n, tid = threadIdx.x, nt = blockDim.x;
    const double lam = P.ctl->lam;
    double* L = SMEM ? sL : P.S;
    for (long long q = tid; q < (long long)n * n; q += nt) {
        const int r = (int)(q / n), c = (int)(q % n);
        if (c > r) continue;
        double v = P.S[q];
        if (!P.freem[r / 6] || !P.freem[c / 6]) v = (r == c) ? 1.0 : 0.0;
        if (r == c) v += lam * fmax(v, 1e-9);
        Sel<SMEM>(L, n, r, c) = v;
    }
    for (int i = tid; i < n; i += nt) P.dxp[i] = P.freem[i / 6] ? P.g[i] : 0.0;
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        if (tid == 0) {
            double dkk = Sel<SMEM>(L, n, k, k);
            if (!(dkk > 0.0)) dkk = 1e-8;
            Sel<SMEM>(L, n, k, k) = sqrt(dkk);
        }
        __syncthreads();
        const double inv = 1.0 / Sel<SMEM>(L, n, k, k);
        for (int i = k + 1 + tid; i < n; i += nt) Sel<SMEM>(L, n, i, k) *= inv;
        __syncthreads();
        for (int i = k + 1 + tid / 32; i < n; i += nt / 32) {
            const double lik = Sel<SMEM>(L, n, i, k);
            for (int j = k + 1 + (tid & 31); j <= i; j += 32) Sel<SMEM>(L, n, i, j) -= lik * Sel<SMEM>(L, n, j, k);
        }
        __syncthreads();
    }
    double* x = P.dxp;
    for (int j = 0; j < n; ++j) {
        if (tid == 0) x[j] /= Sel<SMEM>(L, n, j, j);
        __syncthreads();
        const double xj = x[j];
        for (int i = j + 1 + tid; i < n; i += nt) x[i] -= Sel<SMEM>(L, n, i, j) * xj;
        __syncthreads();
    }
    for (int j = n - 1; j >= 0; --j) {
        if (tid == 0) x[j] /= Sel<SMEM>(L, n, j, j);
        __syncthreads();
        const double xj = x[j];
        for (int i = tid; i < j; i += nt) x[i] -= Sel<SMEM>(L, n, j, i) * xj;
        __syncthreads();
    }
    int bad = 0;
    for (int i = tid; i < n; i += nt) bad |= !isfinite(x[i]);
    if (__syncthreads_or(bad) && tid == 0) P.ctl->nonfinite = 1;
}

template <int SO>
__global__ void k_lba_backsub(LbaK P)
{
    if (P.ctl->skip) return;
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= P.nl) return;
    double rhs[3] = {(double)P.bl[3 * (long long)l], (double)P.bl[3 * (long long)l + 1],
                     (double)P.bl[3 * (long long)l + 2]};
    const int e0 = P.offs[l] * SO, e1 = P.offs[l + 1] * SO;
    for (int e = e0; e < e1; ++e) {
        const int s = P.slot[e];
        if (s < 0) continue;
        const float* h = P.Hpl + (long long)e * 18;
        const double* x = P.dxp + s * 6;
        for (int a = 0; a < 6; ++a)
            for (int c = 0; c < 3; ++c) rhs[c] -= (double)h[a * 3 + c] * x[a];
    }
    const double* Hi = P.Hi + (long long)l * 9;
    bool bad = false;
    for (int c = 0; c < 3; ++c) {
        const double v = Hi[c * 3] * rhs[0] + Hi[c * 3 + 1] * rhs[1] + Hi[c * 3 + 2] * rhs[2];
        P.dxl[3 * (long long)l + c] = v;
        bad |= !isfinite(v);
    }
    if (bad) atomicOr(&P.ctl->nonfinite, 1);
}

// a finite step is applied (T_cw <- exp(xi) T_cw for free keyframes, landmarks += step, rho floored) and lam halves;
// a non-finite one leaves the state and multiplies lam by 10 (ba.py's guard)
__global__ void k_lba_apply(LbaK P)
{
    LbaCtl& c = *P.ctl;
    if (c.skip) return;
    const int bad = c.nonfinite;
    if (!bad) {
        for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < P.nl; l += gridDim.x * blockDim.x) {
            const double* d = P.dxl + 3 * (long long)l;
            if (P.model == XCB_LBA_EUCLID) {
                for (int k = 0; k < 3; ++k) P.lm[3 * (long long)l + k] += d[k];
            } else {
                P.lm[3 * (long long)l] += d[0];
                P.lm[3 * (long long)l + 1] += d[1];
                P.rho[l] = fmax(P.rho[l] + d[2], P.rho_floor);
            }
        }
        if (blockIdx.x == 0)
            for (int k = threadIdx.x; k < P.nk; k += blockDim.x)
                if (P.freem[k]) se3_left_update(P.dxp + 6 * k, P.Tcw + 12 * k);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (bad) {
            c.lam = fmin(c.lam * 10.0, 1e3);
            c.nonfin_steps += 1;
        } else {
            c.lam = fmax(c.lam * 0.5, 1e-7);
            c.accepted += 1;
        }
    }
}

// nearest rotation of every R_cw (polar factor by Newton's iteration X <- (X + X^-T) / 2)
__global__ void k_lba_project(LbaK P)
{
    for (int k = threadIdx.x; k < P.nk; k += blockDim.x) {
        double X[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) X[i * 3 + j] = P.Tcw[k * 12 + i * 4 + j];
        for (int it = 0; it < 12; ++it) {
            // X^-T = cofactor(X) / det(X)
            const double C[9] = {X[4] * X[8] - X[5] * X[7], X[5] * X[6] - X[3] * X[8], X[3] * X[7] - X[4] * X[6],
                                 X[2] * X[7] - X[1] * X[8], X[0] * X[8] - X[2] * X[6], X[1] * X[6] - X[0] * X[7],
                                 X[1] * X[5] - X[2] * X[4], X[2] * X[3] - X[0] * X[5], X[0] * X[4] - X[1] * X[3]};
            const double det = X[0] * C[0] + X[1] * C[1] + X[2] * C[2];
            if (!(fabs(det) > 1e-300)) break;
            double dmax = 0.0;
            for (int i = 0; i < 9; ++i) {
                const double nx = 0.5 * (X[i] + C[i] / det);
                dmax = fmax(dmax, fabs(nx - X[i]));
                X[i] = nx;
            }
            if (dmax < 1e-16) break;
        }
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) P.Tcw[k * 12 + i * 4 + j] = X[i * 3 + j];
    }
}

__global__ void k_lba_final(LbaK P, double* stats)
{
    double acc = 0.0;
    for (long long i = threadIdx.x; i < 2LL * P.N; i += blockDim.x) acc += (double)P.resw[i] * (double)P.resw[i];
    const double chi = block_sum(acc);
    if (threadIdx.x == 0) {
        const LbaCtl& c = *P.ctl;
        stats[0] = (c.have_best && c.chi_best != 0.0) ? c.chi_best : chi;
        stats[1] = chi;
        stats[2] = c.have_rms0 ? c.rms0 : sqrt(chi / (double)(P.N > 0 ? P.N : 1));
        stats[3] = sqrt(chi / (double)(P.N > 0 ? P.N : 1));
        stats[4] = c.lam;
        stats[5] = c.accepted;
        stats[6] = c.rejected;
        stats[7] = c.nonfin_steps;
        stats[8] = c.overflow;
        stats[9] = 0.0;
    }
}

// ----------------------------------------------------------------------------------------------------- host side
struct Layout {
    size_t Tcw32, lm32, rho32, Jp, Jlm, resw, Hll, bl, Hpl, kslot, S, g, dxp, dxl, Hi, bestT, bestL, bestR, ctl, total;
};

Layout layout(const xcb_lba_problem* p)
{
    const size_t nk = p->nk, nl = p->nl, N = p->N, n = 6 * nk;
    const bool id = p->model == XCB_LBA_INVDEPTH;
    Layout L{};
    size_t o = 0;
    auto take = [&](size_t bytes) {
        const size_t at = o;
        o += (bytes + 255) & ~(size_t)255;
        return at;
    };
    L.Tcw32 = take(nk * 12 * 4);
    L.lm32 = take(nl * 3 * 4);
    L.rho32 = take(nl * 4);
    L.Jp = take(N * (id ? 24 : 12) * 4);
    L.Jlm = take(id ? 0 : N * 6 * 4);
    L.resw = take(N * 2 * 4);
    L.Hll = take(nl * 9 * 4);
    L.bl = take(nl * 3 * 4);
    L.Hpl = take(N * (id ? 36 : 18) * 4);
    L.kslot = take(id ? N * 2 * 4 : 0);
    L.S = take(n * n * 8);
    L.g = take(n * 8);
    L.dxp = take(n * 8);
    L.dxl = take(nl * 3 * 8);
    L.Hi = take(nl * 9 * 8);
    L.bestT = take(nk * 12 * 8);
    L.bestL = take(nl * 3 * 8);
    L.bestR = take(nl * 8);
    L.ctl = take(sizeof(LbaCtl));
    L.total = o;
    return L;
}

int fail(int code, const std::string& m)
{
    xcb_set_last_error(m);
    return code;
}

}  // namespace

extern "C" size_t xcb_lba_workspace_bytes(const xcb_lba_problem* p)
{
    if (!p || p->nk < 0 || p->nl < 0 || p->N < 0) return 0;
    return layout(p).total;
}

extern "C" int xcb_lba_solve(const xcb_lba_problem* p, int iters, double lam0, double* stats, void* workspace,
                             size_t workspace_bytes, void* stream)
{
    if (!p || !stats) return fail(XCB_ERR_ARG, "lba_solve: null argument");
    if (p->model != XCB_LBA_EUCLID && p->model != XCB_LBA_INVDEPTH) return fail(XCB_ERR_ARG, "lba_solve: bad model");
    if (p->nk < 1 || p->nk > XCB_LBA_MAX_SLOTS)
        return fail(XCB_ERR_CAPACITY, "lba_solve: keyframes out of range (1.." + std::to_string(XCB_LBA_MAX_SLOTS) + ")");
    if (p->nl < 0 || p->N < 0 || iters < 0) return fail(XCB_ERR_ARG, "lba_solve: negative size");
    const bool id = p->model == XCB_LBA_INVDEPTH;
    if (!p->Tcw || !p->lm || !p->free_mask || (p->nl && !p->offs) || (p->N && (!p->okf || !p->olm || !p->ouv)) ||
        (id && p->nl && (!p->rho || !p->hidx || !p->hpose)))
        return fail(XCB_ERR_ARG, "lba_solve: null pointer");
    if (id && p->p0 && !p->p4) return fail(XCB_ERR_ARG, "lba_solve: inverse-depth prior needs wbear (p4)");
    if (p->nrot && (!p->rot_a || !p->rot_b || !p->rot_M || !p->rot_sig)) return fail(XCB_ERR_ARG, "lba_solve: rotf");
    const Layout Ly = layout(p);
    if (!workspace || workspace_bytes < Ly.total) return fail(XCB_ERR_ARG, "lba_solve: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    char* w = (char*)workspace;
    LbaK P{};
    P.model = p->model;
    P.so = id ? 2 : 1;
    P.nk = p->nk; P.nl = p->nl; P.N = p->N; P.n = 6 * p->nk; P.nrot = p->nrot;
    P.fx = p->fx; P.cx = p->cx; P.cy = p->cy; P.huber = p->huber; P.rho_floor = p->rho_floor;
    P.Tcw = p->Tcw; P.lm = p->lm; P.rho = p->rho;
    P.okf = p->okf; P.olm = p->olm; P.offs = p->offs; P.freem = p->free_mask;
    P.rot_a = p->rot_a; P.rot_b = p->rot_b; P.rot_M = p->rot_M; P.rot_sig = p->rot_sig;
    P.Tcw32 = (float*)(w + Ly.Tcw32); P.lm32 = (float*)(w + Ly.lm32); P.rho32 = (float*)(w + Ly.rho32);
    P.Jp = (float*)(w + Ly.Jp); P.resw = (float*)(w + Ly.resw); P.Hll = (float*)(w + Ly.Hll);
    P.bl = (float*)(w + Ly.bl); P.Hpl = (float*)(w + Ly.Hpl);
    P.slot = id ? (const int*)(w + Ly.kslot) : p->okf;
    P.S = (double*)(w + Ly.S); P.g = (double*)(w + Ly.g); P.dxp = (double*)(w + Ly.dxp);
    P.dxl = (double*)(w + Ly.dxl); P.Hi = (double*)(w + Ly.Hi); P.bestT = (double*)(w + Ly.bestT);
    P.bestL = (double*)(w + Ly.bestL); P.bestR = (double*)(w + Ly.bestR); P.ctl = (LbaCtl*)(w + Ly.ctl);
    float* Jlm = (float*)(w + Ly.Jlm);
    int* kslot = (int*)(w + Ly.kslot);

    const float fx = (float)p->fx, cx = (float)p->cx, cy = (float)p->cy, hk = (float)p->huber;
    const int n = P.n;
    const bool smem = n <= SOLVE_SMEM_MAX_N;
    static XcbAttrOnce attr;
    {
        const cudaError_t e = xcb_smem_attr_once(attr, (const void*)k_lba_solve<true>,
                                                 (int)((size_t)SOLVE_SMEM_MAX_N * (SOLVE_SMEM_MAX_N + 1) / 2 * 8));
        if (e != cudaSuccess) return fail(XCB_ERR_CUDA, std::string("lba_solve: ") + cudaGetErrorString(e));
    }
    const size_t solve_smem = smem ? (size_t)n * (n + 1) / 2 * 8 : 0;
    int dev = 0, sms = XCB_B200_SMS;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long prep_work = std::max<long long>({(long long)P.nk * 12, (long long)P.nl * 9, (long long)n * n, 1LL});
    const unsigned prep_grid = (unsigned)std::min<long long>((prep_work + 255) / 256, (long long)sms * 4);
    const unsigned schur_grid =
        (unsigned)std::max<long long>(1, std::min<long long>(((long long)P.nl + SCHUR_WARPS - 1) / SCHUR_WARPS,
                                                             (long long)sms * 16));
    const unsigned lm_grid = (unsigned)std::max(1, (P.nl + 255) / 256);

    auto build = [&](bool with_prior) -> int {
        int rc;
        if (!id) {
            rc = xcb_bk_build_blocks(P.Tcw32, P.lm32, p->okf, p->olm, p->ouv, P.Jp, Jlm, P.resw, P.Hll, P.bl, P.Hpl,
                                     P.N, fx, cx, cy, hk, st);
            if (rc == XCB_OK && with_prior && p->p0)
                rc = xcb_bk_depth_prior(P.lm32, p->p0, p->p1, p->p2, p->p3, P.Hll, P.bl, P.nl, hk, st);
        } else {
            rc = xcb_bk_build_blocks_id(P.Tcw32, p->hpose, p->hidx, P.lm32, P.rho32, p->okf, p->olm, p->ouv, P.Jp,
                                        P.resw, kslot, P.Hll, P.bl, P.Hpl, P.N, fx, cx, cy, hk, st);
            if (rc == XCB_OK && with_prior && p->p0)
                rc = xcb_bk_landmark_prior_id(P.lm32, P.rho32, p->p0, p->p1, p->p2, p->p4, p->p3, P.Hll, P.bl, P.nl,
                                              hk, st);
        }
        return rc;
    };

    k_lba_init<<<1, 32, 0, st>>>(P, lam0);
    for (int it = 0; it < iters; ++it) {
        k_lba_prep<<<prep_grid, 256, 0, st>>>(P);
        int rc = build(true);
        if (rc != XCB_OK) return rc;
        k_lba_ctl<<<1, 1024, 0, st>>>(P);
        if (id) k_lba_schur<2><<<schur_grid, SCHUR_WARPS * 32, 0, st>>>(P);
        else k_lba_schur<1><<<schur_grid, SCHUR_WARPS * 32, 0, st>>>(P);
        if (P.nrot) k_lba_rot<<<1, 128, 0, st>>>(P);
        if (smem) k_lba_solve<true><<<1, SOLVE_THREADS, solve_smem, st>>>(P);
        else k_lba_solve<false><<<1, SOLVE_THREADS, 0, st>>>(P);
        if (id) k_lba_backsub<2><<<lm_grid, 256, 0, st>>>(P);
        else k_lba_backsub<1><<<lm_grid, 256, 0, st>>>(P);
        k_lba_apply<<<lm_grid, 256, 0, st>>>(P);
    }
    k_lba_project<<<1, 64, 0, st>>>(P);
    k_lba_prep<<<prep_grid, 256, 0, st>>>(P);
    int rc = build(false);
    if (rc != XCB_OK) return rc;
    k_lba_final<<<1, 1024, 0, st>>>(P, stats);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(XCB_ERR_CUDA, std::string("lba_solve: ") + cudaGetErrorString(e));
    return XCB_OK;
}
