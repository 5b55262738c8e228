// ba_window.cu -- batched sliding-window BA (the reference's stereo window solve) in one persistent launch (sm_100a).
//
// Model = src/xclean/vio/window.py (purely visual window): body poses [dphi, dp] (R <- R Exp(dphi), p <- p + dp),
// camera = body x extrinsic (Rbc, pbc), landmarks (a, b, rho) hosted by a keyframe (q = R_ct (R_ch m + rho (p_h -
// p_t))), left (u, v) and right u_R rows, whitened residuals, Huber IRLS (k = 1.345), optional inverse-depth prior,
// Marquardt damping of the landmark blocks (+lam Hll_ii + 1e-12) and of the reduced system (+lam S_ii + 1e-9), the
// fixed-iteration LM of window.solve (accept if the cost decreases: lam / 10, else lam x 10).  A window may hold one
// slot fixed (its rows / columns replaced by the identity).
//
// Precision split (mode XCB_BA_MIXED): the linearisation, landmark blocks and the Schur complement are FP32 with FP32
// accumulation; the reduced camera system is factored in FP64 (Cholesky); FP64 refinement steps then solve the
// residual of the FP64 normal equations, evaluated matrix-free from FP64 Jacobians recomputed per observation, until
// the correction is below 1e-9 of the step (at most 3); back-substitution and the LM cost are FP64.  Mode XCB_BA_FP64
// builds everything in FP64 (the plain form).
//
// B200 layout: one CTA per SM, persistent; windows are taken from an atomic work counter (largest first, set by the
// host), so uneven windows balance.  Inside a window one warp per landmark: lanes linearise one observation row group
// each and stage it in shared memory; the landmark's sums (Hll, bl, its Hlp blocks) are then taken sequentially over
// the observations (the reference's order), and its contribution to the reduced system is added once per entry
// (lower triangle) instead of once per observation.  The FP64 passes accumulate into warp-private vectors (no
// atomics).  The reduced system (6P x 6P, P <= 20) and its factor stay in shared memory for the whole solve: no host
// round trip per iteration (the reference returns to the host three times per LM iteration).
#include "common.cuh"
#include "ba_kernels.h"

#define BA_WARPS 6
#define BA_THREADS (BA_WARPS * 32)
#define BA_MAXP 20
#define BA_MAXN (6 * BA_MAXP)
#define BA_MAXT 16          // touched slots per landmark (host + observing keyframes)
#define BA_OBS 32           // observation row groups per landmark
#define BA_REFINE_MAX 3

struct BaWin {
    int P, L, n, hold, lm0, s0;
    double fx, fy, cx, cy, B, hk;
    double Rbc[9], pbc[3], Rcb[9], Px[9];
};

// per-warp scratch for one landmark
template <typename T>
struct WarpLm {
    T ob[BA_OBS][33];       // e0 e1 w | Jl[2][3] | Jt[2][6] | Jh[2][6]  (whitened)
    T ux[BA_OBS][2];        // refinement: w (Jt dx_t + Jh dx_h)
    T Hlp[BA_MAXT][18];
    T Tb[BA_MAXT][18];
    T hl[12];               // Hll (9) and bl (3)
    int obt[BA_OBS];        // target slot, -1 = not evaluable
    int ts[BA_MAXT];
    unsigned om[BA_MAXT];   // observations contributing to touched slot a
    double acc[2 * BA_MAXN];
};

#define OB_E 0
#define OB_W 2
#define OB_JL 3
#define OB_JT 9
#define OB_JH 21

// -------------------------------------------------------------------------------------------- small math
template <typename T>
__device__ __forceinline__ void mm3(const T* A, const T* B, T* o)
{
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) o[i * 3 + j] = A[i * 3] * B[j] + A[i * 3 + 1] * B[3 + j] + A[i * 3 + 2] * B[6 + j];
}

__device__ __forceinline__ void so3_exp(const double* w, double* R)
{
    double th2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
    double th = sqrt(th2);
    double K[9] = {0.0, -w[2], w[1], w[2], 0.0, -w[0], -w[1], w[0], 0.0};
    double a, b;
    if (th < 1e-8) { a = 1.0 - th2 / 6.0; b = 0.5 - th2 / 24.0; }
    else { a = sin(th) / th; b = (1.0 - cos(th)) / th2; }
    double KK[9];
    mm3(K, K, KK);
    for (int i = 0; i < 9; ++i) R[i] = (i % 4 == 0 ? 1.0 : 0.0) + a * K[i] + b * KK[i];
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename T>
__device__ __forceinline__ void huber_w(T en, T k, T* wt, T* c)
{
    if (en <= k) { *wt = 1; *c = (T)0.5 * en * en; }
    else { *wt = k / en; *c = k * (en - (T)0.5 * k); }
}

// per-slot camera quantities of one linearisation point (both precisions)
template <typename T>
struct SlotGeo {
    T Rwc[BA_MAXP * 9], pwc[BA_MAXP * 3];
    T N[BA_MAXP * 9];       // Rwb Px
    T M[BA_MAXP * 9];       // Rwc^T Rwb Px
    T Rcb[9];
};

// --------------------------------------------------------------------------------------------- shared layout
struct BaShared {
    BaWin w;
    double Rwb[BA_MAXP * 9], pwb[BA_MAXP * 3];
    double R2[BA_MAXP * 9], p2[BA_MAXP * 3];
    SlotGeo<double> g64;
    SlotGeo<float> g32;
    double g[BA_MAXN], y[BA_MAXN], dx[BA_MAXN], rhs[BA_MAXN], dmp[BA_MAXN];
    float bf[BA_MAXN];
    double red[BA_WARPS];
    double lam;
    int accepted;
    int overflow;
    int win;
};

// dynamic shared memory: [S64 n*n doubles][region: FP32 packed lower S + FP32 warp scratch | FP64 warp scratch]
static __host__ __device__ __forceinline__ size_t ba_off_x(int n) { return ((size_t)n * n * 8 + 15) & ~(size_t)15; }
static __host__ __device__ __forceinline__ size_t ba_s32_bytes(int n)
{
    return (((size_t)n * (n + 1) / 2) * 4 + 15) & ~(size_t)15;
}
static __host__ __device__ __forceinline__ size_t ba_x_bytes(int n)
{
    size_t a = ba_s32_bytes(n) + sizeof(WarpLm<float>) * BA_WARPS;
    size_t b = sizeof(WarpLm<double>) * BA_WARPS;
    return (a > b ? a : b);
}
size_t xcb_ba_smem_bytes(int maxP)
{
    int n = 6 * maxP;
    return ba_off_x(n) + ba_x_bytes(n);
}
__device__ __forceinline__ int tri(int i, int j) { return i * (i + 1) / 2 + j; }   // packed lower, i >= j

// ---------------------------------------------------------------------------------------------- observations
// One observation row group: whitened residual and Jacobians into ob (window.obs_residual / obs_jacobians_ws,
// window.py:126-263).  -> 0 when q2 <= 1e-9 (not evaluable).
template <typename T>
__device__ __forceinline__ int obs_lin(const BaWin& w, const SlotGeo<T>& G, const T lm[3], int h, int t, int cam,
                                       const double* z, T isg, T* ob, bool want_jac)
{
    const T a = lm[0], b = lm[1], rho = lm[2];
    const T* Rh = G.Rwc + 9 * h;
    const T* Rt = G.Rwc + 9 * t;
    T d0 = G.pwc[3 * h] - G.pwc[3 * t], d1 = G.pwc[3 * h + 1] - G.pwc[3 * t + 1], d2 = G.pwc[3 * h + 2] - G.pwc[3 * t + 2];
    T Y0 = Rh[0] * a + Rh[1] * b + Rh[2] + rho * d0;
    T Y1 = Rh[3] * a + Rh[4] * b + Rh[5] + rho * d1;
    T Y2 = Rh[6] * a + Rh[7] * b + Rh[8] + rho * d2;
    T q0 = Rt[0] * Y0 + Rt[3] * Y1 + Rt[6] * Y2;
    T q1 = Rt[1] * Y0 + Rt[4] * Y1 + Rt[7] * Y2;
    T q2 = Rt[2] * Y0 + Rt[5] * Y1 + Rt[8] * Y2;
    if (q2 <= (T)1e-9) return 0;
    const T fx = (T)w.fx, fy = (T)w.fy, B = (T)w.B;
    if (cam == 0) {
        ob[OB_E] = (fx * q0 / q2 + (T)w.cx - (T)z[0]) * isg;
        ob[OB_E + 1] = (fy * q1 / q2 + (T)w.cy - (T)z[1]) * isg;
    } else {
        ob[OB_E] = (fx * (q0 - rho * B) / q2 + (T)w.cx - (T)z[0]) * isg;
        ob[OB_E + 1] = 0;
    }
    if (!want_jac) return 1;
    const T iq = (T)1 / q2;
    T Dp[2][3];
    if (cam == 0) {
        Dp[0][0] = fx * iq * isg; Dp[0][1] = 0; Dp[0][2] = -fx * q0 * iq * iq * isg;
        Dp[1][0] = 0; Dp[1][1] = fy * iq * isg; Dp[1][2] = -fy * q1 * iq * iq * isg;
    } else {
        Dp[0][0] = fx * iq * isg; Dp[0][1] = 0; Dp[0][2] = -fx * (q0 - rho * B) * iq * iq * isg;
        Dp[1][0] = Dp[1][1] = Dp[1][2] = 0;
    }
    T RcR[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) RcR[i * 3 + j] = Rt[i] * Rh[j] + Rt[3 + i] * Rh[3 + j] + Rt[6 + i] * Rh[6 + j];
    T r0 = Rt[0] * d0 + Rt[3] * d1 + Rt[6] * d2;
    T r1 = Rt[1] * d0 + Rt[4] * d1 + Rt[7] * d2;
    T r2 = Rt[2] * d0 + Rt[5] * d1 + Rt[8] * d2;
    if (cam == 1) r0 -= B;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        ob[OB_JL + 3 * r] = Dp[r][0] * RcR[0] + Dp[r][1] * RcR[3] + Dp[r][2] * RcR[6];
        ob[OB_JL + 3 * r + 1] = Dp[r][0] * RcR[1] + Dp[r][1] * RcR[4] + Dp[r][2] * RcR[7];
        ob[OB_JL + 3 * r + 2] = Dp[r][0] * r0 + Dp[r][1] * r1 + Dp[r][2] * r2;
    }
    if (t == h) {
#pragma unroll
        for (int j = 0; j < 24; ++j) ob[OB_JT + j] = 0;
        return 1;
    }
    // target: T1 = [q]x Rcb + rho R_ct Rwb_t Px ; host: T2 = -(RcR [m]x Rcb) - rho R_ct Rwb_h Px
    const T* Rcb = G.Rcb;
    T QR[9], MR[9], Mx[9] = {0, -1, b, 1, 0, -a, -b, a, 0};
    {
        T Qx[9] = {0, -q2, q1, q2, 0, -q0, -q1, q0, 0};
        mm3(Qx, Rcb, QR);
        T Am[9];
        mm3(RcR, Mx, Am);
        mm3(Am, Rcb, MR);
    }
    const T* Mt = G.M + 9 * t;
    const T* Nh = G.N + 9 * h;
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            T t1[3], t2[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                // (R_ct N_h)[i][j] = sum_k Rt[k][i] Nh[k][j]
                T rn = Rt[i] * Nh[j] + Rt[3 + i] * Nh[3 + j] + Rt[6 + i] * Nh[6 + j];
                t1[i] = QR[i * 3 + j] + rho * Mt[i * 3 + j];
                t2[i] = -MR[i * 3 + j] - rho * rn;
            }
            ob[OB_JT + 6 * r + j] = Dp[r][0] * t1[0] + Dp[r][1] * t1[1] + Dp[r][2] * t1[2];
            ob[OB_JH + 6 * r + j] = Dp[r][0] * t2[0] + Dp[r][1] * t2[1] + Dp[r][2] * t2[2];
            // d q / d p (world): -rho R_ct, row j of Rwc_t
            T v = Dp[r][0] * Rt[3 * j] + Dp[r][1] * Rt[3 * j + 1] + Dp[r][2] * Rt[3 * j + 2];
            ob[OB_JT + 6 * r + 3 + j] = -rho * v;
            ob[OB_JH + 6 * r + 3 + j] = rho * v;
        }
    return 1;
}

// observation row groups of landmark gl that the warp scratch holds (the host rejects landmarks with more)
__device__ __forceinline__ int lm_rows(const XcbBaWindows& d, int gl)
{
    return min(d.lm_ob[gl + 1] - d.lm_ob[gl], BA_OBS);
}

// Linearise one landmark into the warp scratch: observations, Hll (damped) and bl, touched slots and their Hlp
// blocks.  -> whether the landmark enters the system (window.build_system's lm_ok); lane-local cost added to *cost.
template <typename T>
__device__ __forceinline__ bool lin_landmark(BaShared& sh, const XcbBaWindows& d, const SlotGeo<T>& G, int l,
                                             double lam, const double* lmp_src, WarpLm<T>& wl, T Hll[9], T bl[3],
                                             int* nt_out, double* cost)
{
    const int lane = threadIdx.x & 31;
    const BaWin& w = sh.w;
    const int gl = w.lm0 + l;
    const int h = d.lm_host[gl];
    const int k0 = d.lm_ob[gl], nob = lm_rows(d, gl);
    const bool h_ok = (unsigned)h < (unsigned)w.P;
    const T lm[3] = {(T)lmp_src[3 * gl], (T)lmp_src[3 * gl + 1], (T)lmp_src[3 * gl + 2]};
    int mt = -1;
    if (lane < nob) {
        const int k = k0 + lane;
        T* ob = wl.ob[lane];
        const int t = d.ob_pose[k];
        if (d.ob_valid[k] && h_ok && (unsigned)t < (unsigned)w.P) {
            if (obs_lin<T>(w, G, lm, h, t, d.ob_cam[k], d.ob_z + 2 * k, (T)d.ob_isig[k], ob, true)) {
                T en = sqrt(ob[OB_E] * ob[OB_E] + ob[OB_E + 1] * ob[OB_E + 1]), wt, cc;
                huber_w<T>(en, (T)w.hk, &wt, &cc);
                ob[OB_W] = wt;
                *cost += (double)cc;
                mt = t;
            }
        }
        wl.obt[lane] = mt;
    }
    // touched slots: observing keyframes other than the host, plus the host when any exists
    const bool pose = mt >= 0 && mt != h;
    unsigned tm = 0;
    {
        unsigned mine = pose ? (1u << mt) : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mine |= __shfl_xor_sync(0xffffffffu, mine, o);
        tm = mine ? (mine | (1u << h)) : 0u;
    }
    int nt = 0;
    for (unsigned m = tm; m; m &= m - 1) {
        const int s = __ffs(m) - 1;
        const unsigned om = __ballot_sync(0xffffffffu, pose && (s == h || mt == s));
        if (lane == 0 && nt < BA_MAXT) { wl.ts[nt] = s; wl.om[nt] = om; }
        ++nt;
    }
    if (nt > BA_MAXT) {     // the host rejects such windows; a caller that did not check gets status -2
        if (lane == 0) sh.overflow = 1;
        nt = BA_MAXT;
    }
    *nt_out = nt;
    __syncwarp();
    // Hll (9) and bl (3): one lane per entry, summed over the observations in order
    if (lane < 12) {
        T acc = 0;
        for (int i = 0; i < nob; ++i) {
            if (wl.obt[i] < 0) continue;
            const T* ob = wl.ob[i];
            const T wt = ob[OB_W];
            if (lane < 9) {
                const int p = lane / 3, q = lane % 3;
                acc += wt * (ob[OB_JL + p] * ob[OB_JL + q] + ob[OB_JL + 3 + p] * ob[OB_JL + 3 + q]);
            } else {
                const int p = lane - 9;
                acc += wt * (ob[OB_JL + p] * ob[OB_E] + ob[OB_JL + 3 + p] * ob[OB_E + 1]);
            }
        }
        wl.hl[lane] = acc;
    }
    // Hlp blocks: target slot a collects w Jl^T Jt of its observations; the host collects w Jl^T Jh of all
    for (int q = lane; q < nt * 18; q += 32) {
        const int a = q / 18, e = q % 18, i = e / 6, j = e % 6;
        const int off = wl.ts[a] == h ? OB_JH : OB_JT;
        T acc = 0;
        for (unsigned m = wl.om[a]; m; m &= m - 1) {
            const T* ob = wl.ob[__ffs(m) - 1];
            acc += ob[OB_W] * (ob[OB_JL + i] * ob[off + j] + ob[OB_JL + 3 + i] * ob[off + 6 + j]);
        }
        wl.Hlp[a][e] = acc;
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 9; ++i) Hll[i] = wl.hl[i];
#pragma unroll
    for (int i = 0; i < 3; ++i) bl[i] = wl.hl[9 + i];
    int nobs = __popc(__ballot_sync(0xffffffffu, mt >= 0));
    if (d.rho_isig[gl] > 0.0) {
        const T ris = (T)d.rho_isig[gl];
        T r0 = (lm[2] - (T)d.rho_meas[gl]) * ris, wt, cc;
        huber_w<T>(fabs(r0), (T)w.hk, &wt, &cc);
        if (lane == 0) *cost += (double)cc;
        Hll[8] += wt * ris * ris;
        bl[2] += wt * ris * r0;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) Hll[i * 4] += (T)lam * Hll[i * 4] + (T)1e-12;
    T det = Hll[0] * (Hll[4] * Hll[8] - Hll[5] * Hll[7]) - Hll[1] * (Hll[3] * Hll[8] - Hll[5] * Hll[6])
            + Hll[2] * (Hll[3] * Hll[7] - Hll[4] * Hll[6]);
    T tr = Hll[0] + Hll[4] + Hll[8];
    return nobs > 0 && det > (T)1e-18 * tr * tr * tr && isfinite(det);
}

// closed-form 3x3 inverse as window.build_system, evaluated in float64 for every precision (the landmark block of a
// low-parallax point is the ill-conditioned step)
template <typename T>
__device__ __forceinline__ void inv3(const T H[9], T Hi[9])
{
    double h[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) h[i] = (double)H[i];
    double det = h[0] * (h[4] * h[8] - h[5] * h[7]) - h[1] * (h[3] * h[8] - h[5] * h[6]) + h[2] * (h[3] * h[7] - h[4] * h[6]);
    double id = 1.0 / det;
    Hi[0] = (T)((h[4] * h[8] - h[5] * h[7]) * id);
    Hi[1] = (T)((h[2] * h[7] - h[1] * h[8]) * id);
    Hi[2] = (T)((h[1] * h[5] - h[2] * h[4]) * id);
    Hi[3] = (T)((h[5] * h[6] - h[3] * h[8]) * id);
    Hi[4] = (T)((h[0] * h[8] - h[2] * h[6]) * id);
    Hi[5] = (T)((h[2] * h[3] - h[0] * h[5]) * id);
    Hi[6] = (T)((h[3] * h[7] - h[4] * h[6]) * id);
    Hi[7] = (T)((h[1] * h[6] - h[0] * h[7]) * id);
    Hi[8] = (T)((h[0] * h[4] - h[1] * h[3]) * id);
}

// ---------------------------------------------------------------------------------------- pass A: build + Schur
// S: packed lower triangle (FP32, mixed) or full n x n (FP64 plain form, lower triangle used); gb: gradient
template <typename T, bool PACKED>
__device__ void pass_build(BaShared& sh, const XcbBaWindows& d, const SlotGeo<T>& G, T* S, T* gb, WarpLm<T>* wls,
                           double* cost_out)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int n = sh.w.n;
    WarpLm<T>& wl = wls[wid];
    double c_local = 0.0;
    for (int l = wid; l < sh.w.L; l += BA_WARPS) {
        const int gl = sh.w.lm0 + l;
        if (!d.lm_mask[gl]) continue;
        const int h = d.lm_host[gl];
        T Hll[9], bl[3];
        int nt;
        const bool ok = lin_landmark<T>(sh, d, G, l, sh.lam, d.lmp, wl, Hll, bl, &nt, &c_local);
        // pose-pose blocks (always) and, for an entering landmark, minus the Schur term
        T Hi[9], HiB[3];
        if (ok) {
            inv3<T>(Hll, Hi);
#pragma unroll
            for (int i = 0; i < 3; ++i) HiB[i] = Hi[i * 3] * bl[0] + Hi[i * 3 + 1] * bl[1] + Hi[i * 3 + 2] * bl[2];
            for (int q = lane; q < nt * 18; q += 32) {
                const int a = q / 18, e = q % 18, i = e / 6, j = e % 6;
                wl.Tb[a][e] = Hi[i * 3] * wl.Hlp[a][j] + Hi[i * 3 + 1] * wl.Hlp[a][6 + j] + Hi[i * 3 + 2] * wl.Hlp[a][12 + j];
            }
            __syncwarp();
        }
        // gradient: sum_obs w Jx^T e - Hlp^T Hll^-1 bl
        for (int q = lane; q < nt * 6; q += 32) {
            const int a = q / 6, i = q % 6, s = wl.ts[a];
            const int off = s == h ? OB_JH : OB_JT;
            T acc = 0;
            for (unsigned m = wl.om[a]; m; m &= m - 1) {
                const T* ob = wl.ob[__ffs(m) - 1];
                acc += ob[OB_W] * (ob[off + i] * ob[OB_E] + ob[off + 6 + i] * ob[OB_E + 1]);
            }
            if (ok) acc -= wl.Hlp[a][i] * HiB[0] + wl.Hlp[a][6 + i] * HiB[1] + wl.Hlp[a][12 + i] * HiB[2];
            atomicAdd(&gb[6 * s + i], acc);
        }
        // reduced system, lower triangle: block (ts[a], ts[b]) with a >= b (ts ascending)
        const int npair = nt * (nt + 1) / 2;
        for (int q = lane; q < npair * 36; q += 32) {
            const int pr = q / 36, e = q % 36, i = e / 6, j = e % 6;
            int a = (int)((sqrtf(8.0f * pr + 1.0f) - 1.0f) * 0.5f);
            while (a * (a + 1) / 2 > pr) --a;
            while ((a + 1) * (a + 2) / 2 <= pr) ++a;
            const int b = pr - a * (a + 1) / 2;
            if (a == b && j > i) continue;
            const int sa = wl.ts[a], sb = wl.ts[b];
            T acc = 0;
            // pose-pose: the same slot, or the (target, host) pair of the target's observations
            if (a == b) {
                const int off = sa == h ? OB_JH : OB_JT;
                for (unsigned m = wl.om[a]; m; m &= m - 1) {
                    const T* ob = wl.ob[__ffs(m) - 1];
                    acc += ob[OB_W] * (ob[off + i] * ob[off + j] + ob[off + 6 + i] * ob[off + 6 + j]);
                }
            } else if (sa == h || sb == h) {
                const int at = sa == h ? b : a;           // the target slot's index
                const int offa = sa == h ? OB_JH : OB_JT, offb = sb == h ? OB_JH : OB_JT;
                for (unsigned m = wl.om[at]; m; m &= m - 1) {
                    const T* ob = wl.ob[__ffs(m) - 1];
                    acc += ob[OB_W] * (ob[offa + i] * ob[offb + j] + ob[offa + 6 + i] * ob[offb + 6 + j]);
                }
            }
            if (ok) acc -= wl.Hlp[a][i] * wl.Tb[b][j] + wl.Hlp[a][6 + i] * wl.Tb[b][6 + j] + wl.Hlp[a][12 + i] * wl.Tb[b][12 + j];
            const int r = 6 * sa + i, c = 6 * sb + j;
            if (PACKED) atomicAdd(&S[tri(r, c)], acc);
            else atomicAdd(&S[r * n + c], acc);
        }
        __syncwarp();
    }
    c_local = warp_sum(c_local);
    if (cost_out && lane == 0) sh.red[wid] = c_local;
}

// ------------------------------------------------------------------------ pass B: FP64 gradient and S_true dx
// warp-private g and y = S dx (matrix-free from FP64 Jacobians), then summed over warps into sh.g / sh.y
__device__ void pass_refine(BaShared& sh, const XcbBaWindows& d, WarpLm<double>* wls, bool want_g)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int n = sh.w.n;
    WarpLm<double>& wl = wls[wid];
    double* gacc = wl.acc;
    double* yacc = wl.acc + BA_MAXN;
    for (int q = lane; q < 2 * BA_MAXN; q += 32) wl.acc[q] = 0.0;
    __syncwarp();
    double c_local = 0.0;
    for (int l = wid; l < sh.w.L; l += BA_WARPS) {
        const int gl = sh.w.lm0 + l;
        if (!d.lm_mask[gl]) continue;
        const int h = d.lm_host[gl];
        double Hll[9], bl[3];
        int nt;
        const bool ok = lin_landmark<double>(sh, d, sh.g64, l, sh.lam, d.lmp, wl, Hll, bl, &nt, &c_local);
        if (nt == 0) { __syncwarp(); continue; }
        // w (J dx) per observation row
        const int nob = lm_rows(d, gl);
        if (lane < nob && wl.obt[lane] >= 0 && wl.obt[lane] != h) {
            const double* ob = wl.ob[lane];
            const int t = wl.obt[lane];
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                double a = 0.0;
#pragma unroll
                for (int j = 0; j < 6; ++j) a += ob[OB_JT + 6 * r + j] * sh.dx[6 * t + j] + ob[OB_JH + 6 * r + j] * sh.dx[6 * h + j];
                wl.ux[lane][r] = ob[OB_W] * a;
            }
        }
        double u[3] = {0.0, 0.0, 0.0}, HiB[3] = {0.0, 0.0, 0.0};
        if (ok) {
            double Hi[9], v[3] = {0.0, 0.0, 0.0};
            inv3<double>(Hll, Hi);
            for (int a = 0; a < nt; ++a) {
                const int s = wl.ts[a];
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 6; ++j) v[i] += wl.Hlp[a][i * 6 + j] * sh.dx[6 * s + j];
            }
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                u[i] = Hi[i * 3] * v[0] + Hi[i * 3 + 1] * v[1] + Hi[i * 3 + 2] * v[2];
                HiB[i] = Hi[i * 3] * bl[0] + Hi[i * 3 + 1] * bl[1] + Hi[i * 3 + 2] * bl[2];
            }
        }
        __syncwarp();
        for (int q = lane; q < nt * 6; q += 32) {
            const int a = q / 6, i = q % 6, s = wl.ts[a];
            const int off = s == h ? OB_JH : OB_JT;
            double ga = 0.0, ya = 0.0;
            for (unsigned m = wl.om[a]; m; m &= m - 1) {
                const int k = __ffs(m) - 1;
                const double* ob = wl.ob[k];
                ga += ob[OB_W] * (ob[off + i] * ob[OB_E] + ob[off + 6 + i] * ob[OB_E + 1]);
                ya += ob[off + i] * wl.ux[k][0] + ob[off + 6 + i] * wl.ux[k][1];
            }
            if (ok) {
                ga -= wl.Hlp[a][i] * HiB[0] + wl.Hlp[a][6 + i] * HiB[1] + wl.Hlp[a][12 + i] * HiB[2];
                ya -= wl.Hlp[a][i] * u[0] + wl.Hlp[a][6 + i] * u[1] + wl.Hlp[a][12 + i] * u[2];
            }
            gacc[6 * s + i] += ga;
            yacc[6 * s + i] += ya;
        }
        __syncwarp();
    }
    c_local = warp_sum(c_local);
    if (lane == 0) sh.red[wid] = c_local;
    __syncthreads();
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        double gs = 0.0, ys = 0.0;
        for (int k = 0; k < BA_WARPS; ++k) { gs += wls[k].acc[q]; ys += wls[k].acc[BA_MAXN + q]; }
        if (want_g) sh.g[q] = gs;
        sh.y[q] = ys;
    }
    __syncthreads();
}

// ------------------------------------------------------------------ pass C: back-substitution (FP64) -> trial lmp
__device__ void pass_backsub(BaShared& sh, const XcbBaWindows& d, WarpLm<double>* wls, double* lmp_trial)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpLm<double>& wl = wls[wid];
    double c_dummy = 0.0;
    for (int l = wid; l < sh.w.L; l += BA_WARPS) {
        const int gl = sh.w.lm0 + l;
        if (!d.lm_mask[gl]) {
            if (lane < 3) lmp_trial[3 * gl + lane] = d.lmp[3 * gl + lane];
            continue;
        }
        double Hll[9], bl[3];
        int nt;
        const bool ok = lin_landmark<double>(sh, d, sh.g64, l, sh.lam, d.lmp, wl, Hll, bl, &nt, &c_dummy);
        if (lane < 3) {
            double out = d.lmp[3 * gl + lane];
            if (ok) {
                double Hi[9];
                inv3<double>(Hll, Hi);
                double v[3] = {bl[0], bl[1], bl[2]};
                for (int a = 0; a < nt; ++a) {
                    const int s = wl.ts[a];
                    for (int i = 0; i < 3; ++i) {
                        double acc = 0.0;
                        for (int j = 0; j < 6; ++j) acc += wl.Hlp[a][i * 6 + j] * sh.dx[6 * s + j];
                        v[i] += acc;
                    }
                }
                double dl[3];
                for (int i = 0; i < 3; ++i) dl[i] = -(Hi[i * 3] * v[0] + Hi[i * 3 + 1] * v[1] + Hi[i * 3 + 2] * v[2]);
                const double r = d.lmp[3 * gl + 2] + dl[2];
                if (r > 1e-9 && isfinite(r)) out = lane == 2 ? r : d.lmp[3 * gl + lane] + dl[lane];
            }
            lmp_trial[3 * gl + lane] = out;
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------------------------- pass D: FP64 cost of a state
__device__ void pass_cost(BaShared& sh, const XcbBaWindows& d, const SlotGeo<double>& G, const double* lmp)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double c = 0.0;
    for (int l = wid; l < sh.w.L; l += BA_WARPS) {
        const int gl = sh.w.lm0 + l;
        if (!d.lm_mask[gl]) continue;
        const int h = d.lm_host[gl];
        if ((unsigned)h >= (unsigned)sh.w.P) continue;
        const double lm[3] = {lmp[3 * gl], lmp[3 * gl + 1], lmp[3 * gl + 2]};
        for (int k = d.lm_ob[gl] + lane; k < d.lm_ob[gl + 1]; k += 32) {
            if (!d.ob_valid[k] || (unsigned)d.ob_pose[k] >= (unsigned)sh.w.P) continue;
            double ob[33];
            if (!obs_lin<double>(sh.w, G, lm, h, d.ob_pose[k], d.ob_cam[k], d.ob_z + 2 * k, d.ob_isig[k], ob, false)) {
                c += 1e6;
                continue;
            }
            double wt, cc;
            huber_w<double>(sqrt(ob[0] * ob[0] + ob[1] * ob[1]), sh.w.hk, &wt, &cc);
            c += cc;
        }
        if (lane == 0 && d.rho_isig[gl] > 0.0) {
            double r0 = (lm[2] - d.rho_meas[gl]) * d.rho_isig[gl], wt, cc;
            huber_w<double>(fabs(r0), sh.w.hk, &wt, &cc);
            c += cc;
        }
    }
    c = warp_sum(c);
    if (lane == 0) sh.red[wid] = c;
}

// ----------------------------------------------------------------------------------- CTA-wide dense FP64 algebra
// in-place lower Cholesky of S (n x n, row-major, lower triangle) -> 0 ok, else -1 (not positive definite)
__device__ int chol_factor(double* S, int n)
{
    __shared__ int bad;
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    for (int j = 0; j < n; ++j) {
        if (threadIdx.x == 0) {
            double dj = S[j * n + j];
            if (!(dj > 0.0) || !isfinite(dj)) { bad = 1; dj = 1.0; }
            S[j * n + j] = sqrt(dj);
        }
        __syncthreads();
        const double dj = S[j * n + j];
        for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) S[i * n + j] /= dj;
        __syncthreads();
        // trailing update of the lower triangle: row i, columns j+1..i
        for (int i = j + 1 + threadIdx.x / 32; i < n; i += blockDim.x / 32) {
            const double lij = S[i * n + j];
            for (int c = j + 1 + (threadIdx.x & 31); c <= i; c += 32) S[i * n + c] -= lij * S[c * n + j];
        }
        __syncthreads();
    }
    return bad ? -1 : 0;
}

// x <- (L L^T)^-1 x, column-oriented (no reductions)
__device__ void chol_solve(const double* Lc, int n, double* x)
{
    for (int j = 0; j < n; ++j) {
        if (threadIdx.x == 0) x[j] /= Lc[j * n + j];
        __syncthreads();
        const double xj = x[j];
        for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) x[i] -= Lc[i * n + j] * xj;
        __syncthreads();
    }
    for (int j = n - 1; j >= 0; --j) {
        if (threadIdx.x == 0) x[j] /= Lc[j * n + j];
        __syncthreads();
        const double xj = x[j];
        for (int i = threadIdx.x; i < j; i += blockDim.x) x[i] -= Lc[j * n + i] * xj;
        __syncthreads();
    }
}

// camera poses and the per-slot products of the Jacobians, FP64 and FP32
__device__ void slot_geo(BaShared& sh, const double* Rwb, const double* pwb)
{
    const int P = sh.w.P;
    SlotGeo<double>& G = sh.g64;
    for (int q = threadIdx.x; q < P * 9; q += blockDim.x) {
        const int s = q / 9, i = (q % 9) / 3, j = q % 3;
        double acc = 0.0, nacc = 0.0;
        for (int k = 0; k < 3; ++k) {
            acc += Rwb[9 * s + 3 * i + k] * sh.w.Rbc[3 * k + j];
            nacc += Rwb[9 * s + 3 * i + k] * sh.w.Px[3 * k + j];
        }
        G.Rwc[q] = acc;
        G.N[q] = nacc;
    }
    for (int q = threadIdx.x; q < P * 3; q += blockDim.x) {
        const int s = q / 3, i = q % 3;
        double acc = pwb[q];
        for (int k = 0; k < 3; ++k) acc += Rwb[9 * s + 3 * i + k] * sh.w.pbc[k];
        G.pwc[q] = acc;
    }
    if (threadIdx.x < 9) G.Rcb[threadIdx.x] = sh.w.Rcb[threadIdx.x];
    __syncthreads();
    for (int q = threadIdx.x; q < P * 9; q += blockDim.x) {
        const int s = q / 9, i = (q % 9) / 3, j = q % 3;
        double acc = 0.0;
        for (int k = 0; k < 3; ++k) acc += G.Rwc[9 * s + 3 * k + i] * G.N[9 * s + 3 * k + j];
        G.M[q] = acc;
    }
    __syncthreads();
    SlotGeo<float>& F = sh.g32;
    for (int q = threadIdx.x; q < P * 9; q += blockDim.x) {
        F.Rwc[q] = (float)G.Rwc[q]; F.N[q] = (float)G.N[q]; F.M[q] = (float)G.M[q];
    }
    for (int q = threadIdx.x; q < P * 3; q += blockDim.x) F.pwc[q] = (float)G.pwc[q];
    if (threadIdx.x < 9) F.Rcb[threadIdx.x] = (float)G.Rcb[threadIdx.x];
    __syncthreads();
}

__device__ double block_sum_red(BaShared& sh)
{
    __syncthreads();
    double s = 0.0;
    for (int i = 0; i < BA_WARPS; ++i) s += sh.red[i];
    __syncthreads();
    return s;
}

// ------------------------------------------------------------------------------------------------- the kernel
__global__ void __launch_bounds__(BA_THREADS, 1) k_ba_windows(XcbBaWindows d, int iters, double lam0, int mode,
                                                              double* stats, double* dx0, int dx0_stride,
                                                              double* lmp_trial, int* counter)
{
    extern __shared__ __align__(16) unsigned char dsm[];
    __shared__ BaShared sh;
    __shared__ double s_norm[2];
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) sh.win = atomicAdd(counter, 1);
        __syncthreads();
        const int wi = sh.win;
        if (wi >= d.nw) break;
        const int w = d.order ? d.order[wi] : wi;
        if (tid == 0) {
            BaWin& W = sh.w;
            W.P = d.P[w]; W.L = d.L[w]; W.n = 6 * W.P; W.hold = d.hold ? d.hold[w] : -1;
            W.lm0 = d.lm_off[w]; W.s0 = d.slot_off[w];
            W.fx = d.cam[6 * w]; W.fy = d.cam[6 * w + 1]; W.cx = d.cam[6 * w + 2]; W.cy = d.cam[6 * w + 3];
            W.B = d.cam[6 * w + 4]; W.hk = d.cam[6 * w + 5];
            for (int i = 0; i < 9; ++i) W.Rbc[i] = d.ext[12 * w + i];
            for (int i = 0; i < 3; ++i) W.pbc[i] = d.ext[12 * w + 9 + i];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) W.Rcb[i * 3 + j] = W.Rbc[j * 3 + i];
            double px[9] = {0.0, -W.pbc[2], W.pbc[1], W.pbc[2], 0.0, -W.pbc[0], -W.pbc[1], W.pbc[0], 0.0};
            for (int i = 0; i < 9; ++i) W.Px[i] = px[i];
            sh.lam = lam0; sh.accepted = 0; sh.overflow = 0;
        }
        __syncthreads();
        const int P = sh.w.P, n = sh.w.n, L = sh.w.L, s0 = sh.w.s0;
        if (P > BA_MAXP || P < 1) {
            if (tid == 0) stats[8 * w + 4] = -1.0;
            __syncthreads();
            continue;
        }
        for (int q = tid; q < P * 9; q += blockDim.x) sh.Rwb[q] = d.Rwb[9 * s0 + q];
        for (int q = tid; q < P * 3; q += blockDim.x) sh.pwb[q] = d.pwb[3 * s0 + q];
        __syncthreads();
        double* S64 = (double*)dsm;
        float* S32 = (float*)(dsm + ba_off_x(n));
        WarpLm<float>* wl32 = (WarpLm<float>*)(dsm + ba_off_x(n) + ba_s32_bytes(n));
        WarpLm<double>* wl64 = (WarpLm<double>*)(dsm + ba_off_x(n));
        double cost0 = 0.0, cur = 0.0;
        for (int it = 0; it < iters; ++it) {
            slot_geo(sh, sh.Rwb, sh.pwb);
            for (int q = tid; q < n; q += blockDim.x) { sh.g[q] = 0.0; sh.y[q] = 0.0; sh.bf[q] = 0.0f; }
            double c_tot = 0.0;
            if (mode == XCB_BA_MIXED) {
                for (int q = tid; q < n * (n + 1) / 2; q += blockDim.x) S32[q] = 0.0f;
                __syncthreads();
                pass_build<float, true>(sh, d, sh.g32, S32, sh.bf, wl32, nullptr);
                __syncthreads();
                for (int q = tid; q < n * n; q += blockDim.x) {
                    const int i = q / n, j = q % n;
                    S64[q] = j <= i ? (double)S32[tri(i, j)] : 0.0;
                }
                for (int q = tid; q < n; q += blockDim.x) sh.rhs[q] = (double)sh.bf[q];
            } else {
                for (int q = tid; q < n * n; q += blockDim.x) S64[q] = 0.0;
                __syncthreads();
                pass_build<double, false>(sh, d, sh.g64, S64, sh.g, wl64, &c_tot);
                c_tot = block_sum_red(sh);
                for (int q = tid; q < n; q += blockDim.x) sh.rhs[q] = sh.g[q];
            }
            __syncthreads();
            // hold, damping (D = lam diag + 1e-9, kept for the refinement residual), RHS = -b
            const int hs = sh.w.hold;
            if (hs >= 0 && hs < P) {
                for (int q = tid; q < 6 * n; q += blockDim.x) {
                    const int i = 6 * hs + q / n, j = q % n;
                    S64[i * n + j] = 0.0;
                    S64[j * n + i] = 0.0;
                }
                __syncthreads();
                for (int q = tid; q < 6; q += blockDim.x) { S64[(6 * hs + q) * n + 6 * hs + q] = 1.0; sh.rhs[6 * hs + q] = 0.0; }
                __syncthreads();
            }
            for (int q = tid; q < n; q += blockDim.x) {
                const double dg = S64[q * n + q];
                sh.dmp[q] = sh.lam * dg + 1e-9;
                S64[q * n + q] = dg + sh.dmp[q];
                sh.dx[q] = -sh.rhs[q];
            }
            __syncthreads();
            const int bad = chol_factor(S64, n);
            if (bad) {
                if (mode == XCB_BA_MIXED) {
                    pass_cost(sh, d, sh.g64, d.lmp);
                    c_tot = block_sum_red(sh);
                }
                if (it == 0) cost0 = c_tot;
                cur = c_tot;
                if (tid == 0) sh.lam *= 10.0;
                __syncthreads();
                continue;
            }
            chol_solve(S64, n, sh.dx);
            if (mode == XCB_BA_MIXED) {
                // FP64 refinement: rho = -g - (S + D) dx with S dx matrix-free from FP64 Jacobians; repeated while the
                // correction exceeds 1e-9 of the step
                for (int rf = 0; rf < BA_REFINE_MAX; ++rf) {
                    pass_refine(sh, d, wl64, rf == 0);
                    if (rf == 0) c_tot = block_sum_red(sh);
                    for (int q = tid; q < n; q += blockDim.x) {
                        double r = -sh.g[q] - sh.y[q] - sh.dmp[q] * sh.dx[q];
                        if (hs >= 0 && q / 6 == hs) r = 0.0;
                        sh.rhs[q] = r;
                    }
                    __syncthreads();
                    chol_solve(S64, n, sh.rhs);
                    if (tid == 0) {
                        double a = 0.0, b = 0.0;
                        for (int q = 0; q < n; ++q) { a += sh.rhs[q] * sh.rhs[q]; b += sh.dx[q] * sh.dx[q]; }
                        s_norm[0] = a; s_norm[1] = b;
                    }
                    __syncthreads();
                    for (int q = tid; q < n; q += blockDim.x) sh.dx[q] += sh.rhs[q];
                    __syncthreads();
                    if (!(s_norm[0] > 1e-18 * s_norm[1])) break;
                }
            }
            if (it == 0) {
                cost0 = c_tot;
                if (dx0)
                    for (int q = tid; q < n; q += blockDim.x) dx0[(size_t)w * dx0_stride + q] = sh.dx[q];
            }
            // trial state: landmarks (back-substitution), poses
            pass_backsub(sh, d, wl64, lmp_trial);
            for (int s = tid; s < P; s += blockDim.x) {
                double Re[9], R[9];
                so3_exp(sh.dx + 6 * s, Re);
                for (int i = 0; i < 9; ++i) R[i] = sh.Rwb[9 * s + i];
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j)
                        sh.R2[9 * s + 3 * i + j] = R[3 * i] * Re[j] + R[3 * i + 1] * Re[3 + j] + R[3 * i + 2] * Re[6 + j];
                for (int i = 0; i < 3; ++i) sh.p2[3 * s + i] = sh.pwb[3 * s + i] + sh.dx[6 * s + 3 + i];
            }
            __syncthreads();
            slot_geo(sh, sh.R2, sh.p2);
            pass_cost(sh, d, sh.g64, lmp_trial);
            const double c_new = block_sum_red(sh);
            const bool acc = c_new < c_tot;
            if (acc) {
                for (int q = tid; q < P * 9; q += blockDim.x) sh.Rwb[q] = sh.R2[q];
                for (int q = tid; q < P * 3; q += blockDim.x) sh.pwb[q] = sh.p2[q];
                const int lm0 = sh.w.lm0;
                for (int q = tid; q < 3 * L; q += blockDim.x) d.lmp[3 * lm0 + q] = lmp_trial[3 * lm0 + q];
            }
            cur = acc ? c_new : c_tot;
            if (tid == 0) {
                if (acc) { sh.lam = fmax(sh.lam / 10.0, 1e-12); sh.accepted += 1; }
                else sh.lam *= 10.0;
            }
            __syncthreads();
        }
        for (int q = tid; q < P * 9; q += blockDim.x) d.Rwb[9 * s0 + q] = sh.Rwb[q];
        for (int q = tid; q < P * 3; q += blockDim.x) d.pwb[3 * s0 + q] = sh.pwb[q];
        if (tid == 0) {
            stats[8 * w + 0] = cost0;
            stats[8 * w + 1] = cur;
            stats[8 * w + 2] = sh.accepted;
            stats[8 * w + 3] = sh.lam;
            stats[8 * w + 4] = sh.overflow ? -2.0 : 0.0;
            stats[8 * w + 5] = iters;
        }
        __syncthreads();
    }
}

cudaError_t xcb_launch_ba_windows(const XcbBaWindows& d, int max_slots, int iters, double lam0, int mode,
                                  double* stats, double* dx0, int dx0_stride, double* lmp_trial, int* counter,
                                  int grid, cudaStream_t st)
{
    size_t sm = xcb_ba_smem_bytes(max_slots);
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_ba_windows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)xcb_ba_smem_bytes(BA_MAXP));
        if (e != cudaSuccess) return e;
        attr = true;
    }
    k_ba_windows<<<grid, BA_THREADS, sm, st>>>(d, iters, lam0, mode, stats, dx0, dx0_stride, lmp_trial, counter);
    return cudaGetLastError();
}

int xcb_ba_max_slots() { return BA_MAXP; }
