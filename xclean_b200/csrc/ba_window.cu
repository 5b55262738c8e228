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
#include "ba_tc.cuh"
#include <cooperative_groups.h>
namespace cg = cooperative_groups;

#define BA_WARPS 11
#define BA_THREADS (BA_WARPS * 32)
#define BA_MAXP 20
#define BA_MAXN (6 * BA_MAXP)
#define BA_MAXT 16          // touched slots per landmark (host + observing keyframes)
#define BA_OBS 32           // observation row groups per landmark
#define BA_REFINE_MAX 3
// per-landmark scratch of the Newton / adjoint kernel (19 doubles); entry 18 flags a landmark held constant
#define BA_LSC_STRIDE 19
#define BA_LSC_FROZEN 18
// per-landmark back-substitution record, written by the float64 build and read by the back-substitution of the same
// LM iteration (the state and the damping are the same): [0] = touched slots nt (-1: more than BA_BSC_NT, recompute;
// -2: no step), [1..3] Hll^-1 bl, [4..4+nt) the slots, [10 + 18 a + 6 i + j] (Hll^-1 Hlp_a)[i][j]
#define BA_BSC_NT 6
#define BA_BSC 118

struct BaWin {
    int P, L, n, hold, lm0, s0;
    double fx, fy, cx, cy, B, hk;
    double Rbc[9], pbc[3], Rcb[9], Px[9];
};

#define OB_E 0
#define OB_W 2
#define OB_JL 3
#define OB_JT 9
#define OB_JH 21
#define OB_N 27

// the pose Jacobian of a staged observation row group: row r, column i of the target (off = OB_JT) or host
// (off = OB_JH) block; the host block's translation columns are minus the target block's
template <typename T>
__device__ __forceinline__ T obj(const T* ob, int off, int r, int i)
{
    if (off == OB_JT) return ob[OB_JT + 6 * r + i];
    return i < 3 ? ob[OB_JH + 3 * r + i] : -ob[OB_JT + 6 * r + i];
}

// per-warp scratch for one landmark
template <typename T>
struct WarpLm {
    T ob[BA_OBS][OB_N];     // e0 e1 w | Jl[2][3] | Jt[2][6] | Jh[2][0..2]  (whitened; Jh[r][3..5] = -Jt[r][3..5])
    T ux[BA_OBS][2];        // refinement: w (Jt dx_t + Jh dx_h)
    T Hlp[BA_MAXT][18];
    T Tb[BA_MAXT][18];
    T hl[12];               // Hll (9) and bl (3)
    int obt[BA_OBS];        // target slot, -1 = not evaluable
    int ts[BA_MAXT];
    unsigned om[BA_MAXT];   // observations contributing to touched slot a
};

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
    double pr_d[BA_MAXN], pr_res[BA_MAXN];     // marginal prior: block deltas (or S x), residual S d + r
    double pr_cost;
    double lam;
    int accepted;
    int overflow;
    int win;
    int lb, le;             // the landmarks (window-local) the landmark passes of this CTA visit
};

// dynamic shared memory: [S64, packed lower, n(n+1)/2 doubles][region: FP32 packed lower S + FP32 warp scratch |
// FP64 warp scratch]
static __host__ __device__ __forceinline__ size_t ba_off_x(int n)
{
    return (((size_t)n * (n + 1) / 2) * 8 + 15) & ~(size_t)15;
}
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

// a landmark held constant: its rows still enter the pose blocks and the gradient, but it has no Schur term and no
// step (frz: the Newton scratch's flags; null: none)
__device__ __forceinline__ bool lm_const(const double* frz, int gl)
{
    return frz != nullptr && frz[(size_t)gl * BA_LSC_STRIDE + BA_LSC_FROZEN] != 0.0;
}

// ---------------------------------------------------------------------------------------------- observations
// One observation row group: whitened residual and Jacobians into ob (window.obs_residual / obs_jacobians_ws,
// window.py:126-263).  jac: 0 the residual only, 1 every Jacobian, 2 the landmark Jacobian only (the pose blocks are
// left unwritten).  -> 0 when q2 <= 1e-9 (not evaluable).
template <typename T>
__device__ __forceinline__ int obs_lin(const BaWin& w, const SlotGeo<T>& G, const T lm[3], int h, int t, int cam,
                                       const double* z, T isg, T* ob, int jac)
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
    if (!jac) return 1;
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
    if (jac == 2) return 1;
    if (t == h) {
#pragma unroll
        for (int j = 0; j < 18; ++j) ob[OB_JT + j] = 0;
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
            ob[OB_JH + 3 * r + j] = Dp[r][0] * t2[0] + Dp[r][1] * t2[1] + Dp[r][2] * t2[2];
            // d q / d p (world): -rho R_ct, row j of Rwc_t
            T v = Dp[r][0] * Rt[3 * j] + Dp[r][1] * Rt[3 * j + 1] + Dp[r][2] * Rt[3 * j + 2];
            ob[OB_JT + 6 * r + 3 + j] = -rho * v;
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
// exp_ob (optional): the window's per-observation whitened squared residuals (final_linearisation's ob_chi2), indexed
// from the window's first observation: inf where the observation is invalid or its point is behind the camera.
template <typename T>
__device__ __forceinline__ bool lin_landmark(BaShared& sh, const XcbBaWindows& d, const SlotGeo<T>& G, int l,
                                             double lam, const double* lmp_src, WarpLm<T>& wl, T Hll[9], T bl[3],
                                             int* nt_out, double* cost, double* exp_ob = nullptr)
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
        double chi2 = XCB_INF;
        if (d.ob_valid[k] && h_ok && (unsigned)t < (unsigned)w.P) {
            if (obs_lin<T>(w, G, lm, h, t, d.ob_cam[k], d.ob_z + 2 * k, (T)d.ob_isig[k], ob, 1)) {
                const T e2 = ob[OB_E] * ob[OB_E] + ob[OB_E + 1] * ob[OB_E + 1];
                T en = sqrt(e2), wt, cc;
                huber_w<T>(en, (T)w.hk, &wt, &cc);
                ob[OB_W] = wt;
                *cost += (double)cc;
                mt = t;
                chi2 = (double)e2;
            }
        }
        wl.obt[lane] = mt;
        if (exp_ob) exp_ob[k - d.lm_ob[w.lm0]] = chi2;
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
            acc += ob[OB_W] * (ob[OB_JL + i] * obj(ob, off, 0, j) + ob[OB_JL + 3 + i] * obj(ob, off, 1, j));
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
// exp_lm / exp_ob (optional, final_linearisation's exports): per landmark of the window [lm_ok, Hll^-1 (9)] (written
// for the landmarks the mask admits; Hll^-1 only where lm_ok), per observation its chi2 (lin_landmark).
template <typename T, bool PACKED>
__device__ void pass_build(BaShared& sh, const XcbBaWindows& d, const SlotGeo<T>& G, T* S, T* gb, WarpLm<T>* wls,
                           double* cost_out, const double* frz = nullptr, double* bsc = nullptr,
                           double* exp_lm = nullptr, double* exp_ob = nullptr)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int n = sh.w.n;
    WarpLm<T>& wl = wls[wid];
    double c_local = 0.0;
    for (int l = sh.lb + wid; l < sh.le; l += BA_WARPS) {
        const int gl = sh.w.lm0 + l;
        if (!d.lm_mask[gl]) continue;
        const int h = d.lm_host[gl];
        T Hll[9], bl[3];
        int nt;
        const bool ok = lin_landmark<T>(sh, d, G, l, sh.lam, d.lmp, wl, Hll, bl, &nt, &c_local, exp_ob)
                        && !lm_const(frz, gl);
        // pose-pose blocks (always) and, for an entering landmark, minus the Schur term
        T Hi[9], HiB[3];
        if (exp_lm && lane == 0) exp_lm[10 * (size_t)l] = ok ? 1.0 : 0.0;
        if (ok) {
            inv3<T>(Hll, Hi);
            if (exp_lm && lane < 9) exp_lm[10 * (size_t)l + 1 + lane] = (double)Hi[lane];
#pragma unroll
            for (int i = 0; i < 3; ++i) HiB[i] = Hi[i * 3] * bl[0] + Hi[i * 3 + 1] * bl[1] + Hi[i * 3 + 2] * bl[2];
            for (int q = lane; q < nt * 18; q += 32) {
                const int a = q / 18, e = q % 18, i = e / 6, j = e % 6;
                wl.Tb[a][e] = Hi[i * 3] * wl.Hlp[a][j] + Hi[i * 3 + 1] * wl.Hlp[a][6 + j] + Hi[i * 3 + 2] * wl.Hlp[a][12 + j];
            }
            __syncwarp();
        }
        if (bsc) {
            double* rec = bsc + (size_t)gl * BA_BSC;
            const bool keep = ok && nt <= BA_BSC_NT;
            if (lane == 0) rec[0] = !ok ? -2.0 : (keep ? (double)nt : -1.0);
            if (keep) {
                if (lane < 3) rec[1 + lane] = (double)HiB[lane];
                if (lane < nt) rec[4 + lane] = (double)wl.ts[lane];
                for (int q = lane; q < nt * 18; q += 32) rec[10 + q] = (double)wl.Tb[q / 18][q % 18];
            }
        }
        // gradient: sum_obs w Jx^T e - Hlp^T Hll^-1 bl
        for (int q = lane; q < nt * 6; q += 32) {
            const int a = q / 6, i = q % 6, s = wl.ts[a];
            const int off = s == h ? OB_JH : OB_JT;
            T acc = 0;
            for (unsigned m = wl.om[a]; m; m &= m - 1) {
                const T* ob = wl.ob[__ffs(m) - 1];
                acc += ob[OB_W] * (obj(ob, off, 0, i) * ob[OB_E] + obj(ob, off, 1, i) * ob[OB_E + 1]);
            }
            if (ok) acc -= wl.Hlp[a][i] * HiB[0] + wl.Hlp[a][6 + i] * HiB[1] + wl.Hlp[a][12 + i] * HiB[2];
            atomicAdd(&gb[6 * s + i], acc);
        }
        // reduced system, lower triangle: block (ts[a], ts[b]) with a >= b (ts ascending).  A lane per (pair, row i)
        // takes the row's entries, so the pair decode, the row's Jacobian entries and its Hlp column are read once per
        // row instead of once per entry
        const int npair = nt * (nt + 1) / 2;
        for (int q = lane; q < npair * 6; q += 32) {
            const int pr = q / 6, i = q % 6;
            int a = (int)((sqrtf(8.0f * pr + 1.0f) - 1.0f) * 0.5f);
            while (a * (a + 1) / 2 > pr) --a;
            while ((a + 1) * (a + 2) / 2 <= pr) ++a;
            const int b = pr - a * (a + 1) / 2;
            const int sa = wl.ts[a], sb = wl.ts[b];
            const int jn = a == b ? i + 1 : 6;
            T acc[6];
#pragma unroll
            for (int j = 0; j < 6; ++j) acc[j] = 0;
            // pose-pose: the same slot, or the (target, host) pair of the target's observations
            const bool pp = a == b || sa == h || sb == h;
            if (pp) {
                const int at = a == b ? a : (sa == h ? b : a);    // the observations: the slot's, or the target's
                const int offa = sa == h ? OB_JH : OB_JT, offb = sb == h ? OB_JH : OB_JT;
                for (unsigned m = wl.om[at]; m; m &= m - 1) {
                    const T* ob = wl.ob[__ffs(m) - 1];
                    const T ri0 = obj(ob, offa, 0, i), ri1 = obj(ob, offa, 1, i), wt = ob[OB_W];
#pragma unroll
                    for (int j = 0; j < 6; ++j) acc[j] += wt * (ri0 * obj(ob, offb, 0, j) + ri1 * obj(ob, offb, 1, j));
                }
            }
            if (ok) {
                const T h0 = wl.Hlp[a][i], h1 = wl.Hlp[a][6 + i], h2 = wl.Hlp[a][12 + i];
#pragma unroll
                for (int j = 0; j < 6; ++j) acc[j] -= h0 * wl.Tb[b][j] + h1 * wl.Tb[b][6 + j] + h2 * wl.Tb[b][12 + j];
            }
            const int r = 6 * sa + i;
#pragma unroll
            for (int j = 0; j < 6; ++j) {
                if (j >= jn) break;
                const int c = 6 * sb + j;
                if (PACKED) atomicAdd(&S[tri(r, c)], acc[j]);
                else atomicAdd(&S[r * n + c], acc[j]);
            }
        }
        __syncwarp();
    }
    c_local = warp_sum(c_local);
    if (cost_out && lane == 0) sh.red[wid] = c_local;
}

// ------------------------------------------------------------------------ pass B: FP64 gradient and S_true dx
// warp-private g and y = S dx (matrix-free from FP64 Jacobians), then summed over warps into sh.g / sh.y
__device__ void pass_refine(BaShared& sh, const XcbBaWindows& d, WarpLm<double>* wls, bool want_g,
                            const double* frz = nullptr, double* bsc = nullptr)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int n = sh.w.n;
    WarpLm<double>& wl = wls[wid];
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        if (want_g) sh.g[q] = 0.0;
        sh.y[q] = 0.0;
    }
    __syncthreads();
    double c_local = 0.0;
    for (int l = sh.lb + wid; l < sh.le; l += BA_WARPS) {
        const int gl = sh.w.lm0 + l;
        if (!d.lm_mask[gl]) continue;
        const int h = d.lm_host[gl];
        double Hll[9], bl[3];
        int nt;
        const bool ok = lin_landmark<double>(sh, d, sh.g64, l, sh.lam, d.lmp, wl, Hll, bl, &nt, &c_local) &&
                        !lm_const(frz, gl);
        if (nt == 0) {
            if (bsc && lane == 0) bsc[(size_t)gl * BA_BSC] = -1.0;     // the back-substitution re-linearises it
            __syncwarp();
            continue;
        }
        // w (J dx) per observation row
        const int nob = lm_rows(d, gl);
        if (lane < nob && wl.obt[lane] >= 0 && wl.obt[lane] != h) {
            const double* ob = wl.ob[lane];
            const int t = wl.obt[lane];
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                double a = 0.0;
#pragma unroll
                for (int j = 0; j < 6; ++j) a += ob[OB_JT + 6 * r + j] * sh.dx[6 * t + j] + obj(ob, OB_JH, r, j) * sh.dx[6 * h + j];
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
            if (bsc && nt <= BA_BSC_NT) {     // the back-substitution record, from these float64 blocks
                double* rec = bsc + (size_t)gl * BA_BSC;
                if (lane < 3) rec[1 + lane] = HiB[lane];
                if (lane < nt) rec[4 + lane] = (double)wl.ts[lane];
                for (int q = lane; q < nt * 18; q += 32) {
                    const int a = q / 18, e = q % 18, i = e / 6, j = e % 6;
                    rec[10 + q] = Hi[i * 3] * wl.Hlp[a][j] + Hi[i * 3 + 1] * wl.Hlp[a][6 + j] + Hi[i * 3 + 2] * wl.Hlp[a][12 + j];
                }
            }
        }
        if (bsc && lane == 0) bsc[(size_t)gl * BA_BSC] = !ok ? -2.0 : (nt <= BA_BSC_NT ? (double)nt : -1.0);
        __syncwarp();
        for (int q = lane; q < nt * 6; q += 32) {
            const int a = q / 6, i = q % 6, s = wl.ts[a];
            const int off = s == h ? OB_JH : OB_JT;
            double ga = 0.0, ya = 0.0;
            for (unsigned m = wl.om[a]; m; m &= m - 1) {
                const int k = __ffs(m) - 1;
                const double* ob = wl.ob[k];
                ga += ob[OB_W] * (obj(ob, off, 0, i) * ob[OB_E] + obj(ob, off, 1, i) * ob[OB_E + 1]);
                ya += obj(ob, off, 0, i) * wl.ux[k][0] + obj(ob, off, 1, i) * wl.ux[k][1];
            }
            if (ok) {
                ga -= wl.Hlp[a][i] * HiB[0] + wl.Hlp[a][6 + i] * HiB[1] + wl.Hlp[a][12 + i] * HiB[2];
                ya -= wl.Hlp[a][i] * u[0] + wl.Hlp[a][6 + i] * u[1] + wl.Hlp[a][12 + i] * u[2];
            }
            if (want_g) atomicAdd(&sh.g[6 * s + i], ga);
            atomicAdd(&sh.y[6 * s + i], ya);
        }
        __syncwarp();
    }
    c_local = warp_sum(c_local);
    if (lane == 0) sh.red[wid] = c_local;
    __syncthreads();
}

// ------------------------------------------------------------------ pass C: back-substitution (FP64) -> trial lmp
// one landmark re-linearised by the whole warp (no record, or none kept): dl = -Hll^-1 (bl + sum_a Hlp_a dx_{slot a})
__device__ void backsub_relin(BaShared& sh, const XcbBaWindows& d, WarpLm<double>& wl, int l, double* lmp_trial,
                              const double* frz)
{
    const int lane = threadIdx.x & 31;
    const int gl = sh.w.lm0 + l;
    double Hll[9], bl[3], c_dummy = 0.0;
    int nt;
    const bool ok = lin_landmark<double>(sh, d, sh.g64, l, sh.lam, d.lmp, wl, Hll, bl, &nt, &c_dummy) &&
                    !lm_const(frz, gl);
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

__device__ void pass_backsub(BaShared& sh, const XcbBaWindows& d, WarpLm<double>* wls, double* lmp_trial,
                             const double* frz = nullptr, const double* bsc = nullptr)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpLm<double>& wl = wls[wid];
    if (!bsc) {
        for (int l = sh.lb + wid; l < sh.le; l += BA_WARPS) {
            const int gl = sh.w.lm0 + l;
            if (!d.lm_mask[gl]) {
                if (lane < 3) lmp_trial[3 * gl + lane] = d.lmp[3 * gl + lane];
                continue;
            }
            backsub_relin(sh, d, wl, l, lmp_trial, frz);
        }
        return;
    }
    // the build's records: dl = -(Hll^-1 bl + sum_a (Hll^-1 Hlp_a) dx_{slot a}).  Ten landmarks per warp, a lane per
    // landmark component, so that the record loads of ten landmarks are in flight together; a landmark without a
    // record (more than BA_BSC_NT touched slots) is re-linearised by the whole warp afterwards
    const int sub = lane / 3, comp = lane - 3 * sub;
    for (int l0 = sh.lb + wid * 10; l0 < sh.le; l0 += BA_WARPS * 10) {
        const int l = l0 + sub;
        const bool mine = lane < 30 && l < sh.le;
        const int gl = sh.w.lm0 + (mine ? l : l0);
        bool masked = false;
        int nt = -2;
        double v = 0.0;
        if (mine) {
            masked = !d.lm_mask[gl];
            if (!masked) {
                const double* rec = bsc + (size_t)gl * BA_BSC;
                nt = (int)rec[0];
                if (nt >= 0) {
                    v = rec[1 + comp];
                    for (int a = 0; a < nt; ++a) {
                        const int sl = (int)rec[4 + a];
                        const double* tb = rec + 10 + 18 * a + 6 * comp;
#pragma unroll
                        for (int j = 0; j < 6; ++j) v += tb[j] * sh.dx[6 * sl + j];
                    }
                }
            }
        }
        const double dl2 = __shfl_sync(0xffffffffu, -v, min(3 * sub + 2, 31));
        const bool redo = mine && !masked && (nt == -1 || nt < -2);
        if (mine && !redo) {
            double out = d.lmp[3 * gl + comp];
            if (!masked && nt >= 0) {
                const double r = d.lmp[3 * gl + 2] + dl2;
                if (r > 1e-9 && isfinite(r)) out = comp == 2 ? r : d.lmp[3 * gl + comp] - v;
            }
            lmp_trial[3 * gl + comp] = out;
        }
        for (unsigned m = __ballot_sync(0xffffffffu, redo && comp == 0); m; m &= m - 1)
            backsub_relin(sh, d, wl, l0 + (__ffs(m) - 1) / 3, lmp_trial, frz);
    }
}

// ------------------------------------------------------------------------------- pass D: FP64 cost of a state
__device__ void pass_cost(BaShared& sh, const XcbBaWindows& d, const SlotGeo<double>& G, const double* lmp)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double c = 0.0;
    for (int l = sh.lb + wid; l < sh.le; l += BA_WARPS) {
        const int gl = sh.w.lm0 + l;
        if (!d.lm_mask[gl]) continue;
        const int h = d.lm_host[gl];
        if ((unsigned)h >= (unsigned)sh.w.P) continue;
        const double lm[3] = {lmp[3 * gl], lmp[3 * gl + 1], lmp[3 * gl + 2]};
        for (int k = d.lm_ob[gl] + lane; k < d.lm_ob[gl + 1]; k += 32) {
            if (!d.ob_valid[k] || (unsigned)d.ob_pose[k] >= (unsigned)sh.w.P) continue;
            double ob[OB_N];
            if (!obs_lin<double>(sh.w, G, lm, h, d.ob_pose[k], d.ob_cam[k], d.ob_z + 2 * k, d.ob_isig[k], ob, 0)) {
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
            double dj = S[tri(j, j)];
            if (!(dj > 0.0) || !isfinite(dj)) { bad = 1; dj = 1.0; }
            S[tri(j, j)] = sqrt(dj);
        }
        __syncthreads();
        const double dj = S[tri(j, j)];
        for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) S[tri(i, j)] /= dj;
        __syncthreads();
        // trailing update of the lower triangle: row i, columns j+1..i
        for (int i = j + 1 + threadIdx.x / 32; i < n; i += blockDim.x / 32) {
            double* row = S + tri(i, 0);
            const double lij = row[j];
            for (int c = j + 1 + (threadIdx.x & 31); c <= i; c += 32) row[c] -= lij * S[tri(c, j)];
        }
        __syncthreads();
    }
    return bad ? -1 : 0;
}

// x <- (L L^T)^-1 x, column-oriented (no reductions)
__device__ void chol_solve(const double* Lc, int n, double* x)
{
    for (int j = 0; j < n; ++j) {
        if (threadIdx.x == 0) x[j] /= Lc[tri(j, j)];
        __syncthreads();
        const double xj = x[j];
        for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) x[i] -= Lc[tri(i, j)] * xj;
        __syncthreads();
    }
    for (int j = n - 1; j >= 0; --j) {
        if (threadIdx.x == 0) x[j] /= Lc[tri(j, j)];
        __syncthreads();
        const double xj = x[j];
        const double* row = Lc + tri(j, 0);
        for (int i = threadIdx.x; i < j; i += blockDim.x) x[i] -= row[i] * xj;
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

// ------------------------------------------------------------------------------------------------ marginal prior
// The prior 1/2 |S d + r|^2 of marg.Prior (src/xclean/vio/marg.py:124-140) over pose blocks, added to the reduced
// system, the gradient and the cost as window._full_system and window.solve add it (window.py:865-887, :963-964).
__device__ __forceinline__ bool has_prior(const XcbBaWindows& d, int w) { return d.pr_m != nullptr && d.pr_m[w] > 0; }

// window.so3_log_nb (src/xclean/vio/window.py:65-105)
__device__ void so3_log_dev(const double* R, double* w)
{
    double c = (R[0] + R[4] + R[8] - 1.0) * 0.5;
    c = fmin(fmax(c, -1.0), 1.0);
    const double th = acos(c);
    const double v0 = R[7] - R[5], v1 = R[2] - R[6], v2 = R[3] - R[1];
    if (th < 1e-6) { w[0] = 0.5 * v0; w[1] = 0.5 * v1; w[2] = 0.5 * v2; return; }
    if (th > 3.141592653589793 - 1e-4) {
        // near pi: the axis from the symmetric part, its sign from the skew part
        double B[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) B[3 * i + j] = (R[3 * i + j] + R[3 * j + i]) * 0.5;
        int i = 0;
        if (B[4] > B[4 * i]) i = 1;
        if (B[8] > B[4 * i]) i = 2;
        const double den = sqrt(fmax((B[4 * i] - c) / (1.0 - c), 0.0));
        double ax[3];
        for (int j = 0; j < 3; ++j) ax[j] = (B[3 * j + i] - (j == i ? c : 0.0)) / fmax(den * (1.0 - c), 1e-12);
        ax[i] = den;
        const double nrm = sqrt(ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2]);
        const double sg = ax[0] * v0 + ax[1] * v1 + ax[2] * v2 < 0 ? -1.0 : 1.0;
        for (int j = 0; j < 3; ++j) w[j] = sg * th * ax[j] / nrm;
        return;
    }
    const double f = th / (2.0 * sin(th));
    w[0] = f * v0; w[1] = f * v1; w[2] = f * v2;
}

// residual S d + r at the slot poses (Rwb, pwb) into sh.pr_res; -> 1/2 |S d + r|^2 (every thread)
__device__ double prior_residual(BaShared& sh, const XcbBaWindows& d, int w, const double* Rwb, const double* pwb)
{
    const int m = d.pr_m[w], nb = d.pr_nb[w], nc = 6 * nb, b0 = d.pr_boff[w];
    const double* S = d.pr_S + d.pr_soff[w];
    const double* r = d.pr_r + d.pr_roff[w];
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        const int s = d.pr_blk[b0 + k];
        const double* x0 = d.pr_x0 + 12 * (size_t)(b0 + k);
        const double* R = Rwb + 9 * s;
        double A[9];                                    // R0^T R
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) A[3 * i + j] = x0[i] * R[j] + x0[3 + i] * R[3 + j] + x0[6 + i] * R[6 + j];
        so3_log_dev(A, sh.pr_d + 6 * k);
        for (int i = 0; i < 3; ++i) sh.pr_d[6 * k + 3 + i] = pwb[3 * s + i] - x0[9 + i];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        double acc = 0.0;
        for (int j = 0; j < nc; ++j) acc += S[(size_t)i * nc + j] * sh.pr_d[j];
        sh.pr_res[i] = acc + r[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double c = 0.0;
        for (int i = 0; i < m; ++i) c += sh.pr_res[i] * sh.pr_res[i];
        sh.pr_cost = 0.5 * c;
    }
    __syncthreads();
    return sh.pr_cost;
}

__device__ __forceinline__ int prior_col(const XcbBaWindows& d, int w, int i)
{
    return 6 * d.pr_blk[d.pr_boff[w] + i / 6] + i % 6;
}

// S^T S into the packed lower reduced system, S^T res (sh.pr_res) into grad (may be null) and into grad2 (may be null)
__device__ void prior_system(BaShared& sh, const XcbBaWindows& d, int w, double* S64, double* grad, double* grad2)
{
    const int m = d.pr_m[w], nc = 6 * d.pr_nb[w];
    const double* S = d.pr_S + d.pr_soff[w];
    if (S64)
        for (int q = threadIdx.x; q < nc * nc; q += blockDim.x) {
            const int i = q / nc, j = q % nc;
            if (j > i) continue;
            double acc = 0.0;
            for (int k = 0; k < m; ++k) acc += S[(size_t)k * nc + i] * S[(size_t)k * nc + j];
            int ci = prior_col(d, w, i), cj = prior_col(d, w, j);
            if (ci < cj) { const int t = ci; ci = cj; cj = t; }
            S64[tri(ci, cj)] += acc;
        }
    for (int i = threadIdx.x; i < nc; i += blockDim.x) {
        double acc = 0.0;
        for (int k = 0; k < m; ++k) acc += S[(size_t)k * nc + i] * sh.pr_res[k];
        const int ci = prior_col(d, w, i);
        if (grad) grad[ci] += acc;
        if (grad2) grad2[ci] += acc;
    }
    __syncthreads();
}

// y += S^T S x on the prior's columns (the refinement's matrix-free product; uses sh.pr_d as scratch)
__device__ void prior_apply(BaShared& sh, const XcbBaWindows& d, int w, const double* x, double* y)
{
    const int m = d.pr_m[w], nc = 6 * d.pr_nb[w];
    const double* S = d.pr_S + d.pr_soff[w];
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
        double acc = 0.0;
        for (int j = 0; j < nc; ++j) acc += S[(size_t)k * nc + j] * x[prior_col(d, w, j)];
        sh.pr_d[k] = acc;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nc; i += blockDim.x) {
        double acc = 0.0;
        for (int k = 0; k < m; ++k) acc += S[(size_t)k * nc + i] * sh.pr_d[k];
        y[prior_col(d, w, i)] += acc;
    }
    __syncthreads();
}

// ------------------------------------------------------------------------------------------------- the kernel
__global__ void __launch_bounds__(BA_THREADS, 1) k_ba_windows(XcbBaWindows d, int iters, double lam0, int mode,
                                                              double* stats, double* dx0, int dx0_stride,
                                                              double* lmp_trial, int* counter, const double* frz,
                                                              size_t trial_doubles)
{
    extern __shared__ __align__(16) unsigned char dsm[];
    __shared__ BaShared sh;
    __shared__ double s_norm[2];
    __shared__ double* s_bsc;
    __shared__ int s_short;
    // the back-substitution records follow the trial states when the scratch holds them (float64 mode); the batch's
    // landmark count is taken from the windows themselves, not from the caller
    if (threadIdx.x == 0) {
        long long Lt = 0;
        for (int w = 0; w < d.nw; ++w) Lt = max(Lt, (long long)d.lm_off[w] + d.L[w]);
        const size_t off = ((size_t)3 * Lt + 31) / 32 * 32;
        s_short = (size_t)3 * Lt > trial_doubles;
        s_bsc = off + (size_t)Lt * BA_BSC <= trial_doubles ? lmp_trial + off : nullptr;
    }
    __syncthreads();
    if (s_short) {
        // the trial states do not fit the scratch: nothing is written but every window's status
        if (blockIdx.x == 0)
            for (int w = threadIdx.x; w < d.nw; w += blockDim.x) stats[8 * w + 4] = XCB_BA_STATUS_SCRATCH;
        return;
    }
    double* const bsc = s_bsc;
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
            sh.lb = 0; sh.le = W.L;
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
                pass_build<float, true>(sh, d, sh.g32, S32, sh.bf, wl32, nullptr, frz);
                __syncthreads();
                for (int q = tid; q < n * (n + 1) / 2; q += blockDim.x) S64[q] = (double)S32[q];
                for (int q = tid; q < n; q += blockDim.x) sh.rhs[q] = (double)sh.bf[q];
            } else {
                for (int q = tid; q < n * (n + 1) / 2; q += blockDim.x) S64[q] = 0.0;
                __syncthreads();
                // the landmark records and chi2 only when the window's row of dx0 holds them
                const long long Mw = (long long)d.lm_ob[sh.w.lm0 + L] - d.lm_ob[sh.w.lm0];
                double* exl = mode == XCB_BA_LINEARISE && (long long)n * n + n + 10LL * L + Mw <= dx0_stride
                                  ? dx0 + (size_t)w * dx0_stride + (size_t)n * n + n : nullptr;
                pass_build<double, true>(sh, d, sh.g64, S64, sh.g, wl64, &c_tot, frz, bsc, exl,
                                         exl ? exl + 10 * (size_t)L : nullptr);
                c_tot = block_sum_red(sh);
                for (int q = tid; q < n; q += blockDim.x) sh.rhs[q] = sh.g[q];
            }
            __syncthreads();
            const bool pri = has_prior(d, w);
            if (pri) {
                // the prior at the linearisation point: its information into the system, its gradient into the
                // right-hand side source (and the float64 gradient), its cost into the iteration's cost
                c_tot += prior_residual(sh, d, w, sh.Rwb, sh.pwb);
                prior_system(sh, d, w, S64, sh.rhs, mode == XCB_BA_MIXED ? nullptr : sh.g);
            }
            if (mode == XCB_BA_LINEARISE) {
                // final_linearisation's visual part (window.py:985-1008): the reduced system at the current state, no
                // hold, no step; dx0 receives, for each window, H (n x n, row-major), b (n), the landmark records
                // [lm_ok, Hll^-1] (10 L, from pass_build) and the observations' chi2 (from lin_landmark)
                double* o = dx0 + (size_t)w * dx0_stride;
                for (int q = tid; q < n * n; q += blockDim.x) {
                    const int i = q / n, j = q % n;
                    o[q] = S64[i >= j ? tri(i, j) : tri(j, i)];
                }
                for (int q = tid; q < n; q += blockDim.x) o[(size_t)n * n + q] = sh.g[q];
                cost0 = c_tot;
                cur = c_tot;
                __syncthreads();
                break;
            }
            // hold, damping (D = lam diag + 1e-9, kept for the refinement residual), RHS = -b
            const int hs = sh.w.hold;
            if (hs >= 0 && hs < P) {
                for (int q = tid; q < 6 * n; q += blockDim.x) {
                    const int i = 6 * hs + q / n, j = q % n;
                    S64[i >= j ? tri(i, j) : tri(j, i)] = 0.0;
                }
                __syncthreads();
                for (int q = tid; q < 6; q += blockDim.x) { S64[tri(6 * hs + q, 6 * hs + q)] = 1.0; sh.rhs[6 * hs + q] = 0.0; }
                __syncthreads();
            }
            for (int q = tid; q < n; q += blockDim.x) {
                const double dg = S64[tri(q, q)];
                sh.dmp[q] = sh.lam * dg + 1e-9;
                S64[tri(q, q)] = dg + sh.dmp[q];
                sh.dx[q] = -sh.rhs[q];
            }
            __syncthreads();
            const int bad = chol_factor(S64, n);
            if (bad) {
                if (mode == XCB_BA_MIXED) {
                    pass_cost(sh, d, sh.g64, d.lmp);
                    c_tot = block_sum_red(sh) + (pri ? sh.pr_cost : 0.0);
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
                    pass_refine(sh, d, wl64, rf == 0, frz, rf == 0 ? bsc : nullptr);
                    if (rf == 0) c_tot = block_sum_red(sh) + (pri ? sh.pr_cost : 0.0);
                    if (pri) {
                        if (rf == 0) prior_system(sh, d, w, nullptr, sh.g, nullptr);   // pr_res: this state's
                        prior_apply(sh, d, w, sh.dx, sh.y);
                    }
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
            pass_backsub(sh, d, wl64, lmp_trial, frz, bsc);
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
            double c_new = block_sum_red(sh);
            if (pri) c_new += prior_residual(sh, d, w, sh.R2, sh.p2);
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

// =====================================================================================================================
// Exact second derivatives of the window cost: Newton polish and the implicit adjoint.
//
// The cost C(x, theta) = sum_k huber(|e_k|) + sum_l huber(|r_l|) (the same terms as above).  Its exact Hessian H is
// never formed: H p comes from evaluating the analytic gradient (w J^T e, the Jacobians of obs_lin) in dual numbers
// along p, which also gives the mixed derivative (d2C / dtheta dx) p when the analytic theta-gradient is evaluated the
// same way.  At a stationary point (the converged solve) this equals the Hessian of C in the pose charts used here
// (R <- R Exp(dphi), p <- p + dp), the terms of the chart's connection being proportional to the gradient.
// H x = b is solved by conjugate gradients preconditioned with the Gauss-Newton system: its Schur complement is built
// and Cholesky-factored once per linearisation, each preconditioner application is two landmark passes and one
// triangular solve with that factor, each CG iteration one dual pass for H p.
// =====================================================================================================================
struct Dual {
    double v, e;
    __host__ __device__ Dual() : v(0.0), e(0.0) {}
    __host__ __device__ Dual(double x) : v(x), e(0.0) {}
    __host__ __device__ Dual(double x, double y) : v(x), e(y) {}
    __device__ Dual& operator+=(const Dual& o) { v += o.v; e += o.e; return *this; }
    __device__ Dual& operator-=(const Dual& o) { v -= o.v; e -= o.e; return *this; }
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.e + b.e); }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.e - b.e); }
__device__ __forceinline__ Dual operator-(Dual a) { return Dual(-a.v, -a.e); }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.e * b.v + a.v * b.e); }
__device__ __forceinline__ Dual operator/(Dual a, Dual b)
{
    const double iv = 1.0 / b.v;
    return Dual(a.v * iv, (a.e - a.v * iv * b.e) * iv);
}
__device__ __forceinline__ bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
__device__ __forceinline__ bool operator<(Dual a, Dual b) { return a.v < b.v; }
__device__ __forceinline__ bool operator>(Dual a, Dual b) { return a.v > b.v; }
__device__ __forceinline__ Dual sqrt(Dual a)
{
    const double s = ::sqrt(a.v);
    return Dual(s, s > 0.0 ? 0.5 * a.e / s : 0.0);
}
__device__ __forceinline__ Dual fabs(Dual a) { return a.v < 0.0 ? -a : a; }

#define NT_MODE_GRAD 0          // value parts: the exact gradient
#define NT_MODE_HV 1            // dual parts: H p
#define NT_MODE_THETA 2         // dual parts of the theta-gradient: (d2C / dtheta dx) p
#define NT_THETA 11             // fx, fy, cx, cy, B, omega (3), t (3)

// per-landmark scratch of the exact solves (global memory): b (rhs), r (residual), p (direction, the dual pass's
// tangent), x (solution), z (preconditioned residual), Hp, and the frozen flag: a landmark whose Gauss-Newton step
// would take its inverse depth to <= 1e-9 is never moved by window.solve (apply_update's positive-depth rule), so the
// state it converges to is stationary in every variable but those landmarks, which are constants here
#define NT_LM_STRIDE 19
#define NT_FROZEN 18
static_assert(NT_LM_STRIDE == BA_LSC_STRIDE && NT_FROZEN == BA_LSC_FROZEN, "one layout of the landmark scratch");
#define NT_B 0
#define NT_R 3
#define NT_P 6
#define NT_X 9
#define NT_Z 12
#define NT_HP 15

struct NtShared {
    double gp[BA_MAXN];         // value accumulators of the pose gradient
    double hp[BA_MAXN];         // dual accumulators (H p)
    double th[NT_THETA];
    double red2;
    double cred;                // this CTA's partial of a cluster reduction
};

// ---------------------------------------------------------------------------------------------------------------------
// Reductions over the CTAs of a thread-block cluster (distributed shared memory).  The Newton kernel gives each window a
// cluster whose CTAs take slices of the window's landmarks; these sums run in rank order, so every CTA holds the same
// bits afterwards and every CTA takes the same branches.  Every thread of every CTA calls them, with a block-uniform
// partial; with one CTA per cluster they return at once.
__device__ double cl_reduce(NtShared& nt, double v, bool mx)
{
    cg::cluster_group cl = cg::this_cluster();
    const unsigned C = cl.num_blocks();
    if (C == 1) return v;
    if (threadIdx.x == 0) nt.cred = v;
    cl.sync();
    double s = 0.0;
    for (unsigned r = 0; r < C; ++r) {
        const double x = *cl.map_shared_rank(&nt.cred, r);
        s = mx ? (r == 0 ? x : fmax(s, x)) : s + x;
    }
    cl.sync();
    return s;
}

// a[0, len) in shared memory summed over the cluster's CTAs into every CTA: each CTA totals its slice in rank order,
// then copies the others' slices from their owners
__device__ void cl_sum_array(double* a, int len)
{
    cg::cluster_group cl = cg::this_cluster();
    const int C = (int)cl.num_blocks(), r = (int)cl.block_rank();
    if (C == 1) return;
    cl.sync();
    const int b0 = (int)((long long)len * r / C), b1 = (int)((long long)len * (r + 1) / C);
    for (int q = b0 + threadIdx.x; q < b1; q += blockDim.x) {
        double t = 0.0;
        for (int k = 0; k < C; ++k) t += *cl.map_shared_rank(a + q, k);
        a[q] = t;
    }
    cl.sync();
    for (int q = threadIdx.x; q < len; q += blockDim.x) {
        int o = 0;
        while (o + 1 < C && q >= (int)((long long)len * (o + 1) / C)) ++o;
        if (o != r) a[q] = *cl.map_shared_rank(a + q, o);
    }
    cl.sync();
}

__device__ __forceinline__ bool held(const BaShared& sh, int q) { return sh.w.hold >= 0 && q / 6 == sh.w.hold; }

// geometry of the state moved along p: Rwb (I + eps hat(p_phi)), pwb + eps p_p (p = zp per slot)
__device__ void slot_geo_dual(const BaShared& sh, const double* zp, SlotGeo<Dual>& G)
{
    const int P = sh.w.P;
    for (int s = threadIdx.x; s < P; s += blockDim.x) {
        const double* R0 = sh.Rwb + 9 * s;
        const double w0 = zp[6 * s], w1 = zp[6 * s + 1], w2 = zp[6 * s + 2];
        const double K[9] = {0.0, -w2, w1, w2, 0.0, -w0, -w1, w0, 0.0};
        Dual R[9], p[3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                R[i * 3 + j] = Dual(R0[i * 3 + j],
                                    R0[i * 3] * K[j] + R0[i * 3 + 1] * K[3 + j] + R0[i * 3 + 2] * K[6 + j]);
        for (int i = 0; i < 3; ++i) p[i] = Dual(sh.pwb[3 * s + i], zp[6 * s + 3 + i]);
        Dual Rwc[9], N[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                Dual a = Dual(0.0), b = Dual(0.0);
                for (int k = 0; k < 3; ++k) {
                    a = a + R[i * 3 + k] * Dual(sh.w.Rbc[3 * k + j]);
                    b = b + R[i * 3 + k] * Dual(sh.w.Px[3 * k + j]);
                }
                Rwc[i * 3 + j] = a;
                N[i * 3 + j] = b;
            }
        for (int i = 0; i < 3; ++i) {
            Dual a = p[i];
            for (int k = 0; k < 3; ++k) a = a + R[i * 3 + k] * Dual(sh.w.pbc[k]);
            G.pwc[3 * s + i] = a;
        }
        for (int i = 0; i < 9; ++i) { G.Rwc[9 * s + i] = Rwc[i]; G.N[9 * s + i] = N[i]; }
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                Dual a = Dual(0.0);
                for (int k = 0; k < 3; ++k) a = a + Rwc[3 * k + i] * N[3 * k + j];
                G.M[9 * s + i * 3 + j] = a;
            }
    }
    if (threadIdx.x < 9) G.Rcb[threadIdx.x] = Dual(sh.w.Rcb[threadIdx.x]);
    __syncthreads();
}

// d e / d theta of one observation row group (whitened residual e): columns fx, fy, cx, cy, B, omega (3), t (3) of
// the left-to-right extrinsic at the rectified rig (q_r = Exp(omega) q + rho (t - B e_x)), the row's weight 1/sigma,
// and its pixel (z0, z1).  -> 0 when not evaluable.
template <typename T>
__device__ __forceinline__ int obs_theta(const BaWin& w, const SlotGeo<T>& G, const T lm[3], int h, int t, int cam,
                                         const double* z, double isgd, T de[2][14])
{
    const T a = lm[0], b = lm[1], rho = lm[2];
    const T* Rh = G.Rwc + 9 * h;
    const T* Rt = G.Rwc + 9 * t;
    const T d0 = G.pwc[3 * h] - G.pwc[3 * t], d1 = G.pwc[3 * h + 1] - G.pwc[3 * t + 1],
            d2 = G.pwc[3 * h + 2] - G.pwc[3 * t + 2];
    const T Y0 = Rh[0] * a + Rh[1] * b + Rh[2] + rho * d0;
    const T Y1 = Rh[3] * a + Rh[4] * b + Rh[5] + rho * d1;
    const T Y2 = Rh[6] * a + Rh[7] * b + Rh[8] + rho * d2;
    const T q0 = Rt[0] * Y0 + Rt[3] * Y1 + Rt[6] * Y2;
    const T q1 = Rt[1] * Y0 + Rt[4] * Y1 + Rt[7] * Y2;
    const T q2 = Rt[2] * Y0 + Rt[5] * Y1 + Rt[8] * Y2;
    if (q2 <= (T)1e-9) return 0;
    const T s = (T)isgd, fx = (T)w.fx, fy = (T)w.fy, B = (T)w.B;
    for (int r = 0; r < 2; ++r)
        for (int j = 0; j < 14; ++j) de[r][j] = (T)0.0;
    const T iq = (T)1.0 / q2;
    if (cam == 0) {
        de[0][0] = q0 * iq * s;
        de[1][1] = q1 * iq * s;
        de[0][2] = s;
        de[1][3] = s;
        de[0][11] = fx * q0 * iq + (T)w.cx - (T)z[0];
        de[1][11] = fy * q1 * iq + (T)w.cy - (T)z[1];
        de[0][12] = -s;
        de[1][13] = -s;
    } else {
        const T qr0 = q0 - rho * B;
        de[0][0] = qr0 * iq * s;
        de[0][2] = s;
        de[0][4] = -fx * rho * iq * s;
        const T D0 = fx * iq * s, D2 = -fx * qr0 * iq * iq * s;          // d e_R / d q_r (its u row)
        de[0][5] = D2 * q1;                                              // D (-hat(q))
        de[0][6] = D0 * q2 - D2 * q0;
        de[0][7] = -D0 * q1;
        de[0][8] = D0 * rho;
        de[0][10] = D2 * rho;
        de[0][11] = fx * qr0 * iq + (T)w.cx - (T)z[0];
        de[0][12] = -s;
    }
    return 1;
}

// One pass over the window's landmarks with the state moved along p (sh.dx for the poses, scratch NT_P for the
// landmarks): value parts = the exact gradient, dual parts = H p; in NT_MODE_THETA the theta-gradient's dual parts.
// Outputs: nt.gp / nt.hp (pose accumulators, atomics), per landmark: -gradient -> NT_B (GRAD), (H p)_l -> NT_HP (HV);
// THETA: nt.th and the per-row outputs.  Landmarks that are not variables get zeros.
__device__ void pass_dual(BaShared& sh, NtShared& nt, const XcbBaWindows& d, const SlotGeo<Dual>& G, int mode,
                          double* lsc, double* gisig, double* gz, double mu = 0.0, bool upd = false)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int l = sh.lb + wid; l < sh.le; l += BA_WARPS) {
        const int gl = sh.w.lm0 + l;
        if (!d.lm_mask[gl]) continue;
        const int h = d.lm_host[gl];
        if ((unsigned)h >= (unsigned)sh.w.P) continue;
        double* sc = lsc + (size_t)gl * NT_LM_STRIDE;
        const int k0 = d.lm_ob[gl], nob = lm_rows(d, gl);
        // the landmark moves along p only if it is a variable (its Gauss-Newton block passes the conditioning test,
        // decided below on the same sums; a landmark that is not a variable has p_l = 0 in the scratch)
        const Dual lm[3] = {Dual(d.lmp[3 * gl], sc[NT_P]), Dual(d.lmp[3 * gl + 1], sc[NT_P + 1]),
                            Dual(d.lmp[3 * gl + 2], sc[NT_P + 2])};
        Dual gl3[3] = {Dual(0.0), Dual(0.0), Dual(0.0)}, gh[6];
        double hv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        double gnl[3] = {0.0, 0.0, 0.0}, gnh[6] = {0, 0, 0, 0, 0, 0};      // Gauss-Newton products w J^T (J p)
        int nobs = 0;
        for (int i = 0; i < 6; ++i) gh[i] = Dual(0.0);
        if (lane < nob) {
            const int k = k0 + lane;
            const int t = d.ob_pose[k];
            Dual ob[OB_N];
            if (d.ob_valid[k] && (unsigned)t < (unsigned)sh.w.P &&
                obs_lin<Dual>(sh.w, G, lm, h, t, d.ob_cam[k], d.ob_z + 2 * k, Dual(d.ob_isig[k]), ob, 1)) {
                const Dual en = sqrt(ob[OB_E] * ob[OB_E] + ob[OB_E + 1] * ob[OB_E + 1]);
                Dual wt, cc;
                huber_w<Dual>(en, Dual(sh.w.hk), &wt, &cc);
                nobs = 1;
                const double jp0 = ob[OB_E].e, jp1 = ob[OB_E + 1].e;             // J p (the dual part of e)
                for (int i = 0; i < 3; ++i) {
                    gl3[i] = wt * (ob[OB_JL + i] * ob[OB_E] + ob[OB_JL + 3 + i] * ob[OB_E + 1]);
                    gnl[i] = wt.v * (ob[OB_JL + i].v * jp0 + ob[OB_JL + 3 + i].v * jp1);
                    for (int j = 0; j < 3; ++j)
                        hv[i * 3 + j] = wt.v * (ob[OB_JL + i].v * ob[OB_JL + j].v + ob[OB_JL + 3 + i].v * ob[OB_JL + 3 + j].v);
                }
                if (t != h) {
                    for (int i = 0; i < 6; ++i) {
                        const Dual gt = wt * (ob[OB_JT + i] * ob[OB_E] + ob[OB_JT + 6 + i] * ob[OB_E + 1]);
                        const Dual jh0 = obj(ob, OB_JH, 0, i), jh1 = obj(ob, OB_JH, 1, i);
                        gh[i] = wt * (jh0 * ob[OB_E] + jh1 * ob[OB_E + 1]);
                        gnh[i] = wt.v * (jh0.v * jp0 + jh1.v * jp1);
                        if (mode != NT_MODE_THETA) {
                            const double gnt = wt.v * (ob[OB_JT + i].v * jp0 + ob[OB_JT + 6 + i].v * jp1);
                            atomicAdd(&nt.gp[6 * t + i], gt.v);
                            atomicAdd(&nt.hp[6 * t + i], gt.e + mu * gnt);
                        }
                    }
                }
                if (mode == NT_MODE_THETA) {
                    Dual de[2][14];
                    if (obs_theta<Dual>(sh.w, G, lm, h, t, d.ob_cam[k], d.ob_z + 2 * k, d.ob_isig[k], de)) {
                        Dual gth[14];
                        for (int j = 0; j < 14; ++j) gth[j] = wt * (ob[OB_E] * de[0][j] + ob[OB_E + 1] * de[1][j]);
                        for (int j = 0; j < NT_THETA; ++j) atomicAdd(&nt.th[j], -gth[j].e);
                        if (gisig) gisig[k] = -gth[11].e;
                        if (gz) { gz[2 * k] = -gth[12].e; gz[2 * k + 1] = -gth[13].e; }
                    }
                }
            }
        }
        // landmark sums (all lanes), the inverse-depth prior, the variable test
        for (int i = 0; i < 9; ++i) hv[i] = warp_sum(hv[i]);
        nobs = __popc(__ballot_sync(0xffffffffu, nobs != 0));
        for (int i = 0; i < 3; ++i) {
            gl3[i].v = warp_sum(gl3[i].v);
            gl3[i].e = warp_sum(gl3[i].e);
            gnl[i] = warp_sum(gnl[i]);
        }
        for (int i = 0; i < 6; ++i) {
            gh[i].v = warp_sum(gh[i].v);
            gh[i].e = warp_sum(gh[i].e);
            gnh[i] = warp_sum(gnh[i]);
        }
        if (d.rho_isig[gl] > 0.0) {
            const Dual ris = Dual(d.rho_isig[gl]);
            const Dual r0 = (lm[2] - Dual(d.rho_meas[gl])) * ris;
            Dual wt, cc;
            huber_w<Dual>(fabs(r0), Dual(sh.w.hk), &wt, &cc);
            gl3[2] = gl3[2] + wt * ris * r0;
            gnl[2] += wt.v * ris.v * r0.e;
            hv[8] += wt.v * d.rho_isig[gl] * d.rho_isig[gl];
        }
        for (int i = 0; i < 3; ++i) hv[i * 4] += 1e-12;
        const double det = hv[0] * (hv[4] * hv[8] - hv[5] * hv[7]) - hv[1] * (hv[3] * hv[8] - hv[5] * hv[6]) +
                           hv[2] * (hv[3] * hv[7] - hv[4] * hv[6]);
        const double tr = hv[0] + hv[4] + hv[8];
        bool var = nobs > 0 && det > 1e-18 * tr * tr * tr && isfinite(det);
        if (mode == NT_MODE_GRAD && upd) {
            // a flag, once set, stays (cleared with the scratch): the set of constant landmarks only grows, so the
            // polish converges on one well-defined problem; the adjoint uses the flags as they are
            bool frozen = sc[NT_FROZEN] != 0.0;
            if (var && !frozen) {      // the Gauss-Newton landmark step at this state, decoupled from the poses
                const double id = 1.0 / det;
                const double i2[3] = {(hv[3] * hv[7] - hv[4] * hv[6]) * id, (hv[1] * hv[6] - hv[0] * hv[7]) * id,
                                      (hv[0] * hv[4] - hv[1] * hv[3]) * id};
                const double step = -(i2[0] * gl3[0].v + i2[1] * gl3[1].v + i2[2] * gl3[2].v);
                frozen = !(lm[2].v + step > 1e-9);
            }
            if (lane == 0) sc[NT_FROZEN] = frozen ? 1.0 : 0.0;
            var = var && !frozen;
        } else {
            var = var && sc[NT_FROZEN] == 0.0;
        }
        if (lane == 0) {
            if (mode != NT_MODE_THETA)
                for (int i = 0; i < 6; ++i) {
                    atomicAdd(&nt.gp[6 * h + i], gh[i].v);
                    atomicAdd(&nt.hp[6 * h + i], gh[i].e + mu * gnh[i]);
                }
            if (mode == NT_MODE_GRAD)
                for (int i = 0; i < 3; ++i) sc[NT_B + i] = var ? -gl3[i].v : 0.0;
            else if (mode == NT_MODE_HV)
                for (int i = 0; i < 3; ++i) sc[NT_HP + i] = var ? gl3[i].e + mu * gnl[i] : 0.0;
        }
        __syncwarp();
    }
}

// Gauss-Newton preconditioner, part 1: y = r_p - sum_l Hpl Hll^-1 r_l (r_p = sh.g, r_l = NT_R) -> sh.y
__device__ void pass_pre_a(BaShared& sh, const XcbBaWindows& d, WarpLm<double>* wls, const double* lsc)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int n = sh.w.n;
    WarpLm<double>& wl = wls[wid];
    for (int q = threadIdx.x; q < n; q += blockDim.x) sh.y[q] = sh.g[q];
    __syncthreads();
    double cdummy = 0.0;
    for (int l = wid; l < sh.w.L; l += BA_WARPS) {
        const int gl = sh.w.lm0 + l;
        if (!d.lm_mask[gl]) continue;
        double Hll[9], bl[3];
        int nt;
        const bool ok = lin_landmark<double>(sh, d, sh.g64, l, 0.0, d.lmp, wl, Hll, bl, &nt, &cdummy);
        if (ok && nt && lsc[(size_t)gl * NT_LM_STRIDE + NT_FROZEN] == 0.0) {
            double Hi[9];
            inv3<double>(Hll, Hi);
            const double* r = lsc + (size_t)gl * NT_LM_STRIDE + NT_R;
            double u[3];
            for (int i = 0; i < 3; ++i) u[i] = Hi[i * 3] * r[0] + Hi[i * 3 + 1] * r[1] + Hi[i * 3 + 2] * r[2];
            for (int q = lane; q < nt * 6; q += 32) {
                const int a = q / 6, j = q % 6;
                atomicAdd(&sh.y[6 * wl.ts[a] + j],
                          -(wl.Hlp[a][j] * u[0] + wl.Hlp[a][6 + j] * u[1] + wl.Hlp[a][12 + j] * u[2]));
            }
        }
        __syncwarp();
    }
    __syncthreads();
}

// part 2: z_l = Hll^-1 (r_l - Hlp delta_p) (delta_p = sh.y) -> NT_Z (zero for landmarks that are not variables)
__device__ void pass_pre_b(BaShared& sh, const XcbBaWindows& d, WarpLm<double>* wls, double* lsc)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpLm<double>& wl = wls[wid];
    double cdummy = 0.0;
    for (int l = wid; l < sh.w.L; l += BA_WARPS) {
        const int gl = sh.w.lm0 + l;
        if (!d.lm_mask[gl]) continue;
        double Hll[9], bl[3];
        int nt;
        const bool ok = lin_landmark<double>(sh, d, sh.g64, l, 0.0, d.lmp, wl, Hll, bl, &nt, &cdummy);
        if (lane == 0) {
            double* sc = lsc + (size_t)gl * NT_LM_STRIDE;
            if (!ok || sc[NT_FROZEN] != 0.0) {
                sc[NT_Z] = sc[NT_Z + 1] = sc[NT_Z + 2] = 0.0;
            } else {
                double Hi[9];
                inv3<double>(Hll, Hi);
                double v[3] = {sc[NT_R], sc[NT_R + 1], sc[NT_R + 2]};
                for (int a = 0; a < nt; ++a) {
                    const int s = wl.ts[a];
                    for (int i = 0; i < 3; ++i) {
                        double acc = 0.0;
                        for (int j = 0; j < 6; ++j) acc += wl.Hlp[a][i * 6 + j] * sh.y[6 * s + j];
                        v[i] -= acc;
                    }
                }
                for (int i = 0; i < 3; ++i) sc[NT_Z + i] = Hi[i * 3] * v[0] + Hi[i * 3 + 1] * v[1] + Hi[i * 3 + 2] * v[2];
            }
        }
        __syncwarp();
    }
    __syncthreads();
}

// the Gauss-Newton reduced system at the current state (no damping but 1e-12 / 1e-9 regularisation), held slot
// identity, Cholesky in S64 -> 0 or -1 (not positive definite)
__device__ int nt_gn_factor(BaShared& sh, const XcbBaWindows& d, double* S64, WarpLm<double>* wl64, const double* lsc)
{
    const int n = sh.w.n, tid = threadIdx.x;
    if (tid == 0) sh.lam = 0.0;
    for (int q = tid; q < n * (n + 1) / 2; q += blockDim.x) S64[q] = 0.0;
    for (int q = tid; q < n; q += blockDim.x) sh.y[q] = 0.0;
    __syncthreads();
    pass_build<double, true>(sh, d, sh.g64, S64, sh.y, wl64, nullptr, lsc);
    __syncthreads();
    const int hs = sh.w.hold;
    if (hs >= 0 && hs < sh.w.P) {
        for (int q = tid; q < 6 * n; q += blockDim.x) {
            const int i = 6 * hs + q / n, j = q % n;
            S64[i >= j ? tri(i, j) : tri(j, i)] = 0.0;
        }
        __syncthreads();
        for (int q = tid; q < 6; q += blockDim.x) S64[tri(6 * hs + q, 6 * hs + q)] = 1.0;
        __syncthreads();
    }
    for (int q = tid; q < n; q += blockDim.x) S64[tri(q, q)] += 1e-9;
    __syncthreads();
    return chol_factor(S64, n);
}

// sum over the window's variables of a_p b_p (poses, the held slot excluded) + a_l b_l (scratch offsets oa, ob)
// (poses = false: the landmark part only; the landmarks of this CTA's slice lb..le)
__device__ double nt_dot(BaShared& sh, NtShared& nt, const double* pa, const double* pb, const double* lsc, int oa,
                         int ob, bool poses = true)
{
    const int tid = threadIdx.x, n = sh.w.n;
    double s = 0.0;
    for (int q = tid; q < n && poses; q += blockDim.x)
        if (!held(sh, q)) s += pa[q] * pb[q];
    for (int l = sh.lb + tid; l < sh.le; l += blockDim.x) {
        const double* sc = lsc + (size_t)(sh.w.lm0 + l) * NT_LM_STRIDE;
        s += sc[oa] * sc[ob] + sc[oa + 1] * sc[ob + 1] + sc[oa + 2] * sc[ob + 2];
    }
    s = warp_sum(s);
    __syncthreads();
    if (tid == 0) nt.red2 = 0.0;
    __syncthreads();
    if ((tid & 31) == 0) atomicAdd(&nt.red2, s);
    __syncthreads();
    return nt.red2;
}

// Gauss-Newton preconditioner: z = M^-1 r (r: sh.g, NT_R -> z: sh.y, NT_Z)
__device__ void nt_precond(BaShared& sh, const XcbBaWindows& d, double* S64, WarpLm<double>* wl64, double* lsc)
{
    pass_pre_a(sh, d, wl64, lsc);
    for (int q = threadIdx.x; q < sh.w.n; q += blockDim.x)
        if (held(sh, q)) sh.y[q] = 0.0;
    __syncthreads();
    chol_solve(S64, sh.w.n, sh.y);
    pass_pre_b(sh, d, wl64, lsc);
}

// H x = b (b_p = sh.rhs, b_l = NT_B) by conjugate gradients preconditioned with the Gauss-Newton system (its factor in
// S64): the adjoint's fallback where the exact reduced system is not positive definite.  -> x (sh.dmp, NT_X); the
// final relative residual; *iters_out the iterations; *neg set if a non-positive curvature p^T H p was met (the state
// is not a strict minimum).  The landmarks of the slice lb..le (the whole window on the fallback's single CTA).
__device__ double nt_solve_exact(BaShared& sh, NtShared& nt, const XcbBaWindows& d, double* S64, unsigned char* dsm,
                                 double* lsc, int maxit, double tol, int* iters_out, int* neg)
{
    const int n = sh.w.n, tid = threadIdx.x;
    WarpLm<double>* wl64 = (WarpLm<double>*)(dsm + ba_off_x(n));
    SlotGeo<Dual>* Gd = (SlotGeo<Dual>*)(dsm + ba_off_x(n));
    for (int q = tid; q < n; q += blockDim.x) { sh.dmp[q] = 0.0; sh.g[q] = held(sh, q) ? 0.0 : sh.rhs[q]; }
    for (int l = tid; l < sh.w.L; l += blockDim.x) {
        double* sc = lsc + (size_t)(sh.w.lm0 + l) * NT_LM_STRIDE;
        for (int i = 0; i < 3; ++i) { sc[NT_X + i] = 0.0; sc[NT_R + i] = sc[NT_B + i]; }
    }
    __syncthreads();
    const double bnorm = sqrt(nt_dot(sh, nt, sh.g, sh.g, lsc, NT_R, NT_R));
    *neg = 0;
    double rel = 0.0;
    int it = 0;
    if (bnorm > 0.0) {
        nt_precond(sh, d, S64, wl64, lsc);
        for (int q = tid; q < n; q += blockDim.x) sh.dx[q] = sh.y[q];
        for (int l = tid; l < sh.w.L; l += blockDim.x) {
            double* sc = lsc + (size_t)(sh.w.lm0 + l) * NT_LM_STRIDE;
            for (int i = 0; i < 3; ++i) sc[NT_P + i] = sc[NT_Z + i];
        }
        __syncthreads();
        double rz = nt_dot(sh, nt, sh.g, sh.y, lsc, NT_R, NT_Z);
        rel = 1.0;
        for (it = 0; it < maxit; ++it) {
            for (int q = tid; q < n; q += blockDim.x) { nt.gp[q] = 0.0; nt.hp[q] = 0.0; }
            __syncthreads();
            slot_geo_dual(sh, sh.dx, *Gd);
            pass_dual(sh, nt, d, *Gd, NT_MODE_HV, lsc, nullptr, nullptr);
            __syncthreads();
            const double pAp = nt_dot(sh, nt, sh.dx, nt.hp, lsc, NT_P, NT_HP);
            if (!(pAp > 0.0)) { *neg = 1; break; }
            const double alpha = rz / pAp;
            for (int q = tid; q < n; q += blockDim.x) {
                if (held(sh, q)) continue;
                sh.dmp[q] += alpha * sh.dx[q];
                sh.g[q] -= alpha * nt.hp[q];
            }
            for (int l = tid; l < sh.w.L; l += blockDim.x) {
                double* sc = lsc + (size_t)(sh.w.lm0 + l) * NT_LM_STRIDE;
                for (int i = 0; i < 3; ++i) {
                    sc[NT_X + i] += alpha * sc[NT_P + i];
                    sc[NT_R + i] -= alpha * sc[NT_HP + i];
                }
            }
            __syncthreads();
            rel = sqrt(nt_dot(sh, nt, sh.g, sh.g, lsc, NT_R, NT_R)) / bnorm;
            if (!(rel > tol)) { ++it; break; }
            nt_precond(sh, d, S64, wl64, lsc);
            const double rz_new = nt_dot(sh, nt, sh.g, sh.y, lsc, NT_R, NT_Z);
            const double beta = rz_new / rz;
            rz = rz_new;
            for (int q = tid; q < n; q += blockDim.x) sh.dx[q] = held(sh, q) ? 0.0 : sh.y[q] + beta * sh.dx[q];
            for (int l = tid; l < sh.w.L; l += blockDim.x) {
                double* sc = lsc + (size_t)(sh.w.lm0 + l) * NT_LM_STRIDE;
                for (int i = 0; i < 3; ++i) sc[NT_P + i] = sc[NT_Z + i] + beta * sc[NT_P + i];
            }
            __syncthreads();
        }
    }
    *iters_out = it;
    return rel;
}

// the exact gradient at the current state: -gradient -> sh.rhs (poses, held slot 0) and NT_B (landmarks)
// (the landmarks of this CTA's slice; cl: the pose gradient summed over the cluster)
__device__ void nt_grad(BaShared& sh, NtShared& nt, const XcbBaWindows& d, unsigned char* dsm, double* lsc,
                        bool upd, bool cl = false)
{
    const int n = sh.w.n, tid = threadIdx.x;
    SlotGeo<Dual>* Gd = (SlotGeo<Dual>*)(dsm + ba_off_x(n));
    for (int q = tid; q < n; q += blockDim.x) { sh.dx[q] = 0.0; nt.gp[q] = 0.0; nt.hp[q] = 0.0; }
    for (int l = sh.lb + tid; l < sh.le; l += blockDim.x)
        for (int i = 0; i < NT_FROZEN; ++i) lsc[(size_t)(sh.w.lm0 + l) * NT_LM_STRIDE + i] = 0.0;
    __syncthreads();
    slot_geo_dual(sh, sh.dx, *Gd);
    pass_dual(sh, nt, d, *Gd, NT_MODE_GRAD, lsc, nullptr, nullptr, 0.0, upd);
    __syncthreads();
    if (cl) cl_sum_array(nt.gp, n);
    for (int q = tid; q < n; q += blockDim.x) sh.rhs[q] = held(sh, q) ? 0.0 : -nt.gp[q];
    __syncthreads();
}

// max-norm of the gradient at the last nt_grad (sh.rhs for the poses, NT_B for the landmark variables)
__device__ double nt_gmax(BaShared& sh, NtShared& nt, const double* lsc)
{
    const int tid = threadIdx.x, n = sh.w.n;
    double gm = 0.0;
    for (int q = tid; q < n; q += blockDim.x) gm = fmax(gm, fabs(sh.rhs[q]));
    for (int l = sh.lb + tid; l < sh.le; l += blockDim.x)
        for (int i = 0; i < 3; ++i) gm = fmax(gm, fabs(lsc[(size_t)(sh.w.lm0 + l) * NT_LM_STRIDE + NT_B + i]));
    for (int o = 16; o > 0; o >>= 1) gm = fmax(gm, __shfl_xor_sync(0xffffffffu, gm, o));
    __syncthreads();
    if (tid == 0) nt.red2 = 0.0;
    __syncthreads();
    if ((tid & 31) == 0) atomicMax((unsigned long long*)&nt.red2, (unsigned long long)__double_as_longlong(gm));
    __syncthreads();
    const double r = nt.red2;
    __syncthreads();
    return r;
}

// =====================================================================================================================
// Landmark-eliminated Newton (the polish).  Near the LM's fixed point the exact Hessian is indefinite in a few landmark
// blocks (landmarks with an outlier row: the second-order term of k|e| outweighs the block's Gauss-Newton curvature),
// and a Newton or trust-region iteration on the joint system stalls there.  Each step therefore
//   (1) moves every variable landmark to the minimum of its own cost with the poses fixed (Newton on its exact 3x3
//       block with Levenberg-Marquardt damping);
//   (2) builds the exact reduced system S = Hpp - Hpl Hll^-1 Hlp over the landmarks whose exact block is positive
//       definite and solves S dp = -g_p (the gradient of the cost with every landmark at its own minimum) by Cholesky,
//       Levenberg-Marquardt damped (mu |S_ii|) while S is not positive definite or the cost does not decrease;
//   (3) moves those landmarks to first order with the poses (dl = -Hll^-1 Hlp dp), runs (1) at the trial poses, and
//       keeps the trial if the cost decreased.
// Second derivatives come from dual numbers: Hll and Hlp from three landmark directions per landmark, Hpp from one pass
// per pose direction over the row groups that have that slot as host or target.
// =====================================================================================================================
#define NT_INNER 32             // Newton iterations per landmark in (1)
#define NT_RETRY 10             // damping increases per step
#define NT_SC (BA_MAXN * (BA_MAXN + 1) / 2)     // doubles of one reduced-system copy
#define NT_CL_MAX 4             // CTAs per window (thread-block cluster); each keeps its own copy
#define NT_RHO_INF 1e-7         // a landmark whose inverse depth falls below this has its minimum at infinity
// polish records in the landmark scratch (the conjugate-gradient slots are free during the polish)
#define NR_HI 0                 // Hll^-1, symmetric: 00 01 02 11 12 22; entry 0 is 0 for a landmark held this step
#define NR_BK 9                 // the landmark before the trial step

// dynamic shared memory of the Newton kernel: [S, packed lower][WarpLm<double> x BA_WARPS | SlotGeo<Dual> of a
// direction][SlotGeo<Dual> with zero tangents]
static __host__ __device__ __forceinline__ size_t nt_x_bytes(int n)
{
    size_t x = ba_x_bytes(n);
    const size_t q = ((sizeof(SlotGeo<Dual>) + 15) & ~(size_t)15) + (size_t)BA_WARPS * 256 * sizeof(int);
    if (q > x) x = q;                   // a direction's geometry and the column passes' row queues
    return (x + 15) & ~(size_t)15;
}

// the Huber cost of landmark gl's row groups at landmark state lm (the geometry G), as pass_cost counts it (1e6 for a
// row group whose point is not in front of its camera), plus its inverse-depth prior; identical on every lane
__device__ double lm_cost(const BaShared& sh, const XcbBaWindows& d, const SlotGeo<double>& G, int gl, int h,
                          const double lm[3])
{
    const int lane = threadIdx.x & 31;
    double c = 0.0;
    for (int k = d.lm_ob[gl] + lane; k < d.lm_ob[gl + 1]; k += 32) {
        if (!d.ob_valid[k] || (unsigned)d.ob_pose[k] >= (unsigned)sh.w.P) continue;
        double ob[OB_N];
        if (!obs_lin<double>(sh.w, G, lm, h, d.ob_pose[k], d.ob_cam[k], d.ob_z + 2 * k, d.ob_isig[k], ob, 0)) {
            c += 1e6;
            continue;
        }
        double wt, cc;
        huber_w<double>(sqrt(ob[0] * ob[0] + ob[1] * ob[1]), sh.w.hk, &wt, &cc);
        c += cc;
    }
    c = warp_sum(c);
    if (d.rho_isig[gl] > 0.0) {
        double r0 = (lm[2] - d.rho_meas[gl]) * d.rho_isig[gl], wt, cc;
        huber_w<double>(fabs(r0), sh.w.hk, &wt, &cc);
        c += cc;
    }
    return c;
}

// the exact landmark block of landmark gl at lm, the poses fixed (G0: the geometry with zero tangents): g (3) the
// gradient, H (9) the exact Hessian block (symmetrised), hv (9) its Gauss-Newton block (the variable test of
// pass_dual), *nobs the evaluable row groups; prior included; identical on every lane
__device__ void lm_exact(const BaShared& sh, const XcbBaWindows& d, const SlotGeo<Dual>& G0, int gl, int h,
                         const double lm[3], double g[3], double H[9], double hv[9], int* nobs)
{
    const int lane = threadIdx.x & 31;
    const int k0 = d.lm_ob[gl], nob = lm_rows(d, gl);
    for (int i = 0; i < 3; ++i) g[i] = 0.0;
    for (int i = 0; i < 9; ++i) { H[i] = 0.0; hv[i] = 0.0; }
    int ok = 0;
    if (lane < nob) {
        const int k = k0 + lane, t = d.ob_pose[k];
        if (d.ob_valid[k] && (unsigned)t < (unsigned)sh.w.P) {
            for (int i = 0; i < 3; ++i) {
                const Dual lmd[3] = {Dual(lm[0], i == 0 ? 1.0 : 0.0), Dual(lm[1], i == 1 ? 1.0 : 0.0),
                                     Dual(lm[2], i == 2 ? 1.0 : 0.0)};
                Dual ob[OB_N];
                if (!obs_lin<Dual>(sh.w, G0, lmd, h, t, d.ob_cam[k], d.ob_z + 2 * k, Dual(d.ob_isig[k]), ob, 2)) break;
                const Dual en = sqrt(ob[OB_E] * ob[OB_E] + ob[OB_E + 1] * ob[OB_E + 1]);
                Dual wt, cc;
                huber_w<Dual>(en, Dual(sh.w.hk), &wt, &cc);
                for (int r = 0; r < 3; ++r) {
                    const Dual gr = wt * (ob[OB_JL + r] * ob[OB_E] + ob[OB_JL + 3 + r] * ob[OB_E + 1]);
                    H[r * 3 + i] = gr.e;
                    if (i == 0) g[r] = gr.v;
                }
                if (i == 0) {
                    ok = 1;
                    for (int p = 0; p < 3; ++p)
                        for (int q = 0; q < 3; ++q)
                            hv[p * 3 + q] = wt.v * (ob[OB_JL + p].v * ob[OB_JL + q].v +
                                                    ob[OB_JL + 3 + p].v * ob[OB_JL + 3 + q].v);
                }
            }
        }
    }
    *nobs = __popc(__ballot_sync(0xffffffffu, ok != 0));
    for (int i = 0; i < 3; ++i) g[i] = warp_sum(g[i]);
    for (int i = 0; i < 9; ++i) { H[i] = warp_sum(H[i]); hv[i] = warp_sum(hv[i]); }
    if (d.rho_isig[gl] > 0.0) {
        // prior huber(|(rho - rho_meas) ris|): gradient wt ris r0, exact curvature ris^2 inside the kink, 0 outside
        const double ris = d.rho_isig[gl], r0 = (lm[2] - d.rho_meas[gl]) * ris;
        double wt, cc;
        huber_w<double>(fabs(r0), sh.w.hk, &wt, &cc);
        g[2] += wt * ris * r0;
        if (fabs(r0) <= sh.w.hk) H[8] += ris * ris;
        hv[8] += wt * ris * ris;
    }
    for (int p = 0; p < 3; ++p)
        for (int q = p + 1; q < 3; ++q) {
            const double m = 0.5 * (H[p * 3 + q] + H[q * 3 + p]);
            H[p * 3 + q] = m;
            H[q * 3 + p] = m;
        }
}

// pass_dual's variable test on the Gauss-Newton block
__device__ __forceinline__ bool lm_var(const double hv0[9], int nobs)
{
    double hv[9];
    for (int i = 0; i < 9; ++i) hv[i] = hv0[i];
    for (int i = 0; i < 3; ++i) hv[i * 4] += 1e-12;
    const double det = hv[0] * (hv[4] * hv[8] - hv[5] * hv[7]) - hv[1] * (hv[3] * hv[8] - hv[5] * hv[6]) +
                       hv[2] * (hv[3] * hv[7] - hv[4] * hv[6]);
    const double tr = hv[0] + hv[4] + hv[8];
    return nobs > 0 && det > 1e-18 * tr * tr * tr && isfinite(det);
}

// (H + tau I)^-1 of a symmetric 3x3 block for the first tau of tau0, 1e-9 tr, 1e-8 tr, ... (none below tau0, none
// above 1e3 tr) that makes it positive definite by Cholesky (pivots above 1e-13 tr); the inverse as 00 01 02 11 12 22.
// -> tau, or -1 when none does
__device__ double spd_inv3(const double H[9], double tau0, double Hi[6])
{
    const double tr = fabs(H[0]) + fabs(H[4]) + fabs(H[8]);
    if (!(tr > 0.0) || !isfinite(tr) || !(tau0 >= 0.0)) return -1.0;
    double tau = tau0;
    for (int a = 0; a < 16 && tau <= 1e3 * tr; ++a) {
        const double eps = 1e-13 * tr;
        const double d0 = H[0] + tau;
        if (d0 > eps) {
            const double l00 = sqrt(d0), l10 = H[3] / l00, l20 = H[6] / l00;
            const double d1 = H[4] + tau - l10 * l10;
            if (d1 > eps) {
                const double l11 = sqrt(d1), l21 = (H[7] - l20 * l10) / l11;
                const double d2 = H[8] + tau - l20 * l20 - l21 * l21;
                if (d2 > eps) {
                    const double l22 = sqrt(d2);
                    // L^-1 (lower), then (L L^T)^-1 = L^-T L^-1
                    const double m00 = 1.0 / l00, m11 = 1.0 / l11, m22 = 1.0 / l22;
                    const double m10 = -l10 * m00 * m11;
                    const double m21 = -l21 * m11 * m22;
                    const double m20 = -(l20 * m00 + l21 * m10) * m22;
                    Hi[0] = m00 * m00 + m10 * m10 + m20 * m20;
                    Hi[1] = m10 * m11 + m20 * m21;
                    Hi[2] = m20 * m22;
                    Hi[3] = m11 * m11 + m21 * m21;
                    Hi[4] = m21 * m22;
                    Hi[5] = m22 * m22;
                    return tau;
                }
            }
        }
        tau = tau > 0.0 ? 10.0 * tau : 1e-9 * tr;
    }
    return -1.0;
}

__device__ __forceinline__ void sym3_mv(const double Hi[6], const double v[3], double o[3])
{
    o[0] = Hi[0] * v[0] + Hi[1] * v[1] + Hi[2] * v[2];
    o[1] = Hi[1] * v[0] + Hi[3] * v[1] + Hi[4] * v[2];
    o[2] = Hi[2] * v[0] + Hi[4] * v[1] + Hi[5] * v[2];
}

// (1) every variable landmark that is not held constant to the minimum of its own cost, the poses fixed (the state in
// sh.Rwb / sh.pwb: sh.g64 and G0 built from it).  Newton on the exact block with Levenberg-Marquardt damping: the
// shift is the smallest of the spd_inv3 sequence that makes the block positive definite (0 where it is) plus mu tr,
// mu / 10 after a decrease and x 10 after none; a step at the cost's rounding level is kept unless the cost rose.
// The cost of every landmark at its final state -> sh.red (per warp: block_sum_red gives the window's).
__device__ void pass_inner(BaShared& sh, const XcbBaWindows& d, const SlotGeo<Dual>& G0, const double* lsc)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double ctot = 0.0;
    for (int l = sh.lb + wid; l < sh.le; l += BA_WARPS) {
        const int gl = sh.w.lm0 + l;
        if (!d.lm_mask[gl]) continue;
        const int h = d.lm_host[gl];
        if ((unsigned)h >= (unsigned)sh.w.P) continue;
        double lm[3] = {d.lmp[3 * gl], d.lmp[3 * gl + 1], d.lmp[3 * gl + 2]};
        double c = lm_cost(sh, d, sh.g64, gl, h, lm);
        const bool frozen = lsc[(size_t)gl * NT_LM_STRIDE + NT_FROZEN] != 0.0;
        bool moved = false;
        double mu = 0.0;
        for (int it = 0; it < NT_INNER && !frozen; ++it) {
            double g[3], H[9], hv[9], Hi[6], dl[3];
            int nobs;
            lm_exact(sh, d, G0, gl, h, lm, g, H, hv, &nobs);
            if (!lm_var(hv, nobs)) break;
            const double tr = fabs(H[0]) + fabs(H[4]) + fabs(H[8]);
            const double tau0 = spd_inv3(H, 0.0, Hi);
            if (tau0 < 0.0) break;
            bool acc = false;
            double dec = 0.0;
            for (int att = 0; att < 12 && !acc; ++att) {
                if (spd_inv3(H, tau0 + mu * tr, Hi) < 0.0) break;
                sym3_mv(Hi, g, dl);
                dec = g[0] * dl[0] + g[1] * dl[1] + g[2] * dl[2];      // -(g.step), the step being -dl
                double tr3[3];
                for (int i = 0; i < 3; ++i) tr3[i] = lm[i] - dl[i];
                if (dec > 0.0 && tr3[2] > 1e-9 && isfinite(tr3[0]) && isfinite(tr3[1]) && isfinite(tr3[2])) {
                    const double c1 = lm_cost(sh, d, sh.g64, gl, h, tr3);
                    const double noise = 1e-12 * fabs(c);
                    acc = c1 <= c - 1e-4 * dec || (0.5 * dec <= noise && c1 <= c + noise);
                    if (acc) {
                        for (int i = 0; i < 3; ++i) lm[i] = tr3[i];
                        c = c1;
                        moved = true;
                    }
                }
                if (acc) mu = mu > 1e-9 ? 0.1 * mu : 0.0;
                else mu = mu > 0.0 ? 10.0 * mu : 1e-6;
            }
            if (!acc || 0.5 * dec <= 1e-12 * fabs(c)) break;      // no decrease, or converged to rounding level
        }
        if (moved && lane < 3) d.lmp[3 * gl + lane] = lm[lane];
        __syncwarp();
        if (lane == 0) ctot += c;
    }
    ctot = warp_sum(ctot);
    if (lane == 0) sh.red[wid] = ctot;
}

// Hpp column c = 6 s + j (G: the geometry moved along e_c): every row group with slot s as its host or its target
// adds the dual part of its pose gradient, d(w J^T e)/dx_c, to the rows >= c of S (packed lower).  A row group's
// terms need no sum over its landmark, so the warp queues the row groups that touch slot s (2-4 of a landmark's
// rows) in wq (this warp's 4 x 64 ints) and evaluates them 32 at a time, a lane each.
__device__ __forceinline__ void hpp_row(const BaShared& sh, const XcbBaWindows& d, const SlotGeo<Dual>& G, int c,
                                        double* S, int k, int gl, int h, int t)
{
    const Dual lm[3] = {Dual(d.lmp[3 * gl]), Dual(d.lmp[3 * gl + 1]), Dual(d.lmp[3 * gl + 2])};
    Dual ob[OB_N];
    if (!obs_lin<Dual>(sh.w, G, lm, h, t, d.ob_cam[k], d.ob_z + 2 * k, Dual(d.ob_isig[k]), ob, 1)) return;
    const Dual en = sqrt(ob[OB_E] * ob[OB_E] + ob[OB_E + 1] * ob[OB_E + 1]);
    Dual wt, cc;
    huber_w<Dual>(en, Dual(sh.w.hk), &wt, &cc);
    for (int i = 0; i < 6; ++i) {
        const Dual gt = wt * (ob[OB_JT + i] * ob[OB_E] + ob[OB_JT + 6 + i] * ob[OB_E + 1]);
        const Dual gh = wt * (obj(ob, OB_JH, 0, i) * ob[OB_E] + obj(ob, OB_JH, 1, i) * ob[OB_E + 1]);
        const int rt = 6 * t + i, rh = 6 * h + i;
        if (rt >= c) atomicAdd(&S[tri(rt, c)], gt.e);
        if (rh >= c) atomicAdd(&S[tri(rh, c)], gh.e);
    }
}

__device__ void pass_hpp_col(BaShared& sh, const XcbBaWindows& d, const SlotGeo<Dual>& G, int s, int c, double* S,
                             int* wq)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int* qk = wq;
    int* ql = wq + 64;
    int* qh = wq + 128;
    int* qt = wq + 192;
    int nq = 0;                                          // queued row groups (the same on every lane)
    for (int l = sh.lb + wid; l < sh.le; l += BA_WARPS) {
        const int gl = sh.w.lm0 + l;
        if (!d.lm_mask[gl]) continue;
        const int h = d.lm_host[gl];
        if ((unsigned)h >= (unsigned)sh.w.P) continue;
        const int k0 = d.lm_ob[gl], nob = lm_rows(d, gl);
        int t = -1;
        bool ev = false;
        if (lane < nob) {
            t = d.ob_pose[k0 + lane];
            ev = d.ob_valid[k0 + lane] && (unsigned)t < (unsigned)sh.w.P && t != h && (h == s || t == s);
        }
        const unsigned m = __ballot_sync(0xffffffffu, ev);
        if (!m) continue;
        if (ev) {
            const int pos = nq + __popc(m & ((1u << lane) - 1u));
            qk[pos] = k0 + lane; ql[pos] = gl; qh[pos] = h; qt[pos] = t;
        }
        nq += __popc(m);
        __syncwarp();
        if (nq >= 32) {
            hpp_row(sh, d, G, c, S, qk[lane], ql[lane], qh[lane], qt[lane]);
            __syncwarp();
            const int rest = nq - 32;
            int a0 = 0, a1 = 0, a2 = 0, a3 = 0;
            if (lane < rest) { a0 = qk[32 + lane]; a1 = ql[32 + lane]; a2 = qh[32 + lane]; a3 = qt[32 + lane]; }
            __syncwarp();
            if (lane < rest) { qk[lane] = a0; ql[lane] = a1; qh[lane] = a2; qt[lane] = a3; }
            __syncwarp();
            nq = rest;
        }
    }
    if (lane < nq) hpp_row(sh, d, G, c, S, qk[lane], ql[lane], qh[lane], qt[lane]);
    __syncwarp();
}

// (2) the landmark terms of the exact reduced system at the current state (G0: zero tangents): per landmark whose exact
// block is positive definite (a landmark whose block is not is not at a minimum of its own cost, and this step holds
// it where it is: no Schur term, no step, its rows still in Hpp and the pose gradient), its Hlp blocks from the three
// landmark directions, S -= Hpl Hll^-1 Hlp (S holds Hpp from the column passes); for every landmark nt.gp += its pose
// gradient; records Hll^-1 in the scratch.  upd: a variable landmark whose minimum lies at infinity (rho below
// NT_RHO_INF, or its own Newton step taking rho to <= 1e-9) is flagged constant here (builds run at accepted states).
// -> the warp's max |g_l| over the variable landmarks (held this step or not) in sh.red.
__device__ void pass_xbuild(BaShared& sh, NtShared& nt, const XcbBaWindows& d, const SlotGeo<Dual>& G0, double* S,
                            WarpLm<double>* wls, double* lsc, bool upd)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpLm<double>& wl = wls[wid];
    double gmax = 0.0;
    for (int l = sh.lb + wid; l < sh.le; l += BA_WARPS) {
        const int gl = sh.w.lm0 + l;
        if (!d.lm_mask[gl]) continue;
        const int h = d.lm_host[gl];
        if ((unsigned)h >= (unsigned)sh.w.P) continue;
        double* sc = lsc + (size_t)gl * NT_LM_STRIDE;
        const int k0 = d.lm_ob[gl], nob = lm_rows(d, gl);
        const double lmv[3] = {d.lmp[3 * gl], d.lmp[3 * gl + 1], d.lmp[3 * gl + 2]};
        int mt = -1, ok = 0;
        double g[3] = {0.0, 0.0, 0.0}, hv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int i = 0; i < 3; ++i) {
            // lane = row group: the dual parts of its gradient along landmark direction i -> wl.ob[lane][0..15)
            // (landmark 3, host pose 6, target pose 6); the value parts on the first direction
            double* st = wl.ob[lane];
            for (int q = 0; q < 15; ++q) st[q] = 0.0;
            if (lane < nob) {
                const int k = k0 + lane, t = d.ob_pose[k];
                if (d.ob_valid[k] && (unsigned)t < (unsigned)sh.w.P) {
                    const Dual lmd[3] = {Dual(lmv[0], i == 0 ? 1.0 : 0.0), Dual(lmv[1], i == 1 ? 1.0 : 0.0),
                                         Dual(lmv[2], i == 2 ? 1.0 : 0.0)};
                    Dual ob[OB_N];
                    if (obs_lin<Dual>(sh.w, G0, lmd, h, t, d.ob_cam[k], d.ob_z + 2 * k, Dual(d.ob_isig[k]), ob, 1)) {
                        const Dual en = sqrt(ob[OB_E] * ob[OB_E] + ob[OB_E + 1] * ob[OB_E + 1]);
                        Dual wt, cc;
                        huber_w<Dual>(en, Dual(sh.w.hk), &wt, &cc);
                        for (int r = 0; r < 3; ++r) {
                            const Dual gr = wt * (ob[OB_JL + r] * ob[OB_E] + ob[OB_JL + 3 + r] * ob[OB_E + 1]);
                            st[r] = gr.e;
                            if (i == 0) g[r] = gr.v;
                        }
                        if (t != h)
                            for (int q = 0; q < 6; ++q) {
                                const Dual gh = wt * (obj(ob, OB_JH, 0, q) * ob[OB_E] + obj(ob, OB_JH, 1, q) * ob[OB_E + 1]);
                                const Dual gt = wt * (ob[OB_JT + q] * ob[OB_E] + ob[OB_JT + 6 + q] * ob[OB_E + 1]);
                                st[3 + q] = gh.e;
                                st[9 + q] = gt.e;
                                if (i == 0) {
                                    atomicAdd(&nt.gp[6 * h + q], gh.v);
                                    atomicAdd(&nt.gp[6 * t + q], gt.v);
                                }
                            }
                        if (i == 0) {
                            ok = 1;
                            mt = t;
                            for (int p = 0; p < 3; ++p)
                                for (int q = 0; q < 3; ++q)
                                    hv[p * 3 + q] = wt.v * (ob[OB_JL + p].v * ob[OB_JL + q].v +
                                                            ob[OB_JL + 3 + p].v * ob[OB_JL + 3 + q].v);
                        }
                    }
                }
            }
            if (i == 0) {
                // touched slots: the observing keyframes other than the host, plus the host when any exists
                const bool pose = mt >= 0 && mt != h;
                unsigned mine = pose ? (1u << mt) : 0u;
                for (int o = 16; o > 0; o >>= 1) mine |= __shfl_xor_sync(0xffffffffu, mine, o);
                const unsigned tm = mine ? (mine | (1u << h)) : 0u;
                int nt_ = 0;
                for (unsigned m = tm; m; m &= m - 1) {
                    const int s = __ffs(m) - 1;
                    const unsigned om = __ballot_sync(0xffffffffu, pose && (s == h || mt == s));
                    if (lane == 0 && nt_ < BA_MAXT) { wl.ts[nt_] = s; wl.om[nt_] = om; }
                    ++nt_;
                }
                if (nt_ > BA_MAXT) {
                    if (lane == 0) sh.overflow = 1;
                    nt_ = BA_MAXT;
                }
                if (lane == 0) wl.hl[9] = (double)nt_;
            }
            __syncwarp();
            const int ntc = (int)wl.hl[9];
            // column i of Hll (lanes 0..2) and row i of every Hlp block
            if (lane < 3) {
                double acc = 0.0;
                for (int m = 0; m < nob; ++m) acc += wl.ob[m][lane];
                wl.hl[lane * 3 + i] = acc;
            }
            for (int q = lane; q < ntc * 6; q += 32) {
                const int a = q / 6, j = q % 6;
                const int off = wl.ts[a] == h ? 3 : 9;
                double acc = 0.0;
                for (unsigned m = wl.om[a]; m; m &= m - 1) acc += wl.ob[__ffs(m) - 1][off + j];
                wl.Hlp[a][i * 6 + j] = acc;
            }
            __syncwarp();
        }
        const int ntc = (int)wl.hl[9];
        const int nobs = __popc(__ballot_sync(0xffffffffu, ok != 0));
        double H[9];
        for (int q = 0; q < 9; ++q) H[q] = wl.hl[q];
        for (int r = 0; r < 3; ++r) g[r] = warp_sum(g[r]);
        for (int q = 0; q < 9; ++q) hv[q] = warp_sum(hv[q]);
        if (d.rho_isig[gl] > 0.0) {
            const double ris = d.rho_isig[gl], r0 = (lmv[2] - d.rho_meas[gl]) * ris;
            double wt, cc;
            huber_w<double>(fabs(r0), sh.w.hk, &wt, &cc);
            g[2] += wt * ris * r0;
            if (fabs(r0) <= sh.w.hk) H[8] += ris * ris;
            hv[8] += wt * ris * ris;
        }
        for (int p = 0; p < 3; ++p)
            for (int q = p + 1; q < 3; ++q) {
                const double m = 0.5 * (H[p * 3 + q] + H[q * 3 + p]);
                H[p * 3 + q] = m;
                H[q * 3 + p] = m;
            }
        double Hi[6];
        const bool fz = sc[NT_FROZEN] != 0.0, lv = lm_var(hv, nobs);
        const bool pd = spd_inv3(H, 0.0, Hi) == 0.0;
        double u[3] = {0.0, 0.0, 0.0};
        if (pd) sym3_mv(Hi, g, u);                                    // Hll^-1 g_l: the landmark's own Newton step is -u
        const bool inf = upd && !fz && lv && (lmv[2] < NT_RHO_INF || (pd && !(lmv[2] - u[2] > 1e-9)));
        const bool var = !fz && !inf && lv && pd;
        __syncwarp();
        if (inf && lane == 0) sc[NT_FROZEN] = 1.0;
        if (!fz && !inf && lv) gmax = fmax(gmax, fmax(fabs(g[0]), fmax(fabs(g[1]), fabs(g[2]))));
        if (var) {
            for (int q = lane; q < ntc * 18; q += 32) {              // Tb = Hll^-1 Hlp
                const int a = q / 18, e = q % 18, i = e / 6, j = e % 6;
                const double* Hl = wl.Hlp[a];
                const double r0 = i == 0 ? Hi[0] : (i == 1 ? Hi[1] : Hi[2]);
                const double r1 = i == 0 ? Hi[1] : (i == 1 ? Hi[3] : Hi[4]);
                const double r2 = i == 0 ? Hi[2] : (i == 1 ? Hi[4] : Hi[5]);
                wl.Tb[a][e] = r0 * Hl[j] + r1 * Hl[6 + j] + r2 * Hl[12 + j];
            }
            __syncwarp();
            const int npair = ntc * (ntc + 1) / 2;
            for (int q = lane; q < npair * 36; q += 32) {
                const int pr = q / 36, e = q % 36, i = e / 6, j = e % 6;
                int a = (int)((sqrtf(8.0f * pr + 1.0f) - 1.0f) * 0.5f);
                while (a * (a + 1) / 2 > pr) --a;
                while ((a + 1) * (a + 2) / 2 <= pr) ++a;
                const int b = pr - a * (a + 1) / 2;
                if (a == b && j > i) continue;
                const double acc = wl.Hlp[a][i] * wl.Tb[b][j] + wl.Hlp[a][6 + i] * wl.Tb[b][6 + j] +
                                   wl.Hlp[a][12 + i] * wl.Tb[b][12 + j];
                atomicAdd(&S[tri(6 * wl.ts[a] + i, 6 * wl.ts[b] + j)], -acc);
            }
            if (lane < 6) sc[NR_HI + lane] = Hi[lane];
        } else if (lane < 9) {
            sc[lane] = 0.0;
        }
        __syncwarp();
    }
    for (int o = 16; o > 0; o >>= 1) gmax = fmax(gmax, __shfl_xor_sync(0xffffffffu, gmax, o));
    if (lane == 0) sh.red[wid] = gmax;
}

// Hlp dp of landmark gl (G: the geometry moved along dp, the landmark's tangent zero): the dual part of its gradient,
// summed over its row groups; identical on every lane
__device__ void lm_hlp(const BaShared& sh, const XcbBaWindows& d, const SlotGeo<Dual>& G, int gl, int h,
                       const double lmv[3], double u[3])
{
    const int lane = threadIdx.x & 31;
    const int k0 = d.lm_ob[gl], nob = lm_rows(d, gl);
    for (int r = 0; r < 3; ++r) u[r] = 0.0;
    if (lane < nob) {
        const int k = k0 + lane, t = d.ob_pose[k];
        if (d.ob_valid[k] && (unsigned)t < (unsigned)sh.w.P && t != h) {
            const Dual lm[3] = {Dual(lmv[0]), Dual(lmv[1]), Dual(lmv[2])};
            Dual ob[OB_N];
            if (obs_lin<Dual>(sh.w, G, lm, h, t, d.ob_cam[k], d.ob_z + 2 * k, Dual(d.ob_isig[k]), ob, 2)) {
                const Dual en = sqrt(ob[OB_E] * ob[OB_E] + ob[OB_E + 1] * ob[OB_E + 1]);
                Dual wt, cc;
                huber_w<Dual>(en, Dual(sh.w.hk), &wt, &cc);
                for (int r = 0; r < 3; ++r)
                    u[r] = (wt * (ob[OB_JL + r] * ob[OB_E] + ob[OB_JL + 3 + r] * ob[OB_E + 1])).e;
            }
        }
    }
    for (int r = 0; r < 3; ++r) u[r] = warp_sum(u[r]);
}

// Hpl v of landmark gl for a landmark tangent v (G0: zero pose tangents), added to acc (poses; shared atomics)
__device__ void lm_hpl(const BaShared& sh, const XcbBaWindows& d, const SlotGeo<Dual>& G0, int gl, int h,
                       const double lmv[3], const double v[3], double* acc)
{
    const int lane = threadIdx.x & 31;
    const int k0 = d.lm_ob[gl], nob = lm_rows(d, gl);
    if (lane < nob) {
        const int k = k0 + lane, t = d.ob_pose[k];
        if (d.ob_valid[k] && (unsigned)t < (unsigned)sh.w.P && t != h) {
            const Dual lm[3] = {Dual(lmv[0], v[0]), Dual(lmv[1], v[1]), Dual(lmv[2], v[2])};
            Dual ob[OB_N];
            if (obs_lin<Dual>(sh.w, G0, lm, h, t, d.ob_cam[k], d.ob_z + 2 * k, Dual(d.ob_isig[k]), ob, 1)) {
                const Dual en = sqrt(ob[OB_E] * ob[OB_E] + ob[OB_E + 1] * ob[OB_E + 1]);
                Dual wt, cc;
                huber_w<Dual>(en, Dual(sh.w.hk), &wt, &cc);
                for (int q = 0; q < 6; ++q) {
                    const Dual gh = wt * (obj(ob, OB_JH, 0, q) * ob[OB_E] + obj(ob, OB_JH, 1, q) * ob[OB_E + 1]);
                    const Dual gt = wt * (ob[OB_JT + q] * ob[OB_E] + ob[OB_JT + 6 + q] * ob[OB_E + 1]);
                    atomicAdd(&acc[6 * h + q], gh.e);
                    atomicAdd(&acc[6 * t + q], gt.e);
                }
            }
        }
    }
    __syncwarp();
}

// (3) the landmarks' first-order step with the poses, dl = -Hll^-1 Hlp dp (G: the geometry at the current state moved
// along dp), for the landmarks the build kept; every landmark's state is saved to the scratch first (restored when the
// trial is rejected)
__device__ void pass_lstep(BaShared& sh, const XcbBaWindows& d, const SlotGeo<Dual>& G, double* lsc)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int l = sh.lb + wid; l < sh.le; l += BA_WARPS) {
        const int gl = sh.w.lm0 + l;
        if (!d.lm_mask[gl]) continue;
        const int h = d.lm_host[gl];
        if ((unsigned)h >= (unsigned)sh.w.P) continue;
        double* sc = lsc + (size_t)gl * NT_LM_STRIDE;
        const double lmv[3] = {d.lmp[3 * gl], d.lmp[3 * gl + 1], d.lmp[3 * gl + 2]};
        if (lane < 3) sc[NR_BK + lane] = lmv[lane];
        if (!(sc[NR_HI] > 0.0)) { __syncwarp(); continue; }
        double u[3], Hi[6], dl[3];
        lm_hlp(sh, d, G, gl, h, lmv, u);
        for (int q = 0; q < 6; ++q) Hi[q] = sc[NR_HI + q];
        sym3_mv(Hi, u, dl);
        const double nr = lmv[2] - dl[2];
        if (nr > 1e-9 && isfinite(nr) && isfinite(dl[0]) && isfinite(dl[1]) && lane < 3)
            d.lmp[3 * gl + lane] = lmv[lane] - dl[lane];
        __syncwarp();
    }
}

// the adjoint's landmark part from a pose part (G: the geometry moved along it): first = true, x_l = -Hll^-1 Hlp x_p
// -> NT_P (0 for the landmarks the build did not keep); false, the refinement x_l += Hll^-1 (r_l - Hlp dx_p) (r_l in
// NT_Z)
__device__ void pass_adj_l(BaShared& sh, const XcbBaWindows& d, const SlotGeo<Dual>& G, double* lsc, bool first)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int l = sh.lb + wid; l < sh.le; l += BA_WARPS) {
        const int gl = sh.w.lm0 + l;
        double* sc = lsc + (size_t)gl * NT_LM_STRIDE;
        const int h = d.lm_host[gl];
        if (!d.lm_mask[gl] || (unsigned)h >= (unsigned)sh.w.P || !(sc[NR_HI] > 0.0)) {
            if (first && lane < 3) sc[NT_P + lane] = 0.0;
            __syncwarp();
            continue;
        }
        const double lmv[3] = {d.lmp[3 * gl], d.lmp[3 * gl + 1], d.lmp[3 * gl + 2]};
        double u[3], Hi[6], x[3];
        lm_hlp(sh, d, G, gl, h, lmv, u);
        if (!first)
            for (int r = 0; r < 3; ++r) u[r] -= sc[NT_Z + r];
        for (int q = 0; q < 6; ++q) Hi[q] = sc[NR_HI + q];
        sym3_mv(Hi, u, x);
        __syncwarp();
        if (lane < 3) sc[NT_P + lane] = (first ? 0.0 : sc[NT_P + lane]) - x[lane];
        __syncwarp();
    }
}

// acc (poses) += sum over the kept landmarks of Hpl Hll^-1 r_l (r_l in NT_Z)
__device__ void pass_adj_y(BaShared& sh, const XcbBaWindows& d, const SlotGeo<Dual>& G0, const double* lsc,
                           double* acc)
{
    const int wid = threadIdx.x >> 5;
    for (int l = sh.lb + wid; l < sh.le; l += BA_WARPS) {
        const int gl = sh.w.lm0 + l;
        const double* sc = lsc + (size_t)gl * NT_LM_STRIDE;
        const int h = d.lm_host[gl];
        if (!d.lm_mask[gl] || (unsigned)h >= (unsigned)sh.w.P || !(sc[NR_HI] > 0.0)) continue;
        const double lmv[3] = {d.lmp[3 * gl], d.lmp[3 * gl + 1], d.lmp[3 * gl + 2]};
        double Hi[6], v[3];
        for (int q = 0; q < 6; ++q) Hi[q] = sc[NR_HI + q];
        sym3_mv(Hi, sc + NT_Z, v);
        lm_hpl(sh, d, G0, gl, h, lmv, v, acc);
    }
}

// restore every landmark the last pass_lstep saved
__device__ void pass_lrestore(BaShared& sh, const XcbBaWindows& d, const double* lsc)
{
    for (int l = sh.lb + threadIdx.x; l < sh.le; l += blockDim.x) {
        const int gl = sh.w.lm0 + l;
        if (!d.lm_mask[gl] || (unsigned)d.lm_host[gl] >= (unsigned)sh.w.P) continue;
        const double* sc = lsc + (size_t)gl * NT_LM_STRIDE;
        for (int i = 0; i < 3; ++i) d.lmp[3 * gl + i] = sc[NR_BK + i];
    }
    __syncthreads();
}

__device__ double block_max_red(BaShared& sh)
{
    __syncthreads();
    double s = 0.0;
    for (int i = 0; i < BA_WARPS; ++i) s = fmax(s, sh.red[i]);
    __syncthreads();
    return s;
}

// the geometry of the state in sh.Rwb / sh.pwb: sh.g64 and the zero-tangent dual copy G0
__device__ void nt_geo(BaShared& sh, SlotGeo<Dual>& G0)
{
    slot_geo(sh, sh.Rwb, sh.pwb);
    for (int q = threadIdx.x; q < sh.w.n; q += blockDim.x) sh.dx[q] = 0.0;
    __syncthreads();
    slot_geo_dual(sh, sh.dx, G0);
}

// the exact reduced system at the state in sh.Rwb / sh.pwb (G0 built from it): S (packed lower, the held slot's rows
// and columns the identity) from the column passes and pass_xbuild, sh.g the pose gradient (held slot 0).  -> the
// largest |g| over the poses and the variable landmarks
__device__ double nt_xsystem(BaShared& sh, NtShared& nt, const XcbBaWindows& d, unsigned char* dsm, double* lsc,
                             bool upd)
{
    const int n = sh.w.n, P = sh.w.P, tid = threadIdx.x;
    double* S = (double*)dsm;
    WarpLm<double>* wl64 = (WarpLm<double>*)(dsm + ba_off_x(n));
    SlotGeo<Dual>* Gd = (SlotGeo<Dual>*)(dsm + ba_off_x(n));           // aliases wl64: never live together
    SlotGeo<Dual>* G0 = (SlotGeo<Dual>*)(dsm + ba_off_x(n) + nt_x_bytes(n));
    // the column passes' row queues (256 ints per warp) after the direction's geometry, in the warp-scratch region
    int* wq = (int*)(dsm + ba_off_x(n) + ((sizeof(SlotGeo<Dual>) + 15) & ~(size_t)15)) + (tid >> 5) * 256;
    const int ntri = n * (n + 1) / 2;
    for (int q = tid; q < ntri; q += blockDim.x) S[q] = 0.0;
    for (int q = tid; q < n; q += blockDim.x) nt.gp[q] = 0.0;
    __syncthreads();
    for (int c = 0; c < n; ++c) {
        if (held(sh, c)) continue;
        for (int q = tid; q < n; q += blockDim.x) sh.dx[q] = q == c ? 1.0 : 0.0;
        __syncthreads();
        slot_geo_dual(sh, sh.dx, *Gd);
        pass_hpp_col(sh, d, *Gd, c / 6, c, S, wq);
        __syncthreads();
    }
    pass_xbuild(sh, nt, d, *G0, S, wl64, lsc, upd);
    double gml = block_max_red(sh);
    // each CTA of the window's cluster built the terms of its landmark slice
    cl_sum_array(S, ntri);
    cl_sum_array(nt.gp, n);
    gml = cl_reduce(nt, gml, true);
    const int hs = sh.w.hold;
    if (hs >= 0 && hs < P) {
        for (int q = tid; q < 6 * n; q += blockDim.x) {
            const int i = 6 * hs + q / n, j = q % n;
            S[i >= j ? tri(i, j) : tri(j, i)] = 0.0;
        }
        __syncthreads();
        for (int q = tid; q < 6; q += blockDim.x) S[tri(6 * hs + q, 6 * hs + q)] = 1.0;
    }
    // the pose gradient (sh.g) and the largest |g| over the poses and the variable landmarks
    double gm = 0.0;
    for (int q = tid; q < n; q += blockDim.x) {
        const bool hq = held(sh, q);
        sh.g[q] = hq ? 0.0 : nt.gp[q];
        if (!hq) gm = fmax(gm, fabs(nt.gp[q]));
    }
    for (int o = 16; o > 0; o >>= 1) gm = fmax(gm, __shfl_xor_sync(0xffffffffu, gm, o));
    __syncthreads();
    if ((tid & 31) == 0) sh.red[tid >> 5] = gm;
    return fmax(block_max_red(sh), gml);
}

// the landmark-eliminated Newton polish of one window (the state in sh.Rwb / sh.pwb and d.lmp); `steps` bounds the
// Newton steps; it stops early at a gradient max-norm of 1e-10, or after three steps in a row at the cost's rounding
// level that did not halve it.  upd: landmarks whose minimum lies at infinity are flagged constant (pass_xbuild).
// -> status (0, or 2 when no damping gave a decrease); *steps_out, *mu_out the steps taken and the final damping
__device__ int nt_polish(BaShared& sh, NtShared& nt, const XcbBaWindows& d, unsigned char* dsm, double* lsc,
                         double* Sc, int steps, bool upd, int* steps_out, double* mu_out)
{
    const int n = sh.w.n, P = sh.w.P, tid = threadIdx.x;
    double* S = (double*)dsm;
    SlotGeo<Dual>* Gd = (SlotGeo<Dual>*)(dsm + ba_off_x(n));           // aliases the warp scratch of the build
    SlotGeo<Dual>* G0 = (SlotGeo<Dual>*)(dsm + ba_off_x(n) + nt_x_bytes(n));
    const int ntri = n * (n + 1) / 2;
    nt_geo(sh, *G0);
    pass_inner(sh, d, *G0, lsc);
    double c0 = cl_reduce(nt, block_sum_red(sh), false);
    double mu = 0.0, gm_prev = 0.0;
    int st = 0, status = 0, stall = 0;
    bool tiny = false;
    while (st < steps) {
        const double gm = nt_xsystem(sh, nt, d, dsm, lsc, upd);
        // three steps in a row at the cost's rounding level that did not halve the gradient: no further progress
        stall = tiny && gm > 0.5 * gm_prev ? stall + 1 : 0;
        if (gm <= 1e-10 || stall >= 3) break;
        gm_prev = gm;
        for (int q = tid; q < ntri; q += blockDim.x) Sc[q] = S[q];
        __syncthreads();
        bool acc = false;
        for (int r = 0; r < NT_RETRY && !acc; ++r) {
            if (r > 0 || mu > 0.0) {
                for (int q = tid; q < ntri; q += blockDim.x) S[q] = Sc[q];
                __syncthreads();
                for (int q = tid; q < n; q += blockDim.x)
                    if (!held(sh, q)) S[tri(q, q)] += mu * fabs(Sc[tri(q, q)]) + 1e-12;
                __syncthreads();
            }
            if (chol_factor(S, n)) {
                mu = mu > 0.0 ? 10.0 * mu : 1e-6;
                continue;
            }
            for (int q = tid; q < n; q += blockDim.x) sh.dmp[q] = -sh.g[q];
            __syncthreads();
            chol_solve(S, n, sh.dmp);
            // the model's decrease -g.dp / 2 (exact for the undamped step)
            double pr = 0.0;
            for (int q = tid; q < n; q += blockDim.x) pr -= sh.g[q] * sh.dmp[q];
            pr = warp_sum(pr);
            __syncthreads();
            if ((tid & 31) == 0) sh.red[tid >> 5] = pr;
            const double pred = 0.5 * block_sum_red(sh);
            // landmarks to first order (geometry at the current state along dp), then the trial poses
            slot_geo_dual(sh, sh.dmp, *Gd);
            pass_lstep(sh, d, *Gd, lsc);
            __syncthreads();
            for (int s = tid; s < P; s += blockDim.x) {
                double Re[9], R[9];
                for (int i = 0; i < 9; ++i) { R[i] = sh.Rwb[9 * s + i]; sh.R2[9 * s + i] = R[i]; }
                for (int i = 0; i < 3; ++i) sh.p2[3 * s + i] = sh.pwb[3 * s + i];
                if (sh.w.hold == s) continue;
                so3_exp(sh.dmp + 6 * s, Re);
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j)
                        sh.Rwb[9 * s + 3 * i + j] = R[3 * i] * Re[j] + R[3 * i + 1] * Re[3 + j] + R[3 * i + 2] * Re[6 + j];
                for (int i = 0; i < 3; ++i) sh.pwb[3 * s + i] += sh.dmp[6 * s + 3 + i];
            }
            __syncthreads();
            nt_geo(sh, *G0);
            pass_inner(sh, d, *G0, lsc);
            const double c1 = cl_reduce(nt, block_sum_red(sh), false);
            // the cost is a float64 sum of ~1e4 terms: below ~1e-10 of it a decrease is rounding noise, so a step whose
            // predicted decrease is that small is kept unless the cost visibly rose
            const double noise = 1e-10 * fabs(c0);
            tiny = pred <= noise;
            acc = (c1 <= c0 - 1e-4 * pred && pred > 0.0) || (tiny && c1 <= c0 + noise);
            if (acc) {
                c0 = c1;
                mu = mu > 1e-9 ? 0.1 * mu : 0.0;
            } else {
                for (int q = tid; q < P * 9; q += blockDim.x) sh.Rwb[q] = sh.R2[q];
                for (int q = tid; q < P * 3; q += blockDim.x) sh.pwb[q] = sh.p2[q];
                __syncthreads();
                pass_lrestore(sh, d, lsc);
                nt_geo(sh, *G0);
                mu = mu > 0.0 ? 10.0 * mu : 1e-6;
            }
        }
        ++st;
        if (!acc) { status = 2; break; }
    }
    *steps_out = st;
    *mu_out = mu;
    return status;
}

// The implicit adjoint's solve H x = b (b: gpose for the poses, 0 for the landmarks) through the exact reduced system at
// the state in sh.Rwb / sh.pwb: x_p = S^-1 b_p, x_l = -Hll^-1 Hlp x_p, then at most two refinement steps on the residual
// b - H x (H x exactly, one dual pass).  -> false when S is not positive definite (then nothing is solved); else x in
// sh.dmp (poses) and NT_P (landmarks), *rel the final relative residual, *iters the refinement steps taken
__device__ bool nt_adjoint_direct(BaShared& sh, NtShared& nt, const XcbBaWindows& d, unsigned char* dsm, double* lsc,
                                  const double* b, double tol, double* rel, int* iters)
{
    const int n = sh.w.n, tid = threadIdx.x;
    double* S = (double*)dsm;
    SlotGeo<Dual>* Gd = (SlotGeo<Dual>*)(dsm + ba_off_x(n));
    SlotGeo<Dual>* G0 = (SlotGeo<Dual>*)(dsm + ba_off_x(n) + nt_x_bytes(n));
    nt_geo(sh, *G0);
    nt_xsystem(sh, nt, d, dsm, lsc, false);
    if (chol_factor(S, n)) return false;
    double b2 = 0.0;
    for (int q = tid; q < n; q += blockDim.x) {
        sh.rhs[q] = held(sh, q) ? 0.0 : b[q];
        sh.dmp[q] = sh.rhs[q];
        b2 += sh.rhs[q] * sh.rhs[q];
    }
    b2 = warp_sum(b2);
    __syncthreads();
    if ((tid & 31) == 0) sh.red[tid >> 5] = b2;
    const double bn = sqrt(block_sum_red(sh));
    chol_solve(S, n, sh.dmp);
    for (int q = tid; q < n; q += blockDim.x) sh.dx[q] = sh.dmp[q];
    __syncthreads();
    slot_geo_dual(sh, sh.dx, *Gd);
    pass_adj_l(sh, d, *Gd, lsc, true);
    __syncthreads();
    int it = 0;
    *rel = 0.0;
    while (bn > 0.0) {
        // r = b - H x: poses -> sh.g, landmarks -> NT_Z
        for (int q = tid; q < n; q += blockDim.x) { nt.gp[q] = 0.0; nt.hp[q] = 0.0; sh.dx[q] = sh.dmp[q]; }
        __syncthreads();
        slot_geo_dual(sh, sh.dx, *Gd);
        pass_dual(sh, nt, d, *Gd, NT_MODE_HV, lsc, nullptr, nullptr);
        __syncthreads();
        cl_sum_array(nt.hp, n);
        for (int q = tid; q < n; q += blockDim.x) sh.g[q] = held(sh, q) ? 0.0 : sh.rhs[q] - nt.hp[q];
        for (int l = sh.lb + tid; l < sh.le; l += blockDim.x) {
            double* sc = lsc + (size_t)(sh.w.lm0 + l) * NT_LM_STRIDE;
            for (int i = 0; i < 3; ++i) sc[NT_Z + i] = -sc[NT_HP + i];
        }
        __syncthreads();
        // the pose part counted by the cluster's rank 0, the landmark part by every CTA for its slice
        const bool r0 = cg::this_cluster().block_rank() == 0;
        *rel = sqrt(cl_reduce(nt, nt_dot(sh, nt, sh.g, sh.g, lsc, NT_Z, NT_Z, r0), false)) / bn;
        if (!(*rel > tol) || it >= 2) break;
        ++it;
        // dx_p = S^-1 (r_p - sum Hpl Hll^-1 r_l), dx_l = Hll^-1 (r_l - Hlp dx_p)
        for (int q = tid; q < n; q += blockDim.x) nt.gp[q] = 0.0;
        __syncthreads();
        pass_adj_y(sh, d, *G0, lsc, nt.gp);
        __syncthreads();
        cl_sum_array(nt.gp, n);
        for (int q = tid; q < n; q += blockDim.x) sh.y[q] = held(sh, q) ? 0.0 : sh.g[q] - nt.gp[q];
        __syncthreads();
        chol_solve(S, n, sh.y);
        for (int q = tid; q < n; q += blockDim.x) sh.dx[q] = sh.y[q];
        __syncthreads();
        slot_geo_dual(sh, sh.dx, *Gd);
        pass_adj_l(sh, d, *Gd, lsc, false);
        __syncthreads();
        for (int q = tid; q < n; q += blockDim.x) sh.dmp[q] += sh.y[q];
        __syncthreads();
    }
    *iters = it;
    return true;
}

__global__ void __launch_bounds__(BA_THREADS, 1) k_ba_newton(XcbBaWindows d, int mode, int steps, int maxit,
                                                             double tol, const double* gpose, double* gtheta,
                                                             double* gisig, double* gz, double* stats, double* lsc,
                                                             int* counter, size_t lsc_doubles, double* scopy)
{
    extern __shared__ __align__(16) unsigned char dsm[];
    __shared__ BaShared sh;
    __shared__ NtShared nt;
    __shared__ int s_short;
    const int tid = threadIdx.x;
    if (tid == 0) {
        long long Lt = 0;
        for (int w = 0; w < d.nw; ++w) Lt = max(Lt, (long long)d.lm_off[w] + d.L[w]);
        s_short = (size_t)BA_LSC_STRIDE * Lt > lsc_doubles;
    }
    __syncthreads();
    if (s_short) {
        // the per-landmark records do not fit the scratch: nothing is written but every window's status
        if (blockIdx.x == 0)
            for (int w = tid; w < d.nw; w += blockDim.x) stats[4 * w + 3] = XCB_BA_STATUS_SCRATCH;
        return;
    }
    // a window per thread-block cluster: its CTAs take slices of the window's landmarks and reduce their sums through
    // distributed shared memory (cl_reduce, cl_sum_array); poses, reduced systems and decisions are the same bits on
    // every CTA, so every CTA takes the same branches
    cg::cluster_group cl = cg::this_cluster();
    const int crank = (int)cl.block_rank(), csize = (int)cl.num_blocks();
    for (;;) {
        if (crank == 0 && tid == 0) sh.win = atomicAdd(counter, 1);
        if (csize > 1) {
            cl.sync();
            if (crank != 0 && tid == 0) sh.win = *cl.map_shared_rank(&sh.win, 0);
            cl.sync();
        }
        __syncthreads();
        const int wi = sh.win;
        if (wi >= d.nw) break;
        const int w = d.order ? d.order[wi] : wi;
        if (tid == 0) {
            BaWin& W = sh.w;
            W.P = d.P[w]; W.L = d.L[w]; W.n = 6 * W.P; W.hold = d.hold ? d.hold[w] : -1;
            sh.lb = (int)((long long)W.L * crank / csize);
            sh.le = (int)((long long)W.L * (crank + 1) / csize);
            W.lm0 = d.lm_off[w]; W.s0 = d.slot_off[w];
            W.fx = d.cam[6 * w]; W.fy = d.cam[6 * w + 1]; W.cx = d.cam[6 * w + 2]; W.cy = d.cam[6 * w + 3];
            W.B = d.cam[6 * w + 4]; W.hk = d.cam[6 * w + 5];
            for (int i = 0; i < 9; ++i) W.Rbc[i] = d.ext[12 * w + i];
            for (int i = 0; i < 3; ++i) W.pbc[i] = d.ext[12 * w + 9 + i];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) W.Rcb[i * 3 + j] = W.Rbc[j * 3 + i];
            double px[9] = {0.0, -W.pbc[2], W.pbc[1], W.pbc[2], 0.0, -W.pbc[0], -W.pbc[1], W.pbc[0], 0.0};
            for (int i = 0; i < 9; ++i) W.Px[i] = px[i];
            sh.lam = 0.0; sh.overflow = 0;
            for (int i = 0; i < NT_THETA; ++i) nt.th[i] = 0.0;
        }
        __syncthreads();
        const int P = sh.w.P, n = sh.w.n, s0 = sh.w.s0;
        if (P > BA_MAXP || P < 1 || has_prior(d, w)) {
            if (tid == 0 && crank == 0) stats[4 * w + 3] = has_prior(d, w) ? XCB_BA_STATUS_PRIOR : -1.0;
            __syncthreads();
            continue;
        }
        for (int q = tid; q < P * 9; q += blockDim.x) sh.Rwb[q] = d.Rwb[9 * s0 + q];
        for (int q = tid; q < P * 3; q += blockDim.x) sh.pwb[q] = d.pwb[3 * s0 + q];
        __syncthreads();
        double* S64 = (double*)dsm;
        WarpLm<double>* wl64 = (WarpLm<double>*)(dsm + ba_off_x(n));
        int iters = 0, status = 0, neg = 0;
        double rel = 0.0, gmax = 0.0;
        const bool upd = mode == XCB_BA_NEWTON_POLISH;      // may flag new constant landmarks
        if (mode != XCB_BA_NEWTON_ADJOINT) {
            // the landmark-eliminated Newton polish (nt_polish), then the gradient at the final state (flagging the
            // landmarks the LM cannot move when `upd`)
            int taken = 0;
            double mu = 0.0;
            if (steps > 0)
                status = nt_polish(sh, nt, d, dsm, lsc, scopy + ((size_t)w * NT_CL_MAX + crank) * NT_SC, steps, upd,
                                   &taken, &mu);
            iters = taken;
            rel = mu;
            slot_geo(sh, sh.Rwb, sh.pwb);
            nt_grad(sh, nt, d, dsm, lsc, upd, true);
            gmax = cl_reduce(nt, nt_gmax(sh, nt, lsc), true);
            if (crank == 0) {
                for (int q = tid; q < P * 9; q += blockDim.x) d.Rwb[9 * s0 + q] = sh.Rwb[q];
                for (int q = tid; q < P * 3; q += blockDim.x) d.pwb[3 * s0 + q] = sh.pwb[q];
            }
        } else if (nt_adjoint_direct(sh, nt, d, dsm, lsc, gpose + 6 * (size_t)s0, tol, &rel, &iters)) {
            // implicit adjoint: H x = dL/dx (poses from gpose, landmarks 0) solved through the exact reduced system,
            // then -(d2C / dtheta dx) x: the theta pass moves the state along x (poses sh.dmp, landmarks NT_P)
            for (int q = tid; q < n; q += blockDim.x) { sh.dx[q] = sh.dmp[q]; nt.gp[q] = 0.0; nt.hp[q] = 0.0; }
            if (tid < NT_THETA) nt.th[tid] = 0.0;
            __syncthreads();
            SlotGeo<Dual>* Gd = (SlotGeo<Dual>*)(dsm + ba_off_x(n));
            slot_geo(sh, sh.Rwb, sh.pwb);
            slot_geo_dual(sh, sh.dx, *Gd);
            pass_dual(sh, nt, d, *Gd, NT_MODE_THETA, lsc, gisig, gz);
            __syncthreads();
            cl_sum_array(nt.th, NT_THETA);
            if (tid < NT_THETA && crank == 0) gtheta[(size_t)w * NT_THETA + tid] = nt.th[tid];
        } else if (crank == 0) {
            // the exact reduced system is not positive definite: conjugate gradients preconditioned with the Gauss-
            // Newton system, by the cluster's rank 0 over every landmark (no cluster barrier on this path)
            if (tid == 0) { sh.lb = 0; sh.le = sh.w.L; }
            __syncthreads();
            slot_geo(sh, sh.Rwb, sh.pwb);
            if (nt_gn_factor(sh, d, S64, wl64, lsc)) status = 1;
            else {
                nt_grad(sh, nt, d, dsm, lsc, false);       // the gradient; constant landmarks as flagged
                for (int q = tid; q < n; q += blockDim.x)
                    sh.rhs[q] = held(sh, q) ? 0.0 : gpose[6 * (size_t)s0 + q];
                for (int l = tid; l < sh.w.L; l += blockDim.x)
                    for (int i = 0; i < NT_FROZEN; ++i) lsc[(size_t)(sh.w.lm0 + l) * NT_LM_STRIDE + i] = 0.0;
                __syncthreads();
                rel = nt_solve_exact(sh, nt, d, S64, dsm, lsc, maxit, tol, &iters, &neg);
                if (neg) status = 2;
                for (int l = tid; l < sh.w.L; l += blockDim.x) {
                    double* sc = lsc + (size_t)(sh.w.lm0 + l) * NT_LM_STRIDE;
                    for (int i = 0; i < 3; ++i) sc[NT_P + i] = sc[NT_X + i];
                }
                for (int q = tid; q < n; q += blockDim.x) { sh.dx[q] = sh.dmp[q]; nt.gp[q] = 0.0; nt.hp[q] = 0.0; }
                if (tid < NT_THETA) nt.th[tid] = 0.0;
                __syncthreads();
                SlotGeo<Dual>* Gd = (SlotGeo<Dual>*)(dsm + ba_off_x(n));
                slot_geo(sh, sh.Rwb, sh.pwb);
                slot_geo_dual(sh, sh.dx, *Gd);
                pass_dual(sh, nt, d, *Gd, NT_MODE_THETA, lsc, gisig, gz);
                __syncthreads();
                if (tid < NT_THETA) gtheta[(size_t)w * NT_THETA + tid] = nt.th[tid];
            }
        }
        const double ovf = cl_reduce(nt, sh.overflow ? 1.0 : 0.0, true);
        if (tid == 0 && crank == 0) {
            stats[4 * w + 0] = iters;
            stats[4 * w + 1] = rel;
            stats[4 * w + 2] = gmax;
            stats[4 * w + 3] = status ? (double)status : (ovf != 0.0 ? -2.0 : 0.0);
        }
        __syncthreads();
    }
}

size_t xcb_ba_newton_smem_bytes(int maxP)
{
    const int n = 6 * maxP;
    return ba_off_x(n) + nt_x_bytes(n) + sizeof(SlotGeo<Dual>);
}

size_t xcb_ba_newton_copy_doubles(int nw) { return (size_t)(nw > 0 ? nw : 1) * NT_CL_MAX * NT_SC; }

cudaError_t xcb_launch_ba_newton(const XcbBaWindows& d, int max_slots, int mode, int steps, int maxit, double tol,
                                 const double* gpose, double* gtheta, double* gisig, double* gz, double* stats,
                                 double* lsc, int* counter, int grid, cudaStream_t st, size_t lsc_doubles,
                                 double* scopy)
{
    static XcbAttrOnce attr;
    cudaError_t e = xcb_smem_attr_once(attr, (const void*)k_ba_newton, (int)xcb_ba_newton_smem_bytes(BA_MAXP));
    if (e != cudaSuccess) return e;
    // CTAs per window: the SMs that one CTA per window would leave idle, at most NT_CL_MAX (grid: the SM count)
    int C = d.nw > 0 ? grid / d.nw : 1;
    C = C < 1 ? 1 : (C > NT_CL_MAX ? NT_CL_MAX : C);
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    cfg.blockDim = dim3(BA_THREADS);
    cfg.dynamicSmemBytes = xcb_ba_newton_smem_bytes(max_slots);
    cfg.stream = st;
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    for (; C >= 1; --C) {
        // as many clusters as the GPU holds at once (persistent: windows from the work counter), at most one per window
        at[0].val.clusterDim.x = C;
        cfg.gridDim = dim3(C);
        int ncl = 0;
        if (cudaOccupancyMaxActiveClusters(&ncl, (const void*)k_ba_newton, &cfg) != cudaSuccess || ncl < 1) {
            cudaGetLastError();
            continue;
        }
        int nc = ncl < d.nw ? ncl : d.nw;
        if (grid / C < nc) nc = grid / C > 1 ? grid / C : 1;
        cfg.gridDim = dim3(nc * C);
        e = cudaLaunchKernelEx(&cfg, k_ba_newton, d, mode, steps, maxit, tol, gpose, gtheta, gisig, gz, stats, lsc,
                               counter, lsc_doubles, scopy);
        return e != cudaSuccess ? e : cudaGetLastError();
    }
    return cudaErrorInvalidConfiguration;
}

cudaError_t xcb_launch_ba_windows(const XcbBaWindows& d, int max_slots, int iters, double lam0, int mode,
                                  double* stats, double* dx0, int dx0_stride, double* lmp_trial, int* counter,
                                  int grid, cudaStream_t st, const double* frz, size_t trial_doubles)
{
    size_t sm = xcb_ba_smem_bytes(max_slots);
    static XcbAttrOnce attr;
    cudaError_t e = xcb_smem_attr_once(attr, (const void*)k_ba_windows, (int)xcb_ba_smem_bytes(BA_MAXP));
    if (e != cudaSuccess) return e;
    k_ba_windows<<<grid, BA_THREADS, sm, st>>>(d, iters, lam0, mode, stats, dx0, dx0_stride, lmp_trial, counter,
                                               frz, trial_doubles);
    return cudaGetLastError();
}

// =====================================================================================================================
// Large windows on every SM.  The persistent kernel above gives each window one CTA, which leaves most of the GPU idle
// when a batch holds fewer windows than SMs (32 windows of 20 keyframes and 6,000 landmarks use 32 of 148 SMs).  This
// path runs the same LM iteration (the same landmark passes, the same reduced system, Cholesky, refinement, back-
// substitution and accept / reject) as a sequence of launches: the landmark passes over chunks of LW_CHUNK landmarks
// of every window at once (each CTA sums its chunk's share of the reduced system, the gradient and the cost in shared
// memory, then adds it to the window's accumulators in global memory), and the per-window steps (Cholesky, solves,
// LM control) one CTA per window.  The LM state lives in global memory (LwState) between the launches.
// =====================================================================================================================
#define LW_CHUNK 256
#define LW_NT (BA_MAXN * (BA_MAXN + 1) / 2)

struct LwState {
    double lam, cost0, cur, ctot;
    int accepted, status, bad, acc, conv, pad;
};

struct LwWork {
    LwState* st;            // [nw]
    double* S;              // [nw][LW_NT] reduced system (float in the mixed build: the first LW_NT floats)
    double* g;              // [nw][BA_MAXN] build gradient (float in the mixed build)
    double* cost;           // [nw] build cost (float64)
    double* Lf;             // [nw][LW_NT] Cholesky factor
    double* dx;             // [nw][BA_MAXN]
    double* dmp;            // [nw][BA_MAXN]
    double* g64;            // [nw][BA_MAXN] refinement: float64 gradient
    double* y64;            // [nw][BA_MAXN] refinement: S_true dx
    double* cost64;         // [nw] refinement: float64 cost
    double* ctrial;         // [nw] trial cost
    double* R2;             // [S][9] trial poses
    double* p2;             // [S][3]
    double* lmp_trial;      // [Lt][3]
    const double* frz;      // the Newton scratch's constant-landmark flags (19 doubles per landmark), or null
};

// one chunk: landmarks [l0, l1) (window-local) of window w
struct LwChunk {
    int w, l0, l1;
};

__device__ void lw_load_window(BaShared& sh, const XcbBaWindows& d, int w)
{
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
    sh.overflow = 0;
}

// CTA set-up of a chunk kernel: the window's parameters, its current poses (or R / p when given) and their geometry.
// -> false when the window is done (failed status)
__device__ bool lw_setup(BaShared& sh, const XcbBaWindows& d, const LwWork& lw, const LwChunk& c, const double* R,
                         const double* p)
{
    if (c.w < 0 || c.w >= d.nw) return false;
    if (threadIdx.x == 0) {
        lw_load_window(sh, d, c.w);
        sh.lam = lw.st[c.w].lam;
        sh.lb = max(c.l0, 0);
        sh.le = min(c.l1, sh.w.L);          // a chunk never reaches past its window's landmarks
        sh.win = lw.st[c.w].status;
    }
    __syncthreads();
    if (sh.win != 0) return false;
    const int P = sh.w.P, s0 = sh.w.s0;
    for (int q = threadIdx.x; q < P * 9; q += blockDim.x) sh.Rwb[q] = (R ? R : d.Rwb)[9 * s0 + q];
    for (int q = threadIdx.x; q < P * 3; q += blockDim.x) sh.pwb[q] = (p ? p : d.pwb)[3 * s0 + q];
    __syncthreads();
    slot_geo(sh, sh.Rwb, sh.pwb);
    return true;
}

// the chunk's share of the reduced system (packed lower), gradient and cost, added to the window's accumulators
template <typename T>
__global__ void __launch_bounds__(BA_THREADS, 1) k_lw_build(XcbBaWindows d, LwWork lw, const LwChunk* chunks)
{
    extern __shared__ __align__(16) unsigned char dsm[];
    __shared__ BaShared sh;
    const LwChunk c = chunks[blockIdx.x];
    if (!lw_setup(sh, d, lw, c, nullptr, nullptr)) return;
    const int n = sh.w.n, nt = n * (n + 1) / 2;
    T* S = (T*)dsm;
    WarpLm<T>* wl = (WarpLm<T>*)(dsm + ((sizeof(T) * (size_t)nt + 15) & ~(size_t)15));
    T* gb;
    if constexpr (sizeof(T) == 4) gb = sh.bf;
    else gb = sh.g;
    for (int q = threadIdx.x; q < nt; q += blockDim.x) S[q] = (T)0;
    for (int q = threadIdx.x; q < n; q += blockDim.x) gb[q] = (T)0;
    __syncthreads();
    double cst = 0.0;
    if constexpr (sizeof(T) == 4)
        pass_build<T, true>(sh, d, sh.g32, S, gb, wl, &cst, lw.frz);
    else
        pass_build<T, true>(sh, d, sh.g64, S, gb, wl, &cst, lw.frz);
    const double ctot = block_sum_red(sh);
    T* Sg = (T*)(lw.S + (size_t)c.w * LW_NT);
    T* gg = (T*)(lw.g + (size_t)c.w * BA_MAXN);
    for (int q = threadIdx.x; q < nt; q += blockDim.x)
        if (S[q] != (T)0) atomicAdd(&Sg[q], S[q]);
    for (int q = threadIdx.x; q < n; q += blockDim.x) atomicAdd(&gg[q], gb[q]);
    if (threadIdx.x == 0) {
        atomicAdd(&lw.cost[c.w], ctot);
        if (sh.overflow) atomicExch(&lw.st[c.w].status, -2);
    }
}

// The mixed build of a chunk with the Schur term on the tensor cores.  The landmarks go through in rounds of TC_LMS
// (the tile's TC_KT columns hold three per landmark), one per warp, the CTA's other warps idle: each warp adds its landmark's pose-pose blocks (the same slot, or a target with the host) and gradient
// to the CTA's packed system with shared-memory atomics, as pass_build does, and writes the landmark's three Schur
// columns U = Hlp^T C (Hll^-1 = C C^T; rows 6 s .. 6 s + 5 of its touched slots s, zero elsewhere) into the round's
// TF32 hi / lo tile; one thread then adds U U^T of the tile to the tensor-memory accumulator (tc_issue), which runs
// while the next round is linearised.  At the end the accumulator is subtracted from the packed system:
// S = sum of pose-pose blocks - sum_l Hlp_l^T Hll_l^-1 Hlp_l.  A landmark whose Hll^-1 is not numerically positive
// definite in float64 keeps the scatter of its Schur blocks.  -> false when a tensor-core wait ran out.
#define TC_LMS (TC_KT / 3)                      // landmarks per tensor-core round: three tile columns each
static_assert(TC_LMS <= BA_WARPS, "a tensor-core round takes one landmark per warp");
__device__ bool pass_build_tc(BaShared& sh, const XcbBaWindows& d, float* S, float* gb, WarpLm<float>* wls,
                              float* tiles, uint64_t* bar, uint32_t tmem, int* fail, const double* frz)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, tid = threadIdx.x;
    WarpLm<float>& wl = wls[wid];
    const SlotGeo<float>& G = sh.g32;
    double c_local = 0.0;
    int rounds = 0;
    for (int base = sh.lb; base < sh.le; base += TC_LMS, ++rounds) {
        const int stg = rounds & 1;
        float* hi = tiles + stg * 2 * TC_TILE_FLOATS;
        float* lo = hi + TC_TILE_FLOATS;
        if (rounds >= 2 && tid == 0 && !*fail && !tc_mbar_wait(&bar[stg], (uint32_t)(((rounds >> 1) - 1) & 1)))
            *fail = 1;
        __syncthreads();
        if (*fail) break;
        for (int q = tid; q < 2 * TC_TILE_FLOATS; q += blockDim.x) hi[q] = 0.0f;     // hi and lo are adjacent
        __syncthreads();
        const int l = base + wid;
        const int gl = sh.w.lm0 + l;
        if (wid < TC_LMS && l < sh.le && d.lm_mask[gl]) {
            const int h = d.lm_host[gl];
            float Hll[9], bl[3];
            int nt;
            const bool ok = lin_landmark<float>(sh, d, G, l, sh.lam, d.lmp, wl, Hll, bl, &nt, &c_local) &&
                            !lm_const(frz, gl);
            float Hi[9], HiB[3] = {0.0f, 0.0f, 0.0f};
            double C[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            bool tcl = false;
            if (ok) {
                inv3<float>(Hll, Hi);
#pragma unroll
                for (int i = 0; i < 3; ++i) HiB[i] = Hi[i * 3] * bl[0] + Hi[i * 3 + 1] * bl[1] + Hi[i * 3 + 2] * bl[2];
                // C: the lower Cholesky factor of Hll^-1 in float64
                double H64[9], I64[9];
#pragma unroll
                for (int i = 0; i < 9; ++i) H64[i] = (double)Hll[i];
                inv3<double>(H64, I64);
                const double a00 = I64[0];
                if (a00 > 0.0) {
                    C[0] = sqrt(a00);
                    C[3] = I64[3] / C[0];
                    C[6] = I64[6] / C[0];
                    const double a11 = I64[4] - C[3] * C[3];
                    if (a11 > 0.0) {
                        C[4] = sqrt(a11);
                        C[7] = (I64[7] - C[6] * C[3]) / C[4];
                        const double a22 = I64[8] - C[6] * C[6] - C[7] * C[7];
                        if (a22 > 0.0) { C[8] = sqrt(a22); tcl = true; }
                    }
                }
                if (!tcl)
                    for (int q = lane; q < nt * 18; q += 32) {
                        const int a = q / 18, e = q % 18, i = e / 6, j = e % 6;
                        wl.Tb[a][e] = Hi[i * 3] * wl.Hlp[a][j] + Hi[i * 3 + 1] * wl.Hlp[a][6 + j] +
                                      Hi[i * 3 + 2] * wl.Hlp[a][12 + j];
                    }
                __syncwarp();
            }
            // gradient: sum_obs w Jx^T e - Hlp^T Hll^-1 bl
            for (int q = lane; q < nt * 6; q += 32) {
                const int a = q / 6, i = q % 6, s = wl.ts[a];
                const int off = s == h ? OB_JH : OB_JT;
                float acc = 0.0f;
                for (unsigned m = wl.om[a]; m; m &= m - 1) {
                    const float* ob = wl.ob[__ffs(m) - 1];
                    acc += ob[OB_W] * (obj(ob, off, 0, i) * ob[OB_E] + obj(ob, off, 1, i) * ob[OB_E + 1]);
                }
                if (ok) acc -= wl.Hlp[a][i] * HiB[0] + wl.Hlp[a][6 + i] * HiB[1] + wl.Hlp[a][12 + i] * HiB[2];
                atomicAdd(&gb[6 * s + i], acc);
            }
            if (ok && tcl) {
                // the landmark's Schur columns 3 wid .. 3 wid + 2 of the round's tile
                for (int q = lane; q < nt * 18; q += 32) {
                    const int a = q / 18, e = q % 18, j = e / 3, c = e % 3;
                    const float u = (float)(wl.Hlp[a][j] * C[c] + wl.Hlp[a][6 + j] * C[3 + c] +
                                            wl.Hlp[a][12 + j] * C[6 + c]);
                    float uh, ul;
                    tc_split(u, uh, ul);
                    const int o = tc_off(6 * wl.ts[a] + j, 3 * wid + c);
                    hi[o] = uh;
                    lo[o] = ul;
                }
            }
            // the pose-pose blocks: (a, a) for every touched slot, (a, host) for the others; with the Schur blocks of
            // a landmark that did not take the tensor-core path
            int hx = 0;
            for (int a = 0; a < nt; ++a)
                if (wl.ts[a] == h) hx = a;
            const bool full = ok && !tcl;
            const int npair = full ? nt * (nt + 1) / 2 : (nt > 0 ? 2 * nt - 1 : 0);
            for (int q = lane; q < npair * 36; q += 32) {
                const int pr = q / 36, e = q % 36, i = e / 6, j = e % 6;
                int a, b;
                if (full) {
                    a = (int)((sqrtf(8.0f * pr + 1.0f) - 1.0f) * 0.5f);
                    while (a * (a + 1) / 2 > pr) --a;
                    while ((a + 1) * (a + 2) / 2 <= pr) ++a;
                    b = pr - a * (a + 1) / 2;
                } else if (pr < nt) {
                    a = b = pr;
                } else {
                    const int t = pr - nt < hx ? pr - nt : pr - nt + 1;
                    a = t > hx ? t : hx;
                    b = t > hx ? hx : t;
                }
                if (a == b && j > i) continue;
                const int sa = wl.ts[a], sb = wl.ts[b];
                float acc = 0.0f;
                if (a == b) {
                    const int off = sa == h ? OB_JH : OB_JT;
                    for (unsigned m = wl.om[a]; m; m &= m - 1) {
                        const float* ob = wl.ob[__ffs(m) - 1];
                        acc += ob[OB_W] * (obj(ob, off, 0, i) * obj(ob, off, 0, j) + obj(ob, off, 1, i) * obj(ob, off, 1, j));
                    }
                } else if (sa == h || sb == h) {
                    const int at = sa == h ? b : a;
                    const int offa = sa == h ? OB_JH : OB_JT, offb = sb == h ? OB_JH : OB_JT;
                    for (unsigned m = wl.om[at]; m; m &= m - 1) {
                        const float* ob = wl.ob[__ffs(m) - 1];
                        acc += ob[OB_W] * (obj(ob, offa, 0, i) * obj(ob, offb, 0, j) + obj(ob, offa, 1, i) * obj(ob, offb, 1, j));
                    }
                }
                if (full)
                    acc -= wl.Hlp[a][i] * wl.Tb[b][j] + wl.Hlp[a][6 + i] * wl.Tb[b][6 + j] + wl.Hlp[a][12 + i] * wl.Tb[b][12 + j];
                atomicAdd(&S[tri(6 * sa + i, 6 * sb + j)], acc);
            }
            __syncwarp();
        }
        tc_fence_proxy();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            tc_issue(tmem, hi, lo, rounds > 0, &bar[stg]);
        }
    }
    if (tid == 0 && !*fail && rounds >= 1) {
        if (!tc_mbar_wait(&bar[(rounds - 1) & 1], (uint32_t)(((rounds - 1) >> 1) & 1))) *fail = 1;
        if (rounds >= 2 && !tc_mbar_wait(&bar[(rounds - 2) & 1], (uint32_t)(((rounds - 2) >> 1) & 1))) *fail = 1;
    }
    if (tid == 0 && rounds >= 1 && !tc_drain(&bar[2])) *fail = 1;
    __syncthreads();
    tc_fence_after();
    const int n = sh.w.n;
    if (!*fail && rounds > 0 && wid < 4) {
        const int r = 32 * wid + lane;
        for (int c0 = 0; c0 < TC_M; c0 += 16) {
            float v[16];
            tc_ld16(tmem, wid, c0, v);
            if (r < n)
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    if (c0 + i <= r) S[tri(r, c0 + i)] -= v[i];
        }
    }
    __syncthreads();
    c_local = warp_sum(c_local);
    if (lane == 0) sh.red[wid] = c_local;
    return !*fail;
}

// dynamic shared memory of k_lw_build_tc: [tiles: 2 stages x (hi, lo)][S packed float][WarpLm<float> per warp]
static __host__ __device__ __forceinline__ size_t lw_tc_s_off() { return 4 * (size_t)TC_TILE_FLOATS * sizeof(float); }
static size_t lw_build_tc_smem(int maxP)
{
    const int n = 6 * maxP, nt = n * (n + 1) / 2;
    return lw_tc_s_off() + ((4 * (size_t)nt + 15) & ~(size_t)15) + sizeof(WarpLm<float>) * BA_WARPS;
}

__global__ void __launch_bounds__(BA_THREADS, 1) k_lw_build_tc(XcbBaWindows d, LwWork lw, const LwChunk* chunks)
{
    extern __shared__ __align__(1024) unsigned char dsm[];
    __shared__ BaShared sh;
    __shared__ __align__(8) uint64_t bar[3];          // two tile stages, the final drain
    __shared__ uint32_t tmem_base;
    __shared__ int fail;
    const LwChunk c = chunks[blockIdx.x];
    if (!lw_setup(sh, d, lw, c, nullptr, nullptr)) return;
    const int tid = threadIdx.x, wid = tid >> 5;
    if (wid == 0) tc_alloc(&tmem_base, 128);
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
    const int n = sh.w.n, nt = n * (n + 1) / 2;
    float* tiles = (float*)dsm;
    float* S = (float*)(dsm + lw_tc_s_off());
    WarpLm<float>* wl = (WarpLm<float>*)(dsm + lw_tc_s_off() + ((4 * (size_t)nt + 15) & ~(size_t)15));
    for (int q = tid; q < nt; q += blockDim.x) S[q] = 0.0f;
    for (int q = tid; q < n; q += blockDim.x) sh.bf[q] = 0.0f;
    __syncthreads();
    const bool good = pass_build_tc(sh, d, S, sh.bf, wl, tiles, bar, tmem, &fail, lw.frz);
    const double ctot = block_sum_red(sh);
    float* Sg = (float*)(lw.S + (size_t)c.w * LW_NT);
    float* gg = (float*)(lw.g + (size_t)c.w * BA_MAXN);
    if (good) {
        for (int q = tid; q < nt; q += blockDim.x)
            if (S[q] != 0.0f) atomicAdd(&Sg[q], S[q]);
        for (int q = tid; q < n; q += blockDim.x) atomicAdd(&gg[q], sh.bf[q]);
    }
    if (tid == 0) {
        atomicAdd(&lw.cost[c.w], ctot);
        if (sh.overflow) atomicExch(&lw.st[c.w].status, -2);
        if (!good) atomicExch(&lw.st[c.w].status, XCB_BA_STATUS_TC);
    }
    tc_fence_before();
    __syncthreads();
    if (wid == 0) tc_dealloc(tmem, 128);
}

// per window: hold, damping, Cholesky, the first solve (the build's float32 right-hand side in the mixed mode)
template <typename T>
__global__ void __launch_bounds__(BA_THREADS, 1) k_lw_solve(XcbBaWindows d, LwWork lw, int mode, int it)
{
    extern __shared__ __align__(16) unsigned char dsm[];
    __shared__ BaShared sh;
    const int w = blockIdx.x, tid = threadIdx.x;
    LwState& st = lw.st[w];
    if (tid == 0) { lw_load_window(sh, d, w); sh.lam = st.lam; sh.win = st.status; }
    __syncthreads();
    if (sh.win != 0) return;
    const int n = sh.w.n, nt = n * (n + 1) / 2;
    double* S64 = (double*)dsm;
    const T* Sg = (const T*)(lw.S + (size_t)w * LW_NT);
    const T* gg = (const T*)(lw.g + (size_t)w * BA_MAXN);
    for (int q = tid; q < nt; q += blockDim.x) S64[q] = (double)Sg[q];
    for (int q = tid; q < n; q += blockDim.x) sh.rhs[q] = (double)gg[q];
    __syncthreads();
    const int hs = sh.w.hold, P = sh.w.P;
    if (hs >= 0 && hs < P) {
        for (int q = tid; q < 6 * n; q += blockDim.x) {
            const int i = 6 * hs + q / n, j = q % n;
            S64[i >= j ? tri(i, j) : tri(j, i)] = 0.0;
        }
        __syncthreads();
        for (int q = tid; q < 6; q += blockDim.x) { S64[tri(6 * hs + q, 6 * hs + q)] = 1.0; sh.rhs[6 * hs + q] = 0.0; }
        __syncthreads();
    }
    double* dmp = lw.dmp + (size_t)w * BA_MAXN;
    for (int q = tid; q < n; q += blockDim.x) {
        const double dg = S64[tri(q, q)];
        sh.dmp[q] = sh.lam * dg + 1e-9;
        S64[tri(q, q)] = dg + sh.dmp[q];
        sh.dx[q] = -sh.rhs[q];
        dmp[q] = sh.dmp[q];
    }
    __syncthreads();
    const int bad = chol_factor(S64, n);
    if (!bad) chol_solve(S64, n, sh.dx);
    double* dx = lw.dx + (size_t)w * BA_MAXN;
    double* Lf = lw.Lf + (size_t)w * LW_NT;
    for (int q = tid; q < n; q += blockDim.x) dx[q] = bad ? 0.0 : sh.dx[q];
    if (!bad)
        for (int q = tid; q < nt; q += blockDim.x) Lf[q] = S64[q];
    for (int q = tid; q < n; q += blockDim.x) { lw.g64[(size_t)w * BA_MAXN + q] = 0.0; lw.y64[(size_t)w * BA_MAXN + q] = 0.0; }
    if (tid == 0) {
        st.bad = bad ? 1 : 0;
        st.conv = 0;
        lw.cost64[w] = 0.0;
        lw.ctrial[w] = 0.0;
        if (mode != XCB_BA_MIXED) st.ctot = lw.cost[w];      // the float64 build's cost
    }
}

// the float64 refinement pass over a chunk: its share of the gradient (first pass), of S_true dx and of the cost
__global__ void __launch_bounds__(BA_THREADS, 1) k_lw_refine(XcbBaWindows d, LwWork lw, const LwChunk* chunks, int rf)
{
    extern __shared__ __align__(16) unsigned char dsm[];
    __shared__ BaShared sh;
    const LwChunk c = chunks[blockIdx.x];
    if (c.w < 0 || c.w >= d.nw) return;
    const LwState& st = lw.st[c.w];
    if (rf > 0 && (st.bad || st.conv)) return;
    if (!lw_setup(sh, d, lw, c, nullptr, nullptr)) return;
    const int n = sh.w.n;
    for (int q = threadIdx.x; q < n; q += blockDim.x) sh.dx[q] = lw.dx[(size_t)c.w * BA_MAXN + q];
    __syncthreads();
    WarpLm<double>* wl = (WarpLm<double>*)dsm;
    pass_refine(sh, d, wl, rf == 0, lw.frz);
    const double ctot = block_sum_red(sh);
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        if (rf == 0) atomicAdd(&lw.g64[(size_t)c.w * BA_MAXN + q], sh.g[q]);
        atomicAdd(&lw.y64[(size_t)c.w * BA_MAXN + q], sh.y[q]);
    }
    if (rf == 0 && threadIdx.x == 0) atomicAdd(&lw.cost64[c.w], ctot);
}

// per window: the refinement's correction (residual of the float64 normal equations, solved with the factor)
__global__ void __launch_bounds__(BA_THREADS, 1) k_lw_refine_solve(XcbBaWindows d, LwWork lw, int rf)
{
    extern __shared__ __align__(16) unsigned char dsm[];
    __shared__ BaShared sh;
    __shared__ double nrm[2];
    const int w = blockIdx.x, tid = threadIdx.x;
    LwState& st = lw.st[w];
    if (st.status != 0) return;
    if (tid == 0 && rf == 0) st.ctot = lw.cost64[w];
    if (st.bad || st.conv) return;
    const int n = 6 * d.P[w], nt = n * (n + 1) / 2, hs = d.hold ? d.hold[w] : -1;
    double* L = (double*)dsm;
    const double* Lf = lw.Lf + (size_t)w * LW_NT;
    for (int q = tid; q < nt; q += blockDim.x) L[q] = Lf[q];
    double* dx = lw.dx + (size_t)w * BA_MAXN;
    double* y = lw.y64 + (size_t)w * BA_MAXN;
    for (int q = tid; q < n; q += blockDim.x) {
        double r = -lw.g64[(size_t)w * BA_MAXN + q] - y[q] - lw.dmp[(size_t)w * BA_MAXN + q] * dx[q];
        if (hs >= 0 && q / 6 == hs) r = 0.0;
        sh.rhs[q] = r;
    }
    __syncthreads();
    chol_solve(L, n, sh.rhs);
    if (tid == 0) {
        double a = 0.0, b = 0.0;
        for (int q = 0; q < n; ++q) { a += sh.rhs[q] * sh.rhs[q]; b += dx[q] * dx[q]; }
        nrm[0] = a; nrm[1] = b;
    }
    __syncthreads();
    for (int q = tid; q < n; q += blockDim.x) { dx[q] += sh.rhs[q]; y[q] = 0.0; }
    if (tid == 0 && !(nrm[0] > 1e-18 * nrm[1])) st.conv = 1;
}

// per window: the trial poses (R Exp(dphi), p + dp) and the first iteration's step
__global__ void k_lw_trial(XcbBaWindows d, LwWork lw, int it, double* dx0, int dx0_stride)
{
    const int w = blockIdx.x;
    const LwState& st = lw.st[w];
    if (st.status != 0 || st.bad) return;
    const int P = d.P[w], s0 = d.slot_off[w];
    const double* dx = lw.dx + (size_t)w * BA_MAXN;
    if (it == 0 && dx0)
        for (int q = threadIdx.x; q < 6 * P; q += blockDim.x) dx0[(size_t)w * dx0_stride + q] = dx[q];
    for (int s = threadIdx.x; s < P; s += blockDim.x) {
        double Re[9];
        so3_exp(dx + 6 * s, Re);
        const double* R = d.Rwb + 9 * (s0 + s);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                lw.R2[9 * (s0 + s) + 3 * i + j] = R[3 * i] * Re[j] + R[3 * i + 1] * Re[3 + j] + R[3 * i + 2] * Re[6 + j];
        for (int i = 0; i < 3; ++i) lw.p2[3 * (s0 + s) + i] = d.pwb[3 * (s0 + s) + i] + dx[6 * s + 3 + i];
    }
}

// the chunk's back-substitution (trial landmark states) and its share of the trial cost
__global__ void __launch_bounds__(BA_THREADS, 1) k_lw_backsub(XcbBaWindows d, LwWork lw, const LwChunk* chunks)
{
    extern __shared__ __align__(16) unsigned char dsm[];
    __shared__ BaShared sh;
    const LwChunk c = chunks[blockIdx.x];
    if (c.w < 0 || c.w >= d.nw || lw.st[c.w].bad) return;
    if (!lw_setup(sh, d, lw, c, nullptr, nullptr)) return;
    const int n = sh.w.n;
    for (int q = threadIdx.x; q < n; q += blockDim.x) sh.dx[q] = lw.dx[(size_t)c.w * BA_MAXN + q];
    __syncthreads();
    WarpLm<double>* wl = (WarpLm<double>*)dsm;
    pass_backsub(sh, d, wl, lw.lmp_trial, lw.frz);
    __syncthreads();
    const int P = sh.w.P, s0 = sh.w.s0;
    for (int q = threadIdx.x; q < P * 9; q += blockDim.x) sh.R2[q] = lw.R2[9 * s0 + q];
    for (int q = threadIdx.x; q < P * 3; q += blockDim.x) sh.p2[q] = lw.p2[3 * s0 + q];
    __syncthreads();
    slot_geo(sh, sh.R2, sh.p2);
    pass_cost(sh, d, sh.g64, lw.lmp_trial);
    const double ct = block_sum_red(sh);
    if (threadIdx.x == 0) atomicAdd(&lw.ctrial[c.w], ct);
}

// per window: accept / reject (window.solve's rule), the poses committed, the next iteration's accumulators cleared
__global__ void k_lw_accept(XcbBaWindows d, LwWork lw, int it)
{
    const int w = blockIdx.x;
    LwState& st = lw.st[w];
    __shared__ int acc;
    if (threadIdx.x == 0) {
        acc = 0;
        if (st.status == 0) {
            const double ct = st.ctot;
            if (it == 0) st.cost0 = ct;
            if (st.bad) {
                st.cur = ct;
                st.lam *= 10.0;
            } else {
                const double cn = lw.ctrial[w];
                acc = cn < ct;
                st.cur = acc ? cn : ct;
                if (acc) { st.lam = fmax(st.lam / 10.0, 1e-12); st.accepted += 1; }
                else st.lam *= 10.0;
            }
        }
        st.acc = acc;
        lw.cost[w] = 0.0;
    }
    __syncthreads();
    const int P = d.P[w], s0 = d.slot_off[w];
    if (acc) {
        for (int q = threadIdx.x; q < P * 9; q += blockDim.x) d.Rwb[9 * s0 + q] = lw.R2[9 * s0 + q];
        for (int q = threadIdx.x; q < P * 3; q += blockDim.x) d.pwb[3 * s0 + q] = lw.p2[3 * s0 + q];
    }
    for (int q = threadIdx.x; q < LW_NT; q += blockDim.x) lw.S[(size_t)w * LW_NT + q] = 0.0;
    for (int q = threadIdx.x; q < BA_MAXN; q += blockDim.x) lw.g[(size_t)w * BA_MAXN + q] = 0.0;
}

// the accepted windows' landmarks take their trial states
__global__ void k_lw_commit(XcbBaWindows d, LwWork lw, const LwChunk* chunks)
{
    const LwChunk c = chunks[blockIdx.x];
    if (c.w < 0 || c.w >= d.nw || !lw.st[c.w].acc) return;
    const int lm0 = d.lm_off[c.w], l0 = max(c.l0, 0), l1 = min(c.l1, d.L[c.w]);
    for (int q = 3 * l0 + threadIdx.x; q < 3 * l1; q += blockDim.x)
        d.lmp[3 * lm0 + q] = lw.lmp_trial[3 * lm0 + q];
}

__global__ void k_lw_init(XcbBaWindows d, LwWork lw, double lam0)
{
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= d.nw) return;
    LwState& st = lw.st[w];
    st.lam = lam0; st.cost0 = 0.0; st.cur = 0.0; st.ctot = 0.0;
    st.accepted = 0; st.bad = 0; st.acc = 0; st.conv = 0;
    st.status = (d.P[w] > BA_MAXP || d.P[w] < 1) ? -1 : 0;
    lw.cost[w] = 0.0;
}

__global__ void k_lw_final(XcbBaWindows d, LwWork lw, double* stats, int iters)
{
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= d.nw) return;
    const LwState& st = lw.st[w];
    stats[8 * w + 0] = st.cost0;
    stats[8 * w + 1] = st.cur;
    stats[8 * w + 2] = st.accepted;
    stats[8 * w + 3] = st.lam;
    stats[8 * w + 4] = st.status;
    stats[8 * w + 5] = iters;
}

size_t xcb_ba_large_scratch_bytes_impl(int nw, int S, int Lt)
{
    const size_t W = (size_t)(nw > 0 ? nw : 1);
    size_t b = 0;
    b += W * sizeof(LwState);
    b += W * LW_NT * 8 * 2;                     // S, Lf
    b += W * BA_MAXN * 8 * 5;                   // g, dx, dmp, g64, y64
    b += W * 8 * 3;                             // cost, cost64, ctrial
    b += (size_t)(S > 0 ? S : 1) * 12 * 8;      // R2, p2
    b += (size_t)(Lt > 0 ? Lt : 1) * 3 * 8;     // lmp_trial
    return b + 16 * 256;
}

static size_t lw_build_smem(int maxP, bool mixed)
{
    const int n = 6 * maxP, nt = n * (n + 1) / 2;
    return mixed ? ((4 * (size_t)nt + 15) & ~(size_t)15) + sizeof(WarpLm<float>) * BA_WARPS
                 : ((8 * (size_t)nt + 15) & ~(size_t)15) + sizeof(WarpLm<double>) * BA_WARPS;
}

cudaError_t xcb_launch_ba_large(const XcbBaWindows& d, int slots, int Lt, const int* chunks, int nchunks,
                                int max_slots, int iters, double lam0, int mode, double* stats, double* dx0,
                                int dx0_stride, void* scratch, size_t scratch_bytes, cudaStream_t st, const double* frz)
{
    if (scratch_bytes < xcb_ba_large_scratch_bytes_impl(d.nw, slots, Lt)) return cudaErrorInvalidValue;
    char* p = (char*)scratch;
    auto take = [&](size_t bytes) {
        char* r = p;
        p += (bytes + 255) & ~(size_t)255;
        return r;
    };
    const size_t W = (size_t)d.nw;
    LwWork lw;
    lw.st = (LwState*)take(W * sizeof(LwState));
    lw.S = (double*)take(W * LW_NT * 8);
    lw.Lf = (double*)take(W * LW_NT * 8);
    lw.g = (double*)take(W * BA_MAXN * 8);
    lw.dx = (double*)take(W * BA_MAXN * 8);
    lw.dmp = (double*)take(W * BA_MAXN * 8);
    lw.g64 = (double*)take(W * BA_MAXN * 8);
    lw.y64 = (double*)take(W * BA_MAXN * 8);
    lw.cost = (double*)take(W * 8);
    lw.cost64 = (double*)take(W * 8);
    lw.ctrial = (double*)take(W * 8);
    lw.R2 = (double*)take((size_t)slots * 9 * 8);
    lw.p2 = (double*)take((size_t)slots * 3 * 8);
    lw.lmp_trial = (double*)take((size_t)Lt * 3 * 8);
    lw.frz = frz;
    if ((size_t)(p - (char*)scratch) > scratch_bytes) return cudaErrorInvalidValue;
    const bool mixed = mode == XCB_BA_MIXED || mode == XCB_BA_MIXED_NOTC;
    const bool tc = mode == XCB_BA_MIXED;
    const size_t sm_build_tc = lw_build_tc_smem(max_slots);
    const int n = 6 * max_slots, nt = n * (n + 1) / 2;
    const size_t sm_build = lw_build_smem(max_slots, mixed), sm_sys = 8 * (size_t)nt;
    const size_t sm_pass = sizeof(WarpLm<double>) * BA_WARPS;
    static XcbAttrOnce a_bf, a_bd, a_sf, a_sd, a_rf, a_rs, a_bs, a_tc;
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = xcb_smem_attr_once(a_tc, (const void*)k_lw_build_tc, (int)lw_build_tc_smem(BA_MAXP));
    if (e == cudaSuccess) e = xcb_smem_attr_once(a_bf, (const void*)k_lw_build<float>, (int)lw_build_smem(BA_MAXP, true));
    if (e == cudaSuccess) e = xcb_smem_attr_once(a_bd, (const void*)k_lw_build<double>, (int)lw_build_smem(BA_MAXP, false));
    if (e == cudaSuccess) e = xcb_smem_attr_once(a_sf, (const void*)k_lw_solve<float>, 8 * LW_NT);
    if (e == cudaSuccess) e = xcb_smem_attr_once(a_sd, (const void*)k_lw_solve<double>, 8 * LW_NT);
    if (e == cudaSuccess) e = xcb_smem_attr_once(a_rf, (const void*)k_lw_refine, (int)sm_pass);
    if (e == cudaSuccess) e = xcb_smem_attr_once(a_rs, (const void*)k_lw_refine_solve, 8 * LW_NT);
    if (e == cudaSuccess) e = xcb_smem_attr_once(a_bs, (const void*)k_lw_backsub, (int)sm_pass);
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(lw.S, 0, W * LW_NT * 8, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(lw.g, 0, W * BA_MAXN * 8, st)) != cudaSuccess) return e;
    const LwChunk* ch = (const LwChunk*)chunks;
    const unsigned nw = (unsigned)d.nw, nc = (unsigned)nchunks;
    k_lw_init<<<(nw + 127) / 128, 128, 0, st>>>(d, lw, lam0);
    for (int it = 0; it < iters; ++it) {
        if (mixed) {
            if (tc)
                k_lw_build_tc<<<nc, BA_THREADS, sm_build_tc, st>>>(d, lw, ch);
            else
                k_lw_build<float><<<nc, BA_THREADS, sm_build, st>>>(d, lw, ch);
            k_lw_solve<float><<<nw, BA_THREADS, sm_sys, st>>>(d, lw, mode, it);
            for (int rf = 0; rf < BA_REFINE_MAX; ++rf) {
                k_lw_refine<<<nc, BA_THREADS, sm_pass, st>>>(d, lw, ch, rf);
                k_lw_refine_solve<<<nw, BA_THREADS, sm_sys, st>>>(d, lw, rf);
            }
        } else {
            k_lw_build<double><<<nc, BA_THREADS, sm_build, st>>>(d, lw, ch);
            k_lw_solve<double><<<nw, BA_THREADS, sm_sys, st>>>(d, lw, mode, it);
        }
        k_lw_trial<<<nw, 64, 0, st>>>(d, lw, it, dx0, dx0_stride);
        k_lw_backsub<<<nc, BA_THREADS, sm_pass, st>>>(d, lw, ch);
        k_lw_accept<<<nw, 256, 0, st>>>(d, lw, it);
        k_lw_commit<<<nc, 256, 0, st>>>(d, lw, ch);
    }
    k_lw_final<<<(nw + 127) / 128, 128, 0, st>>>(d, lw, stats, iters);
    return cudaGetLastError();
}

int xcb_ba_max_slots() { return BA_MAXP; }
