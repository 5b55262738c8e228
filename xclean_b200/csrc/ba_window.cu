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
// accumulation (shared-memory atomics); the reduced camera system is factored in FP64 (Cholesky); one FP64
// refinement step then solves the residual of the FP64 normal equations, evaluated matrix-free from FP64 Jacobians
// recomputed per observation; back-substitution and the LM cost are FP64.  Mode XCB_BA_FP64 builds everything in
// FP64 (the plain form).
//
// B200 layout: one CTA per SM, persistent; windows are taken from an atomic work counter (largest first, set by the
// host), so uneven windows balance.  Inside a window, one warp per landmark, one lane per observation row (<= 32);
// the reduced system (6P x 6P, P <= 20) lives in shared memory for the whole solve: no host round trip per
// iteration (the reference returns to the host three times per LM iteration).
#include "common.cuh"
#include "ba_kernels.h"

#define BA_THREADS 256
#define BA_WARPS (BA_THREADS / 32)
#define BA_MAXP 20
#define BA_MAXN (6 * BA_MAXP)
#define BA_MAXT 16          // touched slots per landmark (host + observing keyframes)

struct BaWin {
    int P, L, n, hold, lm0, s0;
    double fx, fy, cx, cy, B, hk;
    double Rbc[9], pbc[3], Rcb[9], Px[9];
};

// per-warp scratch: touched slot ids, Hlp blocks (3 x 6) and T = Hll^-1 Hlp (3 x 6) per touched slot
template <typename T>
struct WarpLm {
    int ts[BA_MAXT];
    T Hlp[BA_MAXT][18];
    T Tb[BA_MAXT][18];
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

// One observation row group (left: 2 rows, right: 1 row): residual, Jacobians (Jl wrt (a, b, rho); Jt, Jh wrt the
// target / host body pose blocks), whitened.  -> nd (0 when q2 <= 1e-9).  Follows window.obs_residual /
// obs_jacobians_ws (window.py:126-263).
template <typename T>
__device__ __forceinline__ int obs_lin(const BaWin& w, const T* Rwb, const T* Rwc, const T* pwc, const T* lm, int h,
                                       int t, int cam, const double* z, T isg, T e[2], T Jl[2][3], T Jt[2][6],
                                       T Jh[2][6], bool want_jac)
{
    const T a = lm[0], b = lm[1], rho = lm[2];
    const T* Rh = Rwc + 9 * h;
    const T* Rt = Rwc + 9 * t;
    T d0 = pwc[3 * h] - pwc[3 * t], d1 = pwc[3 * h + 1] - pwc[3 * t + 1], d2 = pwc[3 * h + 2] - pwc[3 * t + 2];
    T Y0 = Rh[0] * a + Rh[1] * b + Rh[2] + rho * d0;
    T Y1 = Rh[3] * a + Rh[4] * b + Rh[5] + rho * d1;
    T Y2 = Rh[6] * a + Rh[7] * b + Rh[8] + rho * d2;
    T q0 = Rt[0] * Y0 + Rt[3] * Y1 + Rt[6] * Y2;
    T q1 = Rt[1] * Y0 + Rt[4] * Y1 + Rt[7] * Y2;
    T q2 = Rt[2] * Y0 + Rt[5] * Y1 + Rt[8] * Y2;
    if (q2 <= (T)1e-9) return 0;
    const T fx = (T)w.fx, fy = (T)w.fy, B = (T)w.B;
    int nd;
    if (cam == 0) {
        e[0] = (fx * q0 / q2 + (T)w.cx - (T)z[0]) * isg;
        e[1] = (fy * q1 / q2 + (T)w.cy - (T)z[1]) * isg;
        nd = 2;
    } else {
        e[0] = (fx * (q0 - rho * B) / q2 + (T)w.cx - (T)z[0]) * isg;
        e[1] = 0;
        nd = 1;
    }
    if (!want_jac) return nd;
    T iq = (T)1 / q2;
    T Dp[2][3];
    if (cam == 0) {
        Dp[0][0] = fx * iq; Dp[0][1] = 0; Dp[0][2] = -fx * q0 * iq * iq;
        Dp[1][0] = 0; Dp[1][1] = fy * iq; Dp[1][2] = -fy * q1 * iq * iq;
    } else {
        Dp[0][0] = fx * iq; Dp[0][1] = 0; Dp[0][2] = -fx * (q0 - rho * B) * iq * iq;
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
        Jl[r][0] = (Dp[r][0] * RcR[0] + Dp[r][1] * RcR[3] + Dp[r][2] * RcR[6]) * isg;
        Jl[r][1] = (Dp[r][0] * RcR[1] + Dp[r][1] * RcR[4] + Dp[r][2] * RcR[7]) * isg;
        Jl[r][2] = (Dp[r][0] * r0 + Dp[r][1] * r1 + Dp[r][2] * r2) * isg;
    }
    if (t == h) {
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
            for (int j = 0; j < 6; ++j) Jt[r][j] = Jh[r][j] = 0;
        return nd;
    }
    T Qx[9] = {0, -q2, q1, q2, 0, -q0, -q1, q0, 0};
    T Mx[9] = {0, -1, b, 1, 0, -a, -b, a, 0};
    T Ah[9], Rct[9], Wt[9], Wh[9], T1[9], T2[9], T3[9], Rcb[9], Px[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) { Rcb[i] = (T)w.Rcb[i]; Px[i] = (T)w.Px[i]; }
    mm3(RcR, Mx, Ah);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Rct[i * 3 + j] = Rt[j * 3 + i];
    mm3(Rwb + 9 * t, Px, Wt);
    mm3(Rwb + 9 * h, Px, Wh);
    mm3(Qx, Rcb, T1);
    mm3(Rct, Wt, T2);
#pragma unroll
    for (int i = 0; i < 9; ++i) T1[i] = T1[i] + rho * T2[i];
    mm3(Ah, Rcb, T2);
    mm3(Rct, Wh, T3);
#pragma unroll
    for (int i = 0; i < 9; ++i) T2[i] = -T2[i] - rho * T3[i];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            Jt[r][j] = (Dp[r][0] * T1[j] + Dp[r][1] * T1[3 + j] + Dp[r][2] * T1[6 + j]) * isg;
            Jh[r][j] = (Dp[r][0] * T2[j] + Dp[r][1] * T2[3 + j] + Dp[r][2] * T2[6 + j]) * isg;
            T v = Dp[r][0] * Rct[j] + Dp[r][1] * Rct[3 + j] + Dp[r][2] * Rct[6 + j];
            Jt[r][3 + j] = -rho * v * isg;
            Jh[r][3 + j] = rho * v * isg;
        }
    return nd;
}

template <typename T>
__device__ __forceinline__ void huber_w(T en, T k, T* wt, T* c)
{
    if (en <= k) { *wt = 1; *c = (T)0.5 * en * en; }
    else { *wt = k / en; *c = k * (en - (T)0.5 * k); }
}

// --------------------------------------------------------------------------------------------- shared layout
struct BaShared {
    BaWin w;
    double Rwb[BA_MAXP * 9], pwb[BA_MAXP * 3], Rwc[BA_MAXP * 9], pwc[BA_MAXP * 3];
    float Rwbf[BA_MAXP * 9], Rwcf[BA_MAXP * 9], pwcf[BA_MAXP * 3];
    double R2[BA_MAXP * 9], p2[BA_MAXP * 3];
    double g[BA_MAXN], y[BA_MAXN], dx[BA_MAXN], rhs[BA_MAXN], dmp[BA_MAXN];
    float bf[BA_MAXN];
    double red[BA_WARPS];
    double cost_cur, cost_new, lam;
    int ok, accepted, status;
    int win;
};

// dynamic shared memory: [S64 n*n doubles][S32 n*n floats | FP64 warp scratch][FP32 warp scratch]
static __host__ __device__ __forceinline__ size_t ba_off_s32(int n) { return ((size_t)n * n * 8 + 15) & ~(size_t)15; }
static __host__ __device__ __forceinline__ size_t ba_s32_bytes(int n)
{
    size_t a = (size_t)n * n * 4, b = sizeof(WarpLm<double>) * BA_WARPS;
    return ((a > b ? a : b) + 15) & ~(size_t)15;
}
size_t xcb_ba_smem_bytes(int maxP)
{
    int n = 6 * maxP;
    return ba_off_s32(n) + ba_s32_bytes(n) + sizeof(WarpLm<float>) * BA_WARPS;
}

// ---------------------------------------------------------------------------------- per-landmark linearisation
// Warp-level: lane i holds observation row group i; results: Hll (damped), bl, the touched-slot Hlp blocks in the warp
// scratch.  -> 1 when the landmark enters the system (lm_ok), cost (FP64) added to *cost by lane 0.
template <typename T>
struct LaneObs {
    int nd, t;
    T wt, e[2], Jl[2][3], Jt[2][6], Jh[2][6];
};

template <typename T>
__device__ __forceinline__ bool lin_landmark(const BaShared& sh, const XcbBaWindows& d, const T* Rwb, const T* Rwc,
                                             const T* pwc, int l, double lam, LaneObs<T>& o, T Hll[9], T bl[3],
                                             WarpLm<T>& wl, int* nts, double* cost, const double* lmp_src)
{
    const int lane = threadIdx.x & 31;
    const BaWin& w = sh.w;
    const int gl = w.lm0 + l;
    const int h = d.lm_host[gl];
    const int k0 = d.lm_ob[gl], k1 = d.lm_ob[gl + 1];
    T lm[3] = {(T)lmp_src[3 * gl], (T)lmp_src[3 * gl + 1], (T)lmp_src[3 * gl + 2]};
    o.nd = 0;
    o.t = -1;
    o.wt = 0;
    double c = 0.0;
    const int k = k0 + lane;
    if (k < k1 && d.ob_valid[k]) {
        o.t = d.ob_pose[k];
        o.nd = obs_lin<T>(w, Rwb, Rwc, pwc, lm, h, o.t, d.ob_cam[k], d.ob_z + 2 * k, (T)d.ob_isig[k], o.e, o.Jl, o.Jt,
                          o.Jh, true);
        if (o.nd) {
            T en2 = o.e[0] * o.e[0] + o.e[1] * o.e[1];
            T en = sqrt(en2), cc;
            huber_w<T>(en, (T)w.hk, &o.wt, &cc);
            c = (double)cc;
        } else {
            o.t = -1;
        }
    }
    // landmark block and gradient
    T hv[9], bv[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
        for (int j = 0; j < 3; ++j) hv[i * 3 + j] = o.wt * (o.Jl[0][i] * o.Jl[0][j] + o.Jl[1][i] * o.Jl[1][j]);
        bv[i] = o.wt * (o.Jl[0][i] * o.e[0] + o.Jl[1][i] * o.e[1]);
    }
    if (!o.nd) {
#pragma unroll
        for (int i = 0; i < 9; ++i) hv[i] = 0;
        bv[0] = bv[1] = bv[2] = 0;
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) Hll[i] = warp_sum(hv[i]);
#pragma unroll
    for (int i = 0; i < 3; ++i) bl[i] = warp_sum(bv[i]);
    const int nobs = __popc(__ballot_sync(0xffffffffu, o.nd > 0));
    c = warp_sum(c);
    if (d.rho_isig[gl] > 0.0) {
        T ris = (T)d.rho_isig[gl];
        T r0 = (lm[2] - (T)d.rho_meas[gl]) * ris, wt, cc;
        huber_w<T>(fabs(r0), (T)w.hk, &wt, &cc);
        c += (double)cc;
        Hll[8] += wt * ris * ris;
        bl[2] += wt * ris * r0;
    }
    if (lane == 0 && cost) *cost += c;
    // touched slots: the observing keyframes other than the host, and the host when any exists
    const bool pose_obs = o.nd > 0 && o.t != h;
    unsigned tm = 0;
    {
        unsigned mine = pose_obs ? (1u << o.t) : 0u;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) mine |= __shfl_xor_sync(0xffffffffu, mine, off);
        tm = mine;
        if (tm) tm |= 1u << h;
    }
    int nt = 0;
    for (unsigned m = tm; m; m &= m - 1) {
        if (lane == 0) wl.ts[nt] = __ffs(m) - 1;
        ++nt;
    }
    *nts = nt;
    // Hlp blocks: slot s gets w Jl^T Jt from its own observations and, for the host, w Jl^T Jh from all of them
    {
        unsigned m = tm;
        for (int si = 0; si < nt; ++si) {
            const int s = __ffs(m) - 1;
            m &= m - 1;
            T a[18];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 6; ++j) {
                    T v = 0;
                    if (pose_obs && o.t == s) v += o.wt * (o.Jl[0][i] * o.Jt[0][j] + o.Jl[1][i] * o.Jt[1][j]);
                    if (pose_obs && s == h) v += o.wt * (o.Jl[0][i] * o.Jh[0][j] + o.Jl[1][i] * o.Jh[1][j]);
                    a[i * 6 + j] = v;
                }
#pragma unroll
            for (int q = 0; q < 18; ++q) {
                T v = warp_sum(a[q]);
                if (lane == 0) wl.Hlp[si][q] = v;
            }
        }
    }
    // damping and the conditioning guard (window.build_system)
#pragma unroll
    for (int i = 0; i < 3; ++i) Hll[i * 4] += (T)lam * Hll[i * 4] + (T)1e-12;
    __syncwarp();
    T det = Hll[0] * (Hll[4] * Hll[8] - Hll[5] * Hll[7]) - Hll[1] * (Hll[3] * Hll[8] - Hll[5] * Hll[6])
            + Hll[2] * (Hll[3] * Hll[7] - Hll[4] * Hll[6]);
    T tr = Hll[0] + Hll[4] + Hll[8];
    return nobs > 0 && det > (T)1e-18 * tr * tr * tr && isfinite(det);
}

template <typename T>
__device__ __forceinline__ void inv3(const T H[9], T Hi[9])
{
    // closed form as window.build_system; computed in float64 for every precision (the 3x3 inverse of a low-parallax
    // landmark is the ill-conditioned step)
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
// S (n x n, T) and the gradient gb (n, T) in shared memory, accumulated with shared-memory atomics
template <typename T>
__device__ void pass_build(BaShared& sh, const XcbBaWindows& d, T* S, T* gb, WarpLm<T>* wls, double* cost)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int n = sh.w.n;
    const T* Rwb = nullptr;
    const T* Rwc = nullptr;
    const T* pwc = nullptr;
    if (sizeof(T) == 4) { Rwb = (const T*)sh.Rwbf; Rwc = (const T*)sh.Rwcf; pwc = (const T*)sh.pwcf; }
    else { Rwb = (const T*)sh.Rwb; Rwc = (const T*)sh.Rwc; pwc = (const T*)sh.pwc; }
    WarpLm<T>& wl = wls[wid];
    double c_local = 0.0;
    for (int l = wid; l < sh.w.L; l += BA_WARPS) {
        if (!d.lm_mask[sh.w.lm0 + l]) continue;
        LaneObs<T> o;
        T Hll[9], bl[3];
        int nt;
        const bool ok = lin_landmark<T>(sh, d, Rwb, Rwc, pwc, l, sh.lam, o, Hll, bl, wl, &nt, &c_local, d.lmp);
        const int h = d.lm_host[sh.w.lm0 + l];
        // pose-pose blocks and the pose gradient of this lane's observation
        if (o.nd > 0 && o.t != h) {
            const int t = o.t;
            for (int i = 0; i < 6; ++i) {
                atomicAdd(&gb[6 * t + i], o.wt * (o.Jt[0][i] * o.e[0] + o.Jt[1][i] * o.e[1]));
                atomicAdd(&gb[6 * h + i], o.wt * (o.Jh[0][i] * o.e[0] + o.Jh[1][i] * o.e[1]));
                for (int j = 0; j < 6; ++j) {
                    T tt = o.wt * (o.Jt[0][i] * o.Jt[0][j] + o.Jt[1][i] * o.Jt[1][j]);
                    T hh = o.wt * (o.Jh[0][i] * o.Jh[0][j] + o.Jh[1][i] * o.Jh[1][j]);
                    T th = o.wt * (o.Jt[0][i] * o.Jh[0][j] + o.Jt[1][i] * o.Jh[1][j]);
                    atomicAdd(&S[(6 * t + i) * n + 6 * t + j], tt);
                    atomicAdd(&S[(6 * h + i) * n + 6 * h + j], hh);
                    atomicAdd(&S[(6 * t + i) * n + 6 * h + j], th);
                    atomicAdd(&S[(6 * h + j) * n + 6 * t + i], th);
                }
            }
        }
        if (!ok || nt == 0) { __syncwarp(); continue; }
        T Hi[9];
        inv3<T>(Hll, Hi);
        // T blocks = Hll^-1 Hlp[s]
        for (int q = lane; q < nt * 18; q += 32) {
            const int si = q / 18, e = q % 18, i = e / 6, j = e % 6;
            wl.Tb[si][e] = Hi[i * 3] * wl.Hlp[si][j] + Hi[i * 3 + 1] * wl.Hlp[si][6 + j] + Hi[i * 3 + 2] * wl.Hlp[si][12 + j];
        }
        __syncwarp();
        // gradient: g[s] -= Hlp[s]^T Hll^-1 bl
        T HiB[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) HiB[i] = Hi[i * 3] * bl[0] + Hi[i * 3 + 1] * bl[1] + Hi[i * 3 + 2] * bl[2];
        for (int q = lane; q < nt * 6; q += 32) {
            const int si = q / 6, i = q % 6;
            T acc = wl.Hlp[si][i] * HiB[0] + wl.Hlp[si][6 + i] * HiB[1] + wl.Hlp[si][12 + i] * HiB[2];
            atomicAdd(&gb[6 * wl.ts[si] + i], -acc);
        }
        // Schur: S[s2][s1] -= Hlp[s2]^T T[s1] for every ordered pair of touched slots
        const int np = nt * nt * 36;
        for (int q = lane; q < np; q += 32) {
            const int pr = q / 36, e = q % 36, i = e / 6, j = e % 6;
            const int a2 = pr / nt, a1 = pr % nt;
            T acc = wl.Hlp[a2][i] * wl.Tb[a1][j] + wl.Hlp[a2][6 + i] * wl.Tb[a1][6 + j]
                    + wl.Hlp[a2][12 + i] * wl.Tb[a1][12 + j];
            atomicAdd(&S[(6 * wl.ts[a2] + i) * n + 6 * wl.ts[a1] + j], -acc);
        }
        __syncwarp();
    }
    if (cost) {
        if (lane == 0) sh.red[wid] = c_local;
    }
}

// ------------------------------------------------------------------------ pass B: FP64 gradient and S_true dx
// g (reduced gradient) and y = S dx, matrix-free from FP64 Jacobians (the refinement residual's ingredients)
__device__ void pass_refine(BaShared& sh, const XcbBaWindows& d, WarpLm<double>* wls)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpLm<double>& wl = wls[wid];
    double c_local = 0.0;
    for (int l = wid; l < sh.w.L; l += BA_WARPS) {
        if (!d.lm_mask[sh.w.lm0 + l]) continue;
        LaneObs<double> o;
        double Hll[9], bl[3];
        int nt;
        const bool ok = lin_landmark<double>(sh, d, sh.Rwb, sh.Rwc, sh.pwc, l, sh.lam, o, Hll, bl, wl, &nt, &c_local,
                                             d.lmp);
        const int h = d.lm_host[sh.w.lm0 + l];
        if (o.nd > 0 && o.t != h) {
            const int t = o.t;
            double jx[2];
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                double a = 0.0;
#pragma unroll
                for (int j = 0; j < 6; ++j) a += o.Jt[r][j] * sh.dx[6 * t + j] + o.Jh[r][j] * sh.dx[6 * h + j];
                jx[r] = o.wt * a;
            }
            for (int i = 0; i < 6; ++i) {
                atomicAdd(&sh.g[6 * t + i], o.wt * (o.Jt[0][i] * o.e[0] + o.Jt[1][i] * o.e[1]));
                atomicAdd(&sh.g[6 * h + i], o.wt * (o.Jh[0][i] * o.e[0] + o.Jh[1][i] * o.e[1]));
                atomicAdd(&sh.y[6 * t + i], o.Jt[0][i] * jx[0] + o.Jt[1][i] * jx[1]);
                atomicAdd(&sh.y[6 * h + i], o.Jh[0][i] * jx[0] + o.Jh[1][i] * jx[1]);
            }
        }
        if (!ok || nt == 0) { __syncwarp(); continue; }
        double Hi[9];
        inv3<double>(Hll, Hi);
        // v = sum_s Hlp[s] dx_s, u = Hi v, y[s] -= Hlp[s]^T u ; g[s] -= Hlp[s]^T Hi bl
        double v[3] = {0.0, 0.0, 0.0};
        for (int si = 0; si < nt; ++si) {
            const int s = wl.ts[si];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 6; ++j) v[i] += wl.Hlp[si][i * 6 + j] * sh.dx[6 * s + j];
        }
        double u[3], HiB[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            u[i] = Hi[i * 3] * v[0] + Hi[i * 3 + 1] * v[1] + Hi[i * 3 + 2] * v[2];
            HiB[i] = Hi[i * 3] * bl[0] + Hi[i * 3 + 1] * bl[1] + Hi[i * 3 + 2] * bl[2];
        }
        for (int q = lane; q < nt * 6; q += 32) {
            const int si = q / 6, i = q % 6, s = wl.ts[si];
            double hu = wl.Hlp[si][i] * u[0] + wl.Hlp[si][6 + i] * u[1] + wl.Hlp[si][12 + i] * u[2];
            double hb = wl.Hlp[si][i] * HiB[0] + wl.Hlp[si][6 + i] * HiB[1] + wl.Hlp[si][12 + i] * HiB[2];
            atomicAdd(&sh.y[6 * s + i], -hu);
            atomicAdd(&sh.g[6 * s + i], -hb);
        }
        __syncwarp();
    }
    if (lane == 0) sh.red[wid] = c_local;
}

// ------------------------------------------------------------------ pass C: back-substitution (FP64) -> trial lmp
__device__ void pass_backsub(BaShared& sh, const XcbBaWindows& d, WarpLm<double>* wls, double* lmp_trial)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpLm<double>& wl = wls[wid];
    for (int l = wid; l < sh.w.L; l += BA_WARPS) {
        const int gl = sh.w.lm0 + l;
        if (!d.lm_mask[gl]) {
            if (lane < 3) lmp_trial[3 * gl + lane] = d.lmp[3 * gl + lane];
            continue;
        }
        LaneObs<double> o;
        double Hll[9], bl[3];
        int nt;
        const bool ok = lin_landmark<double>(sh, d, sh.Rwb, sh.Rwc, sh.pwc, l, sh.lam, o, Hll, bl, wl, &nt, nullptr,
                                             d.lmp);
        if (lane == 0) {
            double cur[3] = {d.lmp[3 * gl], d.lmp[3 * gl + 1], d.lmp[3 * gl + 2]};
            double out[3] = {cur[0], cur[1], cur[2]};
            if (ok) {
                double Hi[9];
                inv3<double>(Hll, Hi);
                double v[3] = {bl[0], bl[1], bl[2]};
                for (int si = 0; si < nt; ++si) {
                    const int s = wl.ts[si];
                    for (int i = 0; i < 3; ++i) {
                        double acc = 0.0;
                        for (int j = 0; j < 6; ++j) acc += wl.Hlp[si][i * 6 + j] * sh.dx[6 * s + j];
                        v[i] += acc;
                    }
                }
                double dl[3];
                for (int i = 0; i < 3; ++i) dl[i] = -(Hi[i * 3] * v[0] + Hi[i * 3 + 1] * v[1] + Hi[i * 3 + 2] * v[2]);
                double r = cur[2] + dl[2];
                if (r > 1e-9 && isfinite(r)) { out[0] = cur[0] + dl[0]; out[1] = cur[1] + dl[1]; out[2] = r; }
            }
            lmp_trial[3 * gl] = out[0];
            lmp_trial[3 * gl + 1] = out[1];
            lmp_trial[3 * gl + 2] = out[2];
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------------------------- pass D: FP64 cost of a state
__device__ void pass_cost(BaShared& sh, const XcbBaWindows& d, const double* Rwb, const double* Rwc, const double* pwc,
                          const double* lmp)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double c = 0.0;
    for (int l = wid; l < sh.w.L; l += BA_WARPS) {
        const int gl = sh.w.lm0 + l;
        if (!d.lm_mask[gl]) continue;
        const int h = d.lm_host[gl];
        const double lm[3] = {lmp[3 * gl], lmp[3 * gl + 1], lmp[3 * gl + 2]};
        for (int k = d.lm_ob[gl] + lane; k < d.lm_ob[gl + 1]; k += 32) {
            if (!d.ob_valid[k]) continue;
            double e[2], Jl[2][3], Jt[2][6], Jh[2][6];
            int nd = obs_lin<double>(sh.w, Rwb, Rwc, pwc, lm, h, d.ob_pose[k], d.ob_cam[k], d.ob_z + 2 * k,
                                     d.ob_isig[k], e, Jl, Jt, Jh, false);
            if (!nd) { c += 1e6; continue; }
            double wt, cc;
            huber_w<double>(sqrt(e[0] * e[0] + e[1] * e[1]), sh.w.hk, &wt, &cc);
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
// in-place lower Cholesky of S (n x n, row-major) -> 0 ok, else -1 (not positive definite)
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
        const int m = n - j - 1;
        for (int p = threadIdx.x; p < m * m; p += blockDim.x) {
            const int i = j + 1 + p / m, c = j + 1 + p % m;
            if (c <= i) S[i * n + c] -= S[i * n + j] * S[c * n + j];
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

__device__ void cam_poses_sh(BaShared& sh, const double* Rwb, const double* pwb, double* Rwc, double* pwc)
{
    for (int q = threadIdx.x; q < sh.w.P * 9; q += blockDim.x) {
        const int s = q / 9, i = (q % 9) / 3, j = q % 3;
        double acc = 0.0;
        for (int k = 0; k < 3; ++k) acc += Rwb[9 * s + 3 * i + k] * sh.w.Rbc[3 * k + j];
        Rwc[q] = acc;
    }
    for (int q = threadIdx.x; q < sh.w.P * 3; q += blockDim.x) {
        const int s = q / 3, i = q % 3;
        double acc = pwb[q];
        for (int k = 0; k < 3; ++k) acc += Rwb[9 * s + 3 * i + k] * sh.w.pbc[k];
        pwc[q] = acc;
    }
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
            sh.lam = lam0; sh.accepted = 0; sh.status = 0;
        }
        __syncthreads();
        const int P = sh.w.P, n = sh.w.n, L = sh.w.L, s0 = sh.w.s0;
        if (P > BA_MAXP) {
            if (tid == 0) { stats[8 * w + 4] = -1.0; }
            __syncthreads();
            continue;
        }
        for (int q = tid; q < P * 9; q += blockDim.x) sh.Rwb[q] = d.Rwb[9 * s0 + q];
        for (int q = tid; q < P * 3; q += blockDim.x) sh.pwb[q] = d.pwb[3 * s0 + q];
        __syncthreads();
        double* S64 = (double*)dsm;
        float* S32 = (float*)(dsm + ba_off_s32(n));
        WarpLm<double>* wl64 = (WarpLm<double>*)(dsm + ba_off_s32(n));
        WarpLm<float>* wl32 = (WarpLm<float>*)(dsm + ba_off_s32(n) + ba_s32_bytes(n));
        double cost0 = 0.0;
        for (int it = 0; it < iters; ++it) {
            cam_poses_sh(sh, sh.Rwb, sh.pwb, sh.Rwc, sh.pwc);
            __syncthreads();
            for (int q = tid; q < P * 9; q += blockDim.x) { sh.Rwbf[q] = (float)sh.Rwb[q]; sh.Rwcf[q] = (float)sh.Rwc[q]; }
            for (int q = tid; q < P * 3; q += blockDim.x) sh.pwcf[q] = (float)sh.pwc[q];
            for (int q = tid; q < n; q += blockDim.x) { sh.g[q] = 0.0; sh.y[q] = 0.0; sh.bf[q] = 0.0f; }
            double c_tot;
            if (mode == XCB_BA_MIXED) {
                for (int q = tid; q < n * n; q += blockDim.x) S32[q] = 0.0f;
                __syncthreads();
                pass_build<float>(sh, d, S32, sh.bf, wl32, nullptr);
                __syncthreads();
                for (int q = tid; q < n * n; q += blockDim.x) S64[q] = (double)S32[q];
                for (int q = tid; q < n; q += blockDim.x) sh.rhs[q] = (double)sh.bf[q];
            } else {
                for (int q = tid; q < n * n; q += blockDim.x) S64[q] = 0.0;
                __syncthreads();
                pass_build<double>(sh, d, S64, sh.g, wl64, &c_tot);
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
                    pass_cost(sh, d, sh.Rwb, sh.Rwc, sh.pwc, d.lmp);
                    c_tot = block_sum_red(sh);
                }
                if (it == 0) cost0 = c_tot;
                if (tid == 0) { sh.lam *= 10.0; sh.cost_cur = c_tot; }
                __syncthreads();
                continue;
            }
            chol_solve(S64, n, sh.dx);
            if (mode == XCB_BA_MIXED) {
                // one FP64 refinement step: rho = -g - (S + D) dx with S dx matrix-free in FP64
                for (int q = tid; q < n; q += blockDim.x) { sh.g[q] = 0.0; sh.y[q] = 0.0; }
                __syncthreads();
                pass_refine(sh, d, wl64);
                c_tot = block_sum_red(sh);
                for (int q = tid; q < n; q += blockDim.x) {
                    double r = -sh.g[q] - sh.y[q] - sh.dmp[q] * sh.dx[q];
                    if (hs >= 0 && q / 6 == hs) r = 0.0;
                    sh.rhs[q] = r;
                }
                __syncthreads();
                chol_solve(S64, n, sh.rhs);
                for (int q = tid; q < n; q += blockDim.x) sh.dx[q] += sh.rhs[q];
                __syncthreads();
            }
            if (it == 0) {
                cost0 = c_tot;
                if (dx0)
                    for (int q = tid; q < n; q += blockDim.x) dx0[(size_t)w * dx0_stride + q] = sh.dx[q];
            }
            // trial state: landmarks (back-substitution), poses
            pass_backsub(sh, d, wl64, lmp_trial);
            for (int s = tid; s < P; s += blockDim.x) {
                double Re[9];
                so3_exp(sh.dx + 6 * s, Re);
                double R[9];
                for (int i = 0; i < 9; ++i) R[i] = sh.Rwb[9 * s + i];
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j)
                        sh.R2[9 * s + 3 * i + j] = R[3 * i] * Re[j] + R[3 * i + 1] * Re[3 + j] + R[3 * i + 2] * Re[6 + j];
                for (int i = 0; i < 3; ++i) sh.p2[3 * s + i] = sh.pwb[3 * s + i] + sh.dx[6 * s + 3 + i];
            }
            __syncthreads();
            // the trial cost: camera poses of the trial state into Rwc / pwc (recomputed next iteration anyway)
            cam_poses_sh(sh, sh.R2, sh.p2, sh.Rwc, sh.pwc);
            __syncthreads();
            pass_cost(sh, d, sh.R2, sh.Rwc, sh.pwc, lmp_trial);
            const double c_new = block_sum_red(sh);
            const bool acc = c_new < c_tot;
            if (acc) {
                for (int q = tid; q < P * 9; q += blockDim.x) sh.Rwb[q] = sh.R2[q];
                for (int q = tid; q < P * 3; q += blockDim.x) sh.pwb[q] = sh.p2[q];
                const int lm0 = sh.w.lm0;
                for (int q = tid; q < 3 * L; q += blockDim.x) d.lmp[3 * lm0 + q] = lmp_trial[3 * lm0 + q];
            }
            if (tid == 0) {
                if (acc) { sh.lam = fmax(sh.lam / 10.0, 1e-12); sh.accepted += 1; sh.cost_cur = c_new; }
                else { sh.lam *= 10.0; sh.cost_cur = c_tot; }
            }
            __syncthreads();
        }
        for (int q = tid; q < P * 9; q += blockDim.x) d.Rwb[9 * s0 + q] = sh.Rwb[q];
        for (int q = tid; q < P * 3; q += blockDim.x) d.pwb[3 * s0 + q] = sh.pwb[q];
        if (tid == 0) {
            stats[8 * w + 0] = cost0;
            stats[8 * w + 1] = sh.cost_cur;
            stats[8 * w + 2] = sh.accepted;
            stats[8 * w + 3] = sh.lam;
            stats[8 * w + 4] = 0.0;
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
