/*
 * ba_oracle.c -- CPU ORACLE of the sliding-window BA (test infrastructure and the CPU baseline; never the product).
 *
 * A restatement, in C and float64, of the reference's stereo window solve src/xclean/vio/window.py:
 *   _cam_poses (:108-122), obs_residual (:126-146), obs_jacobians_ws (:165-263), _huber (:282-286),
 *   build_system (:292-463), visual_cost (:467-493), back_substitute (:497-519), apply_update (:523-547),
 *   so3_exp_nb (:43-62) and the fixed-iteration LM of solve (:889-982) for a purely visual window (no marginal
 *   prior, no IMU terms: those are out of this path), and the pose-free block's posefree_cost / posefree_step
 *   (:550-765).  Loops and expression order follow the
 *   reference's numba code; the reduced system is factored by a plain float64 Cholesky (the reference calls
 *   np.linalg.cholesky + two np.linalg.solve, so the step agrees to rounding, not bit for bit).
 * Extension used by the synthetic windows: `hold` = a slot held fixed (its rows / columns of the reduced system
 * replaced by the identity and its gradient zeroed, as backend/ba._solve_np holds its gauge, ba.py:810-815).
 *
 * Build: gcc -O2 -ffp-contract=off -fno-fast-math -fopenmp (oracle/build.py).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int P, L, M;
    double* Rwb;             /* P*9 (in / out) */
    double* pwb;             /* P*3 (in / out) */
    const double* Rbc;       /* 9 */
    const double* pbc;       /* 3 */
    double* lmp;             /* L*3 (in / out) */
    const int64_t* lm_host;  /* L */
    const uint8_t* lm_mask;  /* L */
    const double* rho_meas;  /* L */
    const double* rho_isig;  /* L */
    const int64_t* ob_start; /* L+1 */
    const int64_t* ob_pose;  /* M */
    const int64_t* ob_cam;   /* M */
    const double* ob_z;      /* M*2 */
    const double* ob_isig;   /* M */
    const uint8_t* ob_valid; /* M */
    double fx, fy, cx, cy, B, huber_k;
    int hold;                /* held slot, -1 = none */
} XoWindow;

#define M3(A, s, i, j) ((A)[(s) * 9 + (i) * 3 + (j)])

static void cam_poses(int P, const double* Rwb, const double* pwb, const double* Rbc, const double* pbc, double* Rwc,
                      double* pwc)
{
    for (int s = 0; s < P; ++s)
        for (int i = 0; i < 3; ++i) {
            for (int j = 0; j < 3; ++j) {
                double acc = 0.0;
                for (int k = 0; k < 3; ++k) acc += M3(Rwb, s, i, k) * Rbc[k * 3 + j];
                M3(Rwc, s, i, j) = acc;
            }
            double acc = pwb[s * 3 + i];
            for (int k = 0; k < 3; ++k) acc += M3(Rwb, s, i, k) * pbc[k];
            pwc[s * 3 + i] = acc;
        }
}

/* -> nd; *q2o = q2; e[0..nd) the unwhitened residual (untouched when q2 <= 1e-9) */
static int obs_residual(const double* Rwc, const double* pwc, const double* lm, int h, int t, int cam, const double* z,
                        double fx, double fy, double cx, double cy, double B, double* e, double* q2o)
{
    double a = lm[0], b = lm[1], rho = lm[2];
    double Y0 = M3(Rwc, h, 0, 0) * a + M3(Rwc, h, 0, 1) * b + M3(Rwc, h, 0, 2) + rho * (pwc[h * 3] - pwc[t * 3]);
    double Y1 = M3(Rwc, h, 1, 0) * a + M3(Rwc, h, 1, 1) * b + M3(Rwc, h, 1, 2) + rho * (pwc[h * 3 + 1] - pwc[t * 3 + 1]);
    double Y2 = M3(Rwc, h, 2, 0) * a + M3(Rwc, h, 2, 1) * b + M3(Rwc, h, 2, 2) + rho * (pwc[h * 3 + 2] - pwc[t * 3 + 2]);
    double q0 = M3(Rwc, t, 0, 0) * Y0 + M3(Rwc, t, 1, 0) * Y1 + M3(Rwc, t, 2, 0) * Y2;
    double q1 = M3(Rwc, t, 0, 1) * Y0 + M3(Rwc, t, 1, 1) * Y1 + M3(Rwc, t, 2, 1) * Y2;
    double q2 = M3(Rwc, t, 0, 2) * Y0 + M3(Rwc, t, 1, 2) * Y1 + M3(Rwc, t, 2, 2) * Y2;
    *q2o = q2;
    if (cam == 0) {
        if (q2 <= 1e-9) return 2;
        e[0] = fx * q0 / q2 + cx - z[0];
        e[1] = fy * q1 / q2 + cy - z[1];
        return 2;
    }
    if (q2 <= 1e-9) return 1;
    e[0] = fx * (q0 - rho * B) / q2 + cx - z[0];
    return 1;
}

static void mm3(const double* A, const double* Bm, double* out)   /* out = A B */
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) out[i * 3 + j] = A[i * 3 + 0] * Bm[0 * 3 + j] + A[i * 3 + 1] * Bm[1 * 3 + j] + A[i * 3 + 2] * Bm[2 * 3 + j];
}

static void mtm3(const double* A, const double* Bm, double* out)  /* out = A^T B */
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) out[i * 3 + j] = A[0 * 3 + i] * Bm[0 * 3 + j] + A[1 * 3 + i] * Bm[1 * 3 + j] + A[2 * 3 + i] * Bm[2 * 3 + j];
}

/* Jacobians of the unwhitened residual: Jl (nd x 3) wrt (a, b, rho); Jt, Jh (nd x 6) wrt the target / host body
   pose blocks [dphi, dp] (zero when t == h).  Rcb = Rbc^T, Px = [pbc]x. */
static int obs_jacobians(const double* Rwb, const double* Rwc, const double* pwc, const double* Rcb, const double* Px,
                         const double* lm, int h, int t, int cam, double fx, double fy, double B, double Jl[2][3],
                         double Jt[2][6], double Jh[2][6])
{
    double a = lm[0], b = lm[1], rho = lm[2];
    double d0 = pwc[h * 3] - pwc[t * 3], d1 = pwc[h * 3 + 1] - pwc[t * 3 + 1], d2 = pwc[h * 3 + 2] - pwc[t * 3 + 2];
    double Y0 = M3(Rwc, h, 0, 0) * a + M3(Rwc, h, 0, 1) * b + M3(Rwc, h, 0, 2) + rho * d0;
    double Y1 = M3(Rwc, h, 1, 0) * a + M3(Rwc, h, 1, 1) * b + M3(Rwc, h, 1, 2) + rho * d1;
    double Y2 = M3(Rwc, h, 2, 0) * a + M3(Rwc, h, 2, 1) * b + M3(Rwc, h, 2, 2) + rho * d2;
    double q0 = M3(Rwc, t, 0, 0) * Y0 + M3(Rwc, t, 1, 0) * Y1 + M3(Rwc, t, 2, 0) * Y2;
    double q1 = M3(Rwc, t, 0, 1) * Y0 + M3(Rwc, t, 1, 1) * Y1 + M3(Rwc, t, 2, 1) * Y2;
    double q2 = M3(Rwc, t, 0, 2) * Y0 + M3(Rwc, t, 1, 2) * Y1 + M3(Rwc, t, 2, 2) * Y2;
    int nd = cam == 0 ? 2 : 1;
    double iq = 1.0 / q2;
    double Dp[2][3];
    if (cam == 0) {
        Dp[0][0] = fx * iq; Dp[0][1] = 0.0; Dp[0][2] = -fx * q0 * iq * iq;
        Dp[1][0] = 0.0; Dp[1][1] = fy * iq; Dp[1][2] = -fy * q1 * iq * iq;
    } else {
        Dp[0][0] = fx * iq; Dp[0][1] = 0.0; Dp[0][2] = -fx * (q0 - rho * B) * iq * iq;
    }
    double RcR[9];
    mtm3(Rwc + t * 9, Rwc + h * 9, RcR);
    double r0 = M3(Rwc, t, 0, 0) * d0 + M3(Rwc, t, 1, 0) * d1 + M3(Rwc, t, 2, 0) * d2;
    double r1 = M3(Rwc, t, 0, 1) * d0 + M3(Rwc, t, 1, 1) * d1 + M3(Rwc, t, 2, 1) * d2;
    double r2 = M3(Rwc, t, 0, 2) * d0 + M3(Rwc, t, 1, 2) * d1 + M3(Rwc, t, 2, 2) * d2;
    if (cam == 1) r0 -= B;
    for (int r = 0; r < nd; ++r) {
        Jl[r][0] = Dp[r][0] * RcR[0] + Dp[r][1] * RcR[3] + Dp[r][2] * RcR[6];
        Jl[r][1] = Dp[r][0] * RcR[1] + Dp[r][1] * RcR[4] + Dp[r][2] * RcR[7];
        Jl[r][2] = Dp[r][0] * r0 + Dp[r][1] * r1 + Dp[r][2] * r2;
    }
    if (t == h) {
        for (int r = 0; r < nd; ++r)
            for (int j = 0; j < 6; ++j) { Jt[r][j] = 0.0; Jh[r][j] = 0.0; }
        return nd;
    }
    double Qx[9] = {0.0, -q2, q1, q2, 0.0, -q0, -q1, q0, 0.0};
    double Mx[9] = {0.0, -1.0, b, 1.0, 0.0, -a, -b, a, 0.0};
    double Ah[9], Rct[9], Wt[9], Wh[9], T1[9], T2[9], T3[9];
    mm3(RcR, Mx, Ah);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Rct[i * 3 + j] = M3(Rwc, t, j, i);
    mm3(Rwb + t * 9, Px, Wt);
    mm3(Rwb + h * 9, Px, Wh);
    mm3(Qx, Rcb, T1);
    mm3(Rct, Wt, T2);
    for (int i = 0; i < 9; ++i) T1[i] = T1[i] + rho * T2[i];
    mm3(Ah, Rcb, T2);
    mm3(Rct, Wh, T3);
    for (int i = 0; i < 9; ++i) T2[i] = -T2[i] - rho * T3[i];
    for (int r = 0; r < nd; ++r)
        for (int j = 0; j < 3; ++j) {
            Jt[r][j] = Dp[r][0] * T1[0 * 3 + j] + Dp[r][1] * T1[1 * 3 + j] + Dp[r][2] * T1[2 * 3 + j];
            Jh[r][j] = Dp[r][0] * T2[0 * 3 + j] + Dp[r][1] * T2[1 * 3 + j] + Dp[r][2] * T2[2 * 3 + j];
            double v = Dp[r][0] * Rct[0 * 3 + j] + Dp[r][1] * Rct[1 * 3 + j] + Dp[r][2] * Rct[2 * 3 + j];
            Jt[r][3 + j] = -rho * v;
            Jh[r][3 + j] = rho * v;
        }
    return nd;
}

static void huber(double en, double k, double* w, double* c)
{
    if (en <= k) { *w = 1.0; *c = 0.5 * en * en; }
    else { *w = k / en; *c = k * (en - 0.5 * k); }
}

static void prep_extrinsic(const double* Rbc, const double* pbc, double* Rcb, double* Px)
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Rcb[i * 3 + j] = Rbc[j * 3 + i];
    double p[9] = {0.0, -pbc[2], pbc[1], pbc[2], 0.0, -pbc[0], -pbc[1], pbc[0], 0.0};
    memcpy(Px, p, sizeof(p));
}

/* build_system: linearise every valid observation; Schur the landmarks into H (6P x 6P) and bvec.  Hlp (L,P,3,6),
   Hll_inv (L,9), bl_out (L,3), lm_ok (L), ob_chi2 (M).  -> robust cost. */
double xo_ba_build_system(const XoWindow* w, const double* Rwb, const double* pwb, const double* lmp, double lam,
                          double* H, double* bvec, double* Hll_inv, double* bl_out, double* Hlp, uint8_t* lm_ok,
                          double* ob_chi2)
{
    const int P = w->P, L = w->L, n = 6 * P;
    double* Rwc = (double*)malloc(sizeof(double) * 9 * P);
    double* pwc = (double*)malloc(sizeof(double) * 3 * P);
    cam_poses(P, Rwb, pwb, w->Rbc, w->pbc, Rwc, pwc);
    double Rcb[9], Px[9];
    prep_extrinsic(w->Rbc, w->pbc, Rcb, Px);
    memset(H, 0, sizeof(double) * n * n);
    memset(bvec, 0, sizeof(double) * n);
    uint8_t* touched = (uint8_t*)malloc(P);
    double cost = 0.0;
    for (int l = 0; l < L; ++l) {
        lm_ok[l] = 0;
        if (!w->lm_mask[l]) continue;
        int h = (int)w->lm_host[l];
        const double* lm = lmp + 3 * l;
        double Hll[9] = {0}, bl[3] = {0};
        double* Hl = Hlp + (size_t)l * P * 18;
        memset(Hl, 0, sizeof(double) * P * 18);
        memset(touched, 0, P);
        int nobs = 0;
        for (int64_t k = w->ob_start[l]; k < w->ob_start[l + 1]; ++k) {
            ob_chi2[k] = INFINITY;
            if (!w->ob_valid[k]) continue;
            int t = (int)w->ob_pose[k], cam = (int)w->ob_cam[k];
            double e[2] = {0, 0}, q2;
            int nd = obs_residual(Rwc, pwc, lm, h, t, cam, w->ob_z + 2 * k, w->fx, w->fy, w->cx, w->cy, w->B, e, &q2);
            if (q2 <= 1e-9) continue;
            double isg = w->ob_isig[k];
            double en2 = 0.0;
            for (int i = 0; i < nd; ++i) { e[i] *= isg; en2 += e[i] * e[i]; }
            ob_chi2[k] = en2;
            double en = sqrt(en2), wt, c;
            huber(en, w->huber_k, &wt, &c);
            cost += c;
            double Jl[2][3], Jt[2][6], Jh[2][6];
            obs_jacobians(Rwb, Rwc, pwc, Rcb, Px, lm, h, t, cam, w->fx, w->fy, w->B, Jl, Jt, Jh);
            for (int i = 0; i < nd; ++i) {
                for (int j = 0; j < 3; ++j) Jl[i][j] *= isg;
                for (int j = 0; j < 6; ++j) { Jt[i][j] *= isg; Jh[i][j] *= isg; }
            }
            ++nobs;
            for (int i = 0; i < 3; ++i) {
                for (int j = 0; j < 3; ++j) {
                    double acc = 0.0;
                    for (int r = 0; r < nd; ++r) acc += Jl[r][i] * Jl[r][j];
                    Hll[i * 3 + j] += wt * acc;
                }
                double acc = 0.0;
                for (int r = 0; r < nd; ++r) acc += Jl[r][i] * e[r];
                bl[i] += wt * acc;
            }
            if (t == h) continue;
            touched[t] = 1;
            touched[h] = 1;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 6; ++j) {
                    double at = 0.0, ah = 0.0;
                    for (int r = 0; r < nd; ++r) { at += Jl[r][i] * Jt[r][j]; ah += Jl[r][i] * Jh[r][j]; }
                    Hl[t * 18 + i * 6 + j] += wt * at;
                    Hl[h * 18 + i * 6 + j] += wt * ah;
                }
            for (int i = 0; i < 6; ++i) {
                double bt = 0.0, bh = 0.0;
                for (int r = 0; r < nd; ++r) { bt += Jt[r][i] * e[r]; bh += Jh[r][i] * e[r]; }
                bvec[6 * t + i] += wt * bt;
                bvec[6 * h + i] += wt * bh;
                for (int j = 0; j < 6; ++j) {
                    double tt = 0.0, hh = 0.0, th = 0.0;
                    for (int r = 0; r < nd; ++r) {
                        tt += Jt[r][i] * Jt[r][j];
                        hh += Jh[r][i] * Jh[r][j];
                        th += Jt[r][i] * Jh[r][j];
                    }
                    H[(6 * t + i) * n + 6 * t + j] += wt * tt;
                    H[(6 * h + i) * n + 6 * h + j] += wt * hh;
                    H[(6 * t + i) * n + 6 * h + j] += wt * th;
                    H[(6 * h + j) * n + 6 * t + i] += wt * th;
                }
            }
        }
        if (w->rho_isig[l] > 0.0) {
            double r0 = (lm[2] - w->rho_meas[l]) * w->rho_isig[l], wt, c;
            huber(fabs(r0), w->huber_k, &wt, &c);
            cost += c;
            Hll[8] += wt * w->rho_isig[l] * w->rho_isig[l];
            bl[2] += wt * w->rho_isig[l] * r0;
        }
        for (int i = 0; i < 3; ++i) Hll[i * 4] += lam * Hll[i * 4] + 1e-12;
        double det = Hll[0] * (Hll[4] * Hll[8] - Hll[5] * Hll[7]) - Hll[1] * (Hll[3] * Hll[8] - Hll[5] * Hll[6])
                     + Hll[2] * (Hll[3] * Hll[7] - Hll[4] * Hll[6]);
        double tr = Hll[0] + Hll[4] + Hll[8];
        if (nobs == 0 || !(det > 1e-18 * tr * tr * tr) || !isfinite(det)) continue;
        double idet = 1.0 / det;
        double* Hi = Hll_inv + 9 * l;
        Hi[0] = (Hll[4] * Hll[8] - Hll[5] * Hll[7]) * idet;
        Hi[1] = (Hll[2] * Hll[7] - Hll[1] * Hll[8]) * idet;
        Hi[2] = (Hll[1] * Hll[5] - Hll[2] * Hll[4]) * idet;
        Hi[3] = (Hll[5] * Hll[6] - Hll[3] * Hll[8]) * idet;
        Hi[4] = (Hll[0] * Hll[8] - Hll[2] * Hll[6]) * idet;
        Hi[5] = (Hll[2] * Hll[3] - Hll[0] * Hll[5]) * idet;
        Hi[6] = (Hll[3] * Hll[7] - Hll[4] * Hll[6]) * idet;
        Hi[7] = (Hll[1] * Hll[6] - Hll[0] * Hll[7]) * idet;
        Hi[8] = (Hll[0] * Hll[4] - Hll[1] * Hll[3]) * idet;
        lm_ok[l] = 1;
        for (int i = 0; i < 3; ++i) bl_out[3 * l + i] = bl[i];
        double HiB[3], T1[18];
        for (int i = 0; i < 3; ++i) HiB[i] = Hi[i * 3] * bl[0] + Hi[i * 3 + 1] * bl[1] + Hi[i * 3 + 2] * bl[2];
        for (int s1 = 0; s1 < P; ++s1) {
            if (!touched[s1]) continue;
            const double* A1 = Hl + s1 * 18;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 6; ++j)
                    T1[i * 6 + j] = Hi[i * 3] * A1[0 * 6 + j] + Hi[i * 3 + 1] * A1[1 * 6 + j] + Hi[i * 3 + 2] * A1[2 * 6 + j];
            for (int i = 0; i < 6; ++i) {
                double acc = 0.0;
                for (int r = 0; r < 3; ++r) acc += A1[r * 6 + i] * HiB[r];
                bvec[6 * s1 + i] -= acc;
            }
            for (int s2 = 0; s2 < P; ++s2) {
                if (!touched[s2]) continue;
                const double* A2 = Hl + s2 * 18;
                for (int i = 0; i < 6; ++i)
                    for (int j = 0; j < 6; ++j) {
                        double acc = 0.0;
                        for (int r = 0; r < 3; ++r) acc += A2[r * 6 + i] * T1[r * 6 + j];
                        H[(6 * s2 + i) * n + 6 * s1 + j] -= acc;
                    }
            }
        }
    }
    free(Rwc); free(pwc); free(touched);
    return cost;
}

double xo_ba_visual_cost(const XoWindow* w, const double* Rwb, const double* pwb, const double* lmp)
{
    const int P = w->P;
    double* Rwc = (double*)malloc(sizeof(double) * 9 * P);
    double* pwc = (double*)malloc(sizeof(double) * 3 * P);
    cam_poses(P, Rwb, pwb, w->Rbc, w->pbc, Rwc, pwc);
    double cost = 0.0;
    for (int l = 0; l < w->L; ++l) {
        if (!w->lm_mask[l]) continue;
        int h = (int)w->lm_host[l];
        for (int64_t k = w->ob_start[l]; k < w->ob_start[l + 1]; ++k) {
            if (!w->ob_valid[k]) continue;
            double e[2] = {0, 0}, q2;
            int nd = obs_residual(Rwc, pwc, lmp + 3 * l, h, (int)w->ob_pose[k], (int)w->ob_cam[k], w->ob_z + 2 * k,
                                  w->fx, w->fy, w->cx, w->cy, w->B, e, &q2);
            if (q2 <= 1e-9) { cost += 1e6; continue; }
            double en2 = 0.0;
            for (int i = 0; i < nd; ++i) { double t = e[i] * w->ob_isig[k]; en2 += t * t; }
            double wt, c;
            huber(sqrt(en2), w->huber_k, &wt, &c);
            cost += c;
        }
        if (w->rho_isig[l] > 0.0) {
            double r0 = (lmp[3 * l + 2] - w->rho_meas[l]) * w->rho_isig[l], wt, c;
            huber(fabs(r0), w->huber_k, &wt, &c);
            cost += c;
        }
    }
    free(Rwc); free(pwc);
    return cost;
}

void xo_ba_back_substitute(int L, int P, const double* dp, const double* Hll_inv, const double* bl, const double* Hlp,
                           const uint8_t* lm_ok, double* dl)
{
    for (int l = 0; l < L; ++l) {
        for (int i = 0; i < 3; ++i) dl[3 * l + i] = 0.0;
        if (!lm_ok[l]) continue;
        double v[3] = {bl[3 * l], bl[3 * l + 1], bl[3 * l + 2]};
        for (int s = 0; s < P; ++s)
            for (int i = 0; i < 3; ++i) {
                double acc = 0.0;
                for (int j = 0; j < 6; ++j) acc += Hlp[((size_t)l * P + s) * 18 + i * 6 + j] * dp[6 * s + j];
                v[i] += acc;
            }
        for (int i = 0; i < 3; ++i) {
            double acc = 0.0;
            for (int j = 0; j < 3; ++j) acc += Hll_inv[9 * l + i * 3 + j] * v[j];
            dl[3 * l + i] = -acc;
        }
    }
}

void xo_so3_exp(const double* w, double* R)
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

void xo_ba_apply_update(int P, int L, const double* Rwb, const double* pwb, const double* lmp, const double* dp,
                        const double* dl, const uint8_t* lm_ok, double* Rwb_out, double* pwb_out, double* lmp_out)
{
    for (int s = 0; s < P; ++s) {
        double Rexp[9];
        xo_so3_exp(dp + 6 * s, Rexp);
        mm3(Rwb + 9 * s, Rexp, Rwb_out + 9 * s);
        for (int i = 0; i < 3; ++i) pwb_out[3 * s + i] = pwb[3 * s + i] + dp[6 * s + 3 + i];
    }
    for (int l = 0; l < L; ++l) {
        for (int i = 0; i < 3; ++i) lmp_out[3 * l + i] = lmp[3 * l + i];
        if (lm_ok[l]) {
            double r = lmp[3 * l + 2] + dl[3 * l + 2];
            if (r > 1e-9 && isfinite(r)) {
                lmp_out[3 * l] = lmp[3 * l] + dl[3 * l];
                lmp_out[3 * l + 1] = lmp[3 * l + 1] + dl[3 * l + 1];
                lmp_out[3 * l + 2] = r;
            }
        }
    }
}

/* in-place lower Cholesky of a (n x n, row-major); -> 0 ok, -1 not positive definite */
int xo_cholesky(double* a, int n)
{
    for (int j = 0; j < n; ++j) {
        double d = a[j * n + j];
        for (int k = 0; k < j; ++k) d -= a[j * n + k] * a[j * n + k];
        if (!(d > 0.0)) return -1;
        d = sqrt(d);
        a[j * n + j] = d;
        for (int i = j + 1; i < n; ++i) {
            double s = a[i * n + j];
            for (int k = 0; k < j; ++k) s -= a[i * n + k] * a[j * n + k];
            a[i * n + j] = s / d;
        }
    }
    return 0;
}

/* solve L L^T x = b in place */
void xo_chol_solve(const double* Lc, int n, double* x)
{
    for (int i = 0; i < n; ++i) {
        double s = x[i];
        for (int k = 0; k < i; ++k) s -= Lc[i * n + k] * x[k];
        x[i] = s / Lc[i * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = x[i];
        for (int k = i + 1; k < n; ++k) s -= Lc[k * n + i] * x[k];
        x[i] = s / Lc[i * n + i];
    }
}

/* The reduced step of one linearisation: build, hold, damp, Cholesky, solve -> dx (6P) = -(H + D)^-1 b.
   -> cost at the linearisation point; *ok = 0 when the damped system is not positive definite. */
double xo_ba_step(const XoWindow* w, double lam, double* dx, double* Hll_inv, double* bl, double* Hlp, uint8_t* lm_ok,
                  int* ok)
{
    const int P = w->P, n = 6 * P;
    double* H = (double*)malloc(sizeof(double) * n * n);
    double* b = (double*)malloc(sizeof(double) * n);
    double* chi = (double*)malloc(sizeof(double) * (w->M > 0 ? w->M : 1));
    double c = xo_ba_build_system(w, w->Rwb, w->pwb, w->lmp, lam, H, b, Hll_inv, bl, Hlp, lm_ok, chi);
    if (w->hold >= 0 && w->hold < P) {
        int f0 = 6 * w->hold;
        for (int i = f0; i < f0 + 6; ++i) {
            for (int j = 0; j < n; ++j) { H[i * n + j] = 0.0; H[j * n + i] = 0.0; }
            H[i * n + i] = 1.0;
            b[i] = 0.0;
        }
    }
    for (int i = 0; i < n; ++i) H[i * n + i] += lam * H[i * n + i] + 1e-9;
    *ok = xo_cholesky(H, n) == 0;
    if (*ok) {
        for (int i = 0; i < n; ++i) dx[i] = b[i];
        xo_chol_solve(H, n, dx);
        for (int i = 0; i < n; ++i) dx[i] = -dx[i];
    }
    free(H); free(b); free(chi);
    return c;
}

/* window.solve's fixed-iteration LM (purely visual).  Updates Rwb / pwb / lmp in place.  out[0..3] = cost0, cost,
   accepted, lam; dx_first (6P, optional) = the first iteration's pose step. */
void xo_ba_solve(XoWindow* w, int iters, double lam0, double* out, double* dx_first)
{
    const int P = w->P, L = w->L, n = 6 * P;
    double* dx = (double*)malloc(sizeof(double) * n);
    double* Hll_inv = (double*)malloc(sizeof(double) * 9 * (L > 0 ? L : 1));
    double* bl = (double*)malloc(sizeof(double) * 3 * (L > 0 ? L : 1));
    double* Hlp = (double*)malloc(sizeof(double) * 18 * (size_t)P * (L > 0 ? L : 1));
    uint8_t* lm_ok = (uint8_t*)malloc(L > 0 ? L : 1);
    double* dl = (double*)malloc(sizeof(double) * 3 * (L > 0 ? L : 1));
    double* R2 = (double*)malloc(sizeof(double) * 9 * P);
    double* p2 = (double*)malloc(sizeof(double) * 3 * P);
    double* l2 = (double*)malloc(sizeof(double) * 3 * (L > 0 ? L : 1));
    double lam = lam0, cost0 = NAN, cur = NAN;
    int accepted = 0;
    for (int it = 0; it < iters; ++it) {
        int ok;
        double c_tot = xo_ba_step(w, lam, dx, Hll_inv, bl, Hlp, lm_ok, &ok);
        if (it == 0) { cost0 = c_tot; if (dx_first && ok) memcpy(dx_first, dx, sizeof(double) * n); }
        cur = c_tot;
        if (!ok) { lam *= 10.0; continue; }
        xo_ba_back_substitute(L, P, dx, Hll_inv, bl, Hlp, lm_ok, dl);
        xo_ba_apply_update(P, L, w->Rwb, w->pwb, w->lmp, dx, dl, lm_ok, R2, p2, l2);
        double c_new = xo_ba_visual_cost(w, R2, p2, l2);
        if (c_new < c_tot) {
            memcpy(w->Rwb, R2, sizeof(double) * 9 * P);
            memcpy(w->pwb, p2, sizeof(double) * 3 * P);
            memcpy(w->lmp, l2, sizeof(double) * 3 * L);
            lam = lam / 10.0 > 1e-12 ? lam / 10.0 : 1e-12;
            ++accepted;
            cur = c_new;
        } else {
            lam *= 10.0;
        }
    }
    out[0] = cost0; out[1] = cur; out[2] = accepted; out[3] = lam;
    free(dx); free(Hll_inv); free(bl); free(Hlp); free(lm_ok); free(dl); free(R2); free(p2); free(l2);
}

void xo_ba_solve_batch(XoWindow* ws, int nw, int iters, double lam0, int nthreads, double* out)
{
    #pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
    for (int i = 0; i < nw; ++i) xo_ba_solve(&ws[i], iters, lam0, out + 4 * i, NULL);
}

/* ============================================ pose-free landmarks ============================================ */
/* window._pf_block_fast (window.py:550-680): the host left observation and the inverse-depth prior of one pose-free
   landmark, damped by lam, its 3x3 inverse into Hi and the gradient into bl.  -> lm_ok. */
static int pf_block(const double* Rwc, const double* pwc, const double* RcR, int h, double a, double b, double rho,
                    double z0, double z1, double isg, double ris, double rmeas, double fx, double fy, double cx,
                    double cy, double huber_k, double lam, double* Hll, double* bl, double* Hi)
{
    const double* R = Rwc + 9 * (size_t)h;
    const double* p = pwc + 3 * (size_t)h;
    const double d0 = p[0] - p[0], d1 = p[1] - p[1], d2 = p[2] - p[2];
    const double Y0 = R[0] * a + R[1] * b + R[2] + rho * d0;
    const double Y1 = R[3] * a + R[4] * b + R[5] + rho * d1;
    const double Y2 = R[6] * a + R[7] * b + R[8] + rho * d2;
    const double q0 = R[0] * Y0 + R[3] * Y1 + R[6] * Y2;
    const double q1 = R[1] * Y0 + R[4] * Y1 + R[7] * Y2;
    const double q2 = R[2] * Y0 + R[5] * Y1 + R[8] * Y2;
    for (int i = 0; i < 9; ++i) Hll[i] = 0.0;
    for (int i = 0; i < 3; ++i) bl[i] = 0.0;
    int nobs = 0;
    if (q2 > 1e-9) {
        double e0 = fx * q0 / q2 + cx - z0, e1 = fy * q1 / q2 + cy - z1, en2 = 0.0;
        e0 *= isg;
        en2 += e0 * e0;
        e1 *= isg;
        en2 += e1 * e1;
        const double en = sqrt(en2);
        const double w = en <= huber_k ? 1.0 : huber_k / en;
        const double iq = 1.0 / q2;
        const double D[6] = {fx * iq, 0.0, -fx * q0 * iq * iq, 0.0, fy * iq, -fy * q1 * iq * iq};
        const double r0 = R[0] * d0 + R[3] * d1 + R[6] * d2;
        const double r1 = R[1] * d0 + R[4] * d1 + R[7] * d2;
        const double r2 = R[2] * d0 + R[5] * d1 + R[8] * d2;
        double J[2][3];
        for (int r = 0; r < 2; ++r) {
            J[r][0] = D[3 * r] * RcR[0] + D[3 * r + 1] * RcR[3] + D[3 * r + 2] * RcR[6];
            J[r][1] = D[3 * r] * RcR[1] + D[3 * r + 1] * RcR[4] + D[3 * r + 2] * RcR[7];
            J[r][2] = D[3 * r] * r0 + D[3 * r + 1] * r1 + D[3 * r + 2] * r2;
        }
        for (int r = 0; r < 2; ++r)
            for (int j = 0; j < 3; ++j) J[r][j] *= isg;
        nobs += 1;
        const double e[2] = {e0, e1};
        for (int i = 0; i < 3; ++i) {
            for (int j = 0; j < 3; ++j) {
                double acc = 0.0;
                acc += J[0][i] * J[0][j];
                acc += J[1][i] * J[1][j];
                Hll[3 * i + j] += w * acc;
            }
            double acc = 0.0;
            acc += J[0][i] * e[0];
            acc += J[1][i] * e[1];
            bl[i] += w * acc;
        }
    }
    if (ris > 0.0) {
        const double rr = (rho - rmeas) * ris, ar = fabs(rr);
        const double wp = ar <= huber_k ? 1.0 : huber_k / ar;
        Hll[8] += wp * ris * ris;
        bl[2] += wp * ris * rr;
    }
    for (int i = 0; i < 3; ++i) Hll[4 * i] += lam * Hll[4 * i] + 1e-12;
    const double det = Hll[0] * (Hll[4] * Hll[8] - Hll[5] * Hll[7]) - Hll[1] * (Hll[3] * Hll[8] - Hll[5] * Hll[6])
                       + Hll[2] * (Hll[3] * Hll[7] - Hll[4] * Hll[6]);
    const double tr = Hll[0] + Hll[4] + Hll[8];
    if (nobs == 0 || !(det > 1e-18 * tr * tr * tr) || !isfinite(det)) return 0;
    const double idet = 1.0 / det;
    Hi[0] = (Hll[4] * Hll[8] - Hll[5] * Hll[7]) * idet;
    Hi[1] = (Hll[2] * Hll[7] - Hll[1] * Hll[8]) * idet;
    Hi[2] = (Hll[1] * Hll[5] - Hll[2] * Hll[4]) * idet;
    Hi[3] = (Hll[5] * Hll[6] - Hll[3] * Hll[8]) * idet;
    Hi[4] = (Hll[0] * Hll[8] - Hll[2] * Hll[6]) * idet;
    Hi[5] = (Hll[2] * Hll[3] - Hll[0] * Hll[5]) * idet;
    Hi[6] = (Hll[3] * Hll[7] - Hll[4] * Hll[6]) * idet;
    Hi[7] = (Hll[1] * Hll[6] - Hll[0] * Hll[7]) * idet;
    Hi[8] = (Hll[0] * Hll[4] - Hll[1] * Hll[3]) * idet;
    return 1;
}

/* window.posefree_cost (window.py:683-710): the host left observation (q2 <= 1e-9: nothing, or 1e6 when `behind`)
   and the inverse-depth prior of every pose-free landmark, added in landmark order. */
double xo_ba_posefree_cost(int P, const double* Rwb, const double* pwb, const double* Rbc, const double* pbc, int n,
                           const double* lmp, const int64_t* host, const double* rmeas, const double* ris,
                           const double* z, double isg, double fx, double fy, double cx, double cy, double B,
                           double huber_k, int behind)
{
    double* Rwc = (double*)malloc(sizeof(double) * 9 * (size_t)(P > 0 ? P : 1));
    double* pwc = (double*)malloc(sizeof(double) * 3 * (size_t)(P > 0 ? P : 1));
    cam_poses(P, Rwb, pwb, Rbc, pbc, Rwc, pwc);
    double cost = 0.0, e[2], q2, w, c;
    for (int l = 0; l < n; ++l) {
        const int h = (int)host[l];
        obs_residual(Rwc, pwc, lmp + 3 * (size_t)l, h, h, 0, z + 2 * (size_t)l, fx, fy, cx, cy, B, e, &q2);
        if (q2 <= 1e-9) {
            if (behind) cost += 1e6;
        } else {
            double en2 = 0.0;
            const double e0 = e[0] * isg;
            en2 += e0 * e0;
            const double e1 = e[1] * isg;
            en2 += e1 * e1;
            huber(sqrt(en2), huber_k, &w, &c);
            cost += c;
        }
        if (ris[l] > 0.0) {
            const double r0 = (lmp[3 * l + 2] - rmeas[l]) * ris[l];
            huber(fabs(r0), huber_k, &w, &c);
            cost += c;
        }
    }
    free(Rwc);
    free(pwc);
    return cost;
}

/* window.posefree_step (window.py:713-765): every pose-free landmark's damped 3x3 step at lam -> lmp_out (the trial
   state, the input where the step is refused), Hinv_out (written where ok) and ok_out. */
void xo_ba_posefree_step(int P, const double* Rwb, const double* pwb, const double* Rbc, const double* pbc, int n,
                         const double* lmp_in, const int64_t* host, const double* rmeas, const double* ris,
                         const double* z, double isg, double fx, double fy, double cx, double cy, double huber_k,
                         double lam, double* lmp_out, double* Hinv_out, uint8_t* ok_out)
{
    double* Rwc = (double*)malloc(sizeof(double) * 9 * (size_t)(P > 0 ? P : 1));
    double* pwc = (double*)malloc(sizeof(double) * 3 * (size_t)(P > 0 ? P : 1));
    double* RcR = (double*)malloc(sizeof(double) * 9 * (size_t)(P > 0 ? P : 1));
    cam_poses(P, Rwb, pwb, Rbc, pbc, Rwc, pwc);
    for (int s = 0; s < P; ++s) mtm3(Rwc + 9 * s, Rwc + 9 * s, RcR + 9 * s);
    double Hll[9], bl[3], Hi[9];
    for (int l = 0; l < n; ++l) {
        const int h = (int)host[l];
        const double* li = lmp_in + 3 * (size_t)l;
        for (int i = 0; i < 3; ++i) lmp_out[3 * l + i] = li[i];
        const int ok = pf_block(Rwc, pwc, RcR + 9 * h, h, li[0], li[1], li[2], z[2 * l], z[2 * l + 1], isg, ris[l],
                                rmeas[l], fx, fy, cx, cy, huber_k, lam, Hll, bl, Hi);
        ok_out[l] = (uint8_t)ok;
        if (!ok) continue;
        for (int i = 0; i < 9; ++i) Hinv_out[9 * (size_t)l + i] = Hi[i];
        double v[3], d[3];
        for (int i = 0; i < 3; ++i) v[i] = bl[i] + 0.0;
        for (int i = 0; i < 3; ++i) {
            double acc = 0.0;
            acc += Hi[3 * i] * v[0];
            acc += Hi[3 * i + 1] * v[1];
            acc += Hi[3 * i + 2] * v[2];
            d[i] = -acc;
        }
        const double r = li[2] + d[2];
        if (r > 1e-9 && isfinite(r)) {
            lmp_out[3 * l] = li[0] + d[0];
            lmp_out[3 * l + 1] = li[1] + d[1];
            lmp_out[3 * l + 2] = r;
        }
    }
    free(RcR);
    free(pwc);
    free(Rwc);
}
