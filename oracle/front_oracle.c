/*
 * front_oracle.c -- CPU ORACLE of the xclean stereo frontend (test infrastructure only).
 *
 * This file is the checker, never the product: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * load it.  It restates, in plain C, the reference's CPU algorithms for the per-frame hot path:
 *
 *   response      cv2.cornerMinEigenVal(gray, 3, 3) as called in src/xclean/stages/features.py:299, with the SIMD /
 *                 scalar split of OpenCV's separable Sobel as a parameter (the reference calibrates it at start-up,
 *                 src/xclean/front/gpu_front.py:1423-1453); box filter = OpenCV ColumnSum running double sums.
 *   noise floor   features.noise_floor_8u (features.py:57-73): Immerkaer |Laplacian| summed in numpy's float32
 *                 pairwise order (blocks of 128, 8 accumulators), floor = Q (K s)^2 / 255^2.
 *   detect        Frontend._response cell scope (features.py:288-315) + Frontend._detect greedy (features.py:337-403)
 *                 + Frontend._subpix (features.py:318-335), as front/detect.Detector.__call__ (detect.py:60-75) runs
 *                 them with no existing keypoints.
 *   blur / ORB    Frontend.describe (features.py:405-421): reflect-101 pad 32, cv2 ORB (nlevels 1, no orientation),
 *                 whose internal 7x7 sigma-2 Gaussian is OpenCV's float separable filter on a sub-matrix.
 *   stereo        front/stereo1d.stereo_points_band (stereo1d.py:335-472) with _patch_stats / _zncc / _bil / _lk_v
 *                 (stereo1d.py:40-130, :272-332) and shift_rows (:478-489); the patch half-size HALF is a parameter
 *                 (the reference fixes HALF = 5, src/xclean/stereo/epipolar.py:35).  The 3x3 solve / inverse follow
 *                 the LAPACK calls numba makes (np.linalg.solve / inv -> OpenBLAS getf2/getrs, trti2 + dgetri),
 *                 the arithmetic the reference's device kernel reproduces (gpu_front.py:607-704).
 *   hamming       front/mapmatch_fast._bf_mutual (mapmatch_fast.py:46-90) = Frontend.match_desc (features.py:564-595).
 *   predict       vio/window.predict_projection (window.py:1032-1144), the map matcher's predicted pixels and
 *                 innovation covariances.
 *   mapmatch      front/mapmatch.MapMatcher.match (mapmatch.py:148-169) with its numba _gated (mapmatch.py:49-131) and
 *                 grid (:141-146), = front/mapmatch_fast.MapMatcher.match (mapmatch_fast.py:113-184).
 *
 * Build: gcc -O2 -ffp-contract=off -fno-fast-math -fopenmp -shared -fPIC (see oracle/build.py).  Every floating-point
 * step is written out; fma() is used exactly where the restated library uses a fused multiply-add.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned char u8;
typedef int64_t i64;
typedef uint64_t u64;

#define REFL(i, n) ((i) < 0 ? -(i) : ((i) >= (n) ? 2 * (n) - 2 - (i) : (i)))

/* ============================================ response (cornerMinEigenVal) ============================================ */
/* OpenCV cornerEigenValsVecs for CV_8U, aperture 3, block 3: Sobel scale 1/(4*3*255); the smoothing tap row filter uses a
   fused multiply-add chain from zero for x < dy_vend (SIMD body) and a plain sum of products in its scalar tail; the
   derivative column filter fuses for x < dx_vend.  cov products in float32, 3x3 box sum in double (row sums, then a
   running column sum per column and channel), min eigenvalue in float32. */
static void sobel_at(const u8* I, int H, int W, int y, int x, float ks, float k2s, int dy_vend, int dx_vend,
                     float* dxo, float* dyo)
{
    int xm = REFL(x - 1, W), xp = REFL(x + 1, W);
    float rx[3], ry[3];
    for (int j = 0; j < 3; ++j) {
        int yy = REFL(y - 1 + j, H);
        const u8* row = I + (size_t)yy * W;
        float a = (float)row[xm], b = (float)row[x], c = (float)row[xp];
        rx[j] = c - a;
        if (x < dy_vend) {
            float s = a * ks;
            s = fmaf(b, k2s, s);
            s = fmaf(c, ks, s);
            ry[j] = s;
        } else {
            float s = ks * a;
            s = s + k2s * b;
            s = s + ks * c;
            ry[j] = s;
        }
    }
    float t = rx[0] + rx[2];
    if (x < dx_vend) *dxo = fmaf(t, ks, rx[1] * k2s);
    else *dxo = t * ks + rx[1] * k2s;
    *dyo = ry[2] - ry[0];
}

void xo_response(const u8* I, int H, int W, int dy_vend, int dx_vend, float* R)
{
    const float ks = (float)(1.0 / (4 * 3 * 255.0));
    const float k2s = (float)(2.0 * (1.0 / (4 * 3 * 255.0)));
    size_t n = (size_t)H * W;
    float* P = (float*)malloc(sizeof(float) * 3 * n);      /* products dx*dx, dx*dy, dy*dy */
    double* RS = (double*)malloc(sizeof(double) * 3 * n);  /* row sums */
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            float dx, dy;
            sobel_at(I, H, W, y, x, ks, k2s, dy_vend, dx_vend, &dx, &dy);
            size_t o = (size_t)y * W + x;
            P[o] = dx * dx; P[n + o] = dx * dy; P[2 * n + o] = dy * dy;
        }
    for (int ch = 0; ch < 3; ++ch)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                const float* p = P + ch * n + (size_t)y * W;
                int xm = REFL(x - 1, W), xp = REFL(x + 1, W);
                RS[ch * n + (size_t)y * W + x] = ((double)p[xm] + (double)p[x]) + (double)p[xp];
            }
    float* cov = (float*)malloc(sizeof(float) * 3 * n);
    for (int ch = 0; ch < 3; ++ch)
        for (int x = 0; x < W; ++x) {
            const double* col = RS + ch * n + x;
            double a = col[(size_t)REFL(-1, H) * W], b = col[0];
            double S = (0.0 + a) + b;
            for (int y = 0; y < H; ++y) {
                double c = col[(size_t)REFL(y + 1, H) * W];
                double s0 = S + c;
                cov[ch * n + (size_t)y * W + x] = (float)s0;
                S = s0 - a;
                a = b; b = c;
            }
        }
    for (size_t i = 0; i < n; ++i) {
        float a = cov[i] * 0.5f, b = cov[n + i], c = cov[2 * n + i] * 0.5f;
        float t = a - c;
        float v = t * t + b * b;
        R[i] = (a + c) - sqrtf(v);
    }
    free(P); free(RS); free(cov);
}

/* ============================================== noise floor (numpy pairwise) ============================================== */
static inline float lap_abs_at(const u8* I, int W, i64 k)
{
    int Wi = W - 2;
    int y = 1 + (int)(k / Wi), x = 1 + (int)(k % Wi);
    const u8* r0 = I + (size_t)(y - 1) * W + x;
    const u8* r1 = r0 + W;
    const u8* r2 = r1 + W;
    int v = (int)r0[-1] - 2 * (int)r0[0] + (int)r0[1] - 2 * (int)r1[-1] + 4 * (int)r1[0] - 2 * (int)r1[1] + (int)r2[-1]
            - 2 * (int)r2[0] + (int)r2[1];
    return (float)(v < 0 ? -v : v);
}

/* numpy's pairwise_sum for float32 (n <= 128: 8 accumulators; else split at n/2 rounded down to a multiple of 8) */
static float pairwise(const u8* I, int W, i64 st, i64 n)
{
    if (n < 8) {
        float res = -0.0f;
        for (i64 i = 0; i < n; ++i) res = res + lap_abs_at(I, W, st + i);
        return res;
    }
    if (n <= 128) {
        float r[8];
        for (int j = 0; j < 8; ++j) r[j] = lap_abs_at(I, W, st + j);
        i64 i = 8, lim = n - (n % 8);
        for (; i < lim; i += 8)
            for (int j = 0; j < 8; ++j) r[j] = r[j] + lap_abs_at(I, W, st + i + j);
        float res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
        for (; i < n; ++i) res = res + lap_abs_at(I, W, st + i);
        return res;
    }
    i64 n2 = n / 2;
    n2 -= n2 % 8;
    float a = pairwise(I, W, st, n2);
    float b = pairwise(I, W, st + n2, n - n2);
    return a + b;
}

/* -> floor (double); *floor_f = float32 of it (the candidate test compares float32 R with a weakly typed Python float,
   i.e. with float32(floor)) */
double xo_noise_floor(const u8* I, int H, int W, double Q, float* floor_f)
{
    float s = pairwise(I, W, 0, (i64)(H - 2) * (W - 2));
    double K = sqrt(M_PI / 2.0) / (6.0 * (W - 2) * (H - 2));
    double sn = K * (double)s;
    double fl = ((Q * sn) * sn) / (255.0 * 255.0);
    if (floor_f) *floor_f = (float)fl;
    return fl;
}

/* ====================================================== detection ====================================================== */
/* numpy floor_divide on float64 (npy_divmod) */
static double npy_floordiv(double a, double b)
{
    double mod = fmod(a, b);
    double div = (a - mod) / b;
    if (mod != 0.0) {
        if ((b < 0) != (mod < 0)) { mod += b; div -= 1.0; }
    }
    double fd;
    if (div != 0.0) {
        fd = floor(div);
        if (div - fd > 0.5) fd += 1.0;
    } else {
        fd = copysign(0.0, a / b);
    }
    return fd;
}

static inline uint32_t ord_f(float v)
{
    uint32_t u;
    memcpy(&u, &v, 4);
    if (u == 0x80000000u) u = 0u;
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

static int cmp_desc_u64(const void* a, const void* b)
{
    u64 x = *(const u64*)a, y = *(const u64*)b;
    return x < y ? 1 : (x > y ? -1 : 0);
}

double xo_cell(int W, int H, int n) { double s = sqrt((double)W * H / (double)(n > 1 ? n : 1)); return s > 4.0 ? s : 4.0; }
double xo_min_dist(int W, int H, int n)
{
    double r = sqrt((double)W * H / (2.0 * sqrt(3.0) * (double)(n > 1 ? n : 1)));
    return r > 2.0 ? r : 2.0;
}

/* Frontend._response (cell scope) + _detect + _subpix for one frame with no existing keypoints.
   R: the response; floor_f: float32 floor; budget n = n_want.  kp_out (cap x 2 float32).  -> count.
   *n_cand receives the candidate count (diagnostics). */
int xo_detect(const float* R, int H, int W, int budget, float floor_f, int cap, float* kp_out, int* n_cand)
{
    size_t npx = (size_t)H * W;
    int anypos = 0;
    for (size_t i = 0; i < npx; ++i)
        if (R[i] > 0.0f) { anypos = 1; break; }
    if (n_cand) *n_cand = 0;
    if (!anypos || budget <= 0) return 0;
    double s = xo_cell(W, H, budget);
    double r = xo_min_dist(W, H, budget);
    int c = (int)nearbyint(s);
    if (c < 4) c = 4;
    int gwc = (W + c - 1) / c, ghc = (H + c - 1) / c;
    float* cmax = (float*)malloc(sizeof(float) * (size_t)gwc * ghc);
    for (int gy = 0; gy < ghc; ++gy)
        for (int gx = 0; gx < gwc; ++gx) {
            float m = -INFINITY;
            int pad = 0;
            for (int y = gy * c; y < gy * c + c; ++y)
                for (int x = gx * c; x < gx * c + c; ++x) {
                    if (y < H && x < W) { float v = R[(size_t)y * W + x]; if (v > m) m = v; }
                    else pad = 1;
                }
            if (pad && m < 0.0f) m = 0.0f;
            cmax[gy * gwc + gx] = 0.01f * m;
        }
    const int b = 21 / 2 + 1;
    int ncx = (int)ceil(W / s);
    /* candidates with their 64-bit rank keys: response desc, y asc, x asc (np.lexsort((xs, ys, -resp))) */
    size_t capc = 1024, nc = 0;
    u64* key = (u64*)malloc(sizeof(u64) * capc);
    for (int y = b; y < H - b; ++y)
        for (int x = b; x < W - b; ++x) {
            const float* p = R + (size_t)y * W + x;
            float v = p[0];
            int ismax = 1;
            for (int dy = -1; dy <= 1 && ismax; ++dy)
                for (int dx = -1; dx <= 1; ++dx)
                    if (p[dy * W + dx] > v) { ismax = 0; break; }
            if (!ismax) continue;
            if (!(v >= cmax[(y / c) * gwc + x / c])) continue;
            if (!(v >= floor_f)) continue;
            if (nc == capc) { capc *= 2; key = (u64*)realloc(key, sizeof(u64) * capc); }
            key[nc++] = ((u64)ord_f(v) << 32) | ((u64)(0xFFFF - y) << 16) | (u64)(0xFFFF - x);
        }
    if (n_cand) *n_cand = (int)nc;
    qsort(key, nc, sizeof(u64), cmp_desc_u64);
    /* greedy: one pick per cell, none within r (strict <) of an earlier pick; hash grid of size r */
    int ncell = ncx * ((int)ceil(H / s) + 2);
    unsigned char* seen = (unsigned char*)calloc((size_t)ncell + 1, 1);
    int hgx = (int)floor((W - 1) / r) + 3, hgy = (int)floor((H - 1) / r) + 3;
    int* head = (int*)malloc(sizeof(int) * (size_t)hgx * hgy);
    for (int i = 0; i < hgx * hgy; ++i) head[i] = -1;
    int* nxt = (int*)malloc(sizeof(int) * (size_t)(budget + 1));
    int* px = (int*)malloc(sizeof(int) * (size_t)(budget + 1));
    int* py = (int*)malloc(sizeof(int) * (size_t)(budget + 1));
    int np_ = 0;
    double r2 = r * r;
    for (size_t t = 0; t < nc && np_ < budget; ++t) {
        int x = 0xFFFF - (int)(key[t] & 0xFFFF), y = 0xFFFF - (int)((key[t] >> 16) & 0xFFFF);
        int cyc = (int)npy_floordiv((double)y, s), cxc = (int)npy_floordiv((double)x, s);
        int cell = cyc * ncx + cxc;
        if (seen[cell]) continue;
        int hx = (int)floor(x / r), hy = (int)floor(y / r);
        int clash = 0;
        for (int ay = hy - 1; ay <= hy + 1 && !clash; ++ay) {
            if (ay < 0 || ay >= hgy) continue;
            for (int ax = hx - 1; ax <= hx + 1 && !clash; ++ax) {
                if (ax < 0 || ax >= hgx) continue;
                for (int q = head[ay * hgx + ax]; q >= 0; q = nxt[q]) {
                    i64 ddx = (i64)px[q] - x, ddy = (i64)py[q] - y;
                    if ((double)(ddx * ddx + ddy * ddy) < r2) { clash = 1; break; }
                }
            }
        }
        if (clash) continue;
        seen[cell] = 1;
        px[np_] = x; py[np_] = y;
        nxt[np_] = head[hy * hgx + hx];
        head[hy * hgx + hx] = np_;
        ++np_;
    }
    int cnt = np_ < cap ? np_ : cap;
    /* sub-pixel parabola in float64 (Frontend._subpix expression order), then float32 */
    for (int i = 0; i < cnt; ++i) {
        int x = px[i], y = py[i];
        double fx = x, fy = y;
        if (x > 0 && x < W - 1 && y > 0 && y < H - 1) {
            const float* q = R + (size_t)y * W + x;
            double cc = q[0], l = q[-1], rr = q[1], u = q[-W], d = q[W];
            double denx = (l - 2.0 * cc) + rr;
            double deny = (u - 2.0 * cc) + d;
            double dx = denx < 0.0 ? (0.5 * (l - rr)) / denx : 0.0;
            double dy = deny < 0.0 ? (0.5 * (u - d)) / deny : 0.0;
            dx = dx < -0.5 ? -0.5 : (dx > 0.5 ? 0.5 : dx);
            dy = dy < -0.5 ? -0.5 : (dy > 0.5 ? 0.5 : dy);
            fx += dx; fy += dy;
        }
        kp_out[2 * i] = (float)fx;
        kp_out[2 * i + 1] = (float)fy;
    }
    free(cmax); free(key); free(seen); free(head); free(nxt); free(px); free(py);
    return cnt;
}

/* ======================================================== ORB ======================================================== */
/* 7x7 Gaussian (cv2.getGaussianKernel(7, 2, CV_32F)) on the reflect-101 pad-32 image: row pass fused for x < vr (SIMD
   body), scalar tail otherwise; symmetric column pass fused for x < vc; round half to even, saturate to u8. */
void xo_blur(const u8* I, int H, int W, const float* kf, int vr, int vc, u8* out)
{
    int Hp = H + 64, Wp = W + 64;
    float* RB = (float*)malloc(sizeof(float) * (size_t)Hp * Wp);
    for (int y = 0; y < Hp; ++y) {
        const u8* row = I + (size_t)REFL(y - 32, H) * W;
        for (int x = 0; x < Wp; ++x) {
            float p[7];
            for (int k = 0; k < 7; ++k) { int xx = REFL(x - 3 + k, Wp); p[k] = (float)row[REFL(xx - 32, W)]; }
            float s;
            if (x < vr) { s = p[0] * kf[0]; for (int k = 1; k < 7; ++k) s = fmaf(p[k], kf[k], s); }
            else { s = kf[0] * p[0]; for (int k = 1; k < 7; ++k) s = s + kf[k] * p[k]; }
            RB[(size_t)y * Wp + x] = s;
        }
    }
    for (int y = 0; y < Hp; ++y)
        for (int x = 0; x < Wp; ++x) {
            float S0 = RB[(size_t)y * Wp + x], s;
            if (x < vc) {
                s = kf[3] * S0;
                for (int k = 1; k <= 3; ++k) {
                    float t = RB[(size_t)REFL(y + k, Hp) * Wp + x] + RB[(size_t)REFL(y - k, Hp) * Wp + x];
                    s = fmaf(kf[3 + k], t, s);
                }
            } else {
                s = kf[3] * S0 + 0.0f;
                for (int k = 1; k <= 3; ++k) {
                    float t = RB[(size_t)REFL(y + k, Hp) * Wp + x] + RB[(size_t)REFL(y - k, Hp) * Wp + x];
                    s = s + kf[3 + k] * t;
                }
            }
            float rv = nearbyintf(s);
            int v = (int)rv;
            out[(size_t)y * Wp + x] = (u8)(v < 0 ? 0 : (v > 255 ? 255 : v));
        }
    free(RB);
}

/* 256 tests (x1, y1, x2, y2) at the keypoint rounded half-to-even in float32 (cvRound of KeyPoint.pt = kp + 32) */
void xo_orb(const u8* B, int Wp, const float* kp, int n, const int8_t* pat, u8* desc)
{
    for (int i = 0; i < n; ++i) {
        int cx = (int)nearbyintf(kp[2 * i] + 32.0f), cy = (int)nearbyintf(kp[2 * i + 1] + 32.0f);
        const u8* c = B + (size_t)cy * Wp + cx;
        for (int by = 0; by < 32; ++by) {
            int v = 0;
            for (int bb = 0; bb < 8; ++bb) {
                const int8_t* q = pat + 4 * (8 * by + bb);
                int t0 = c[(int)q[1] * Wp + (int)q[0]], t1 = c[(int)q[3] * Wp + (int)q[2]];
                v |= (t0 < t1) << bb;
            }
            desc[32 * i + by] = (u8)v;
        }
    }
}

/* ======================================================= stereo ======================================================= */
/* shift_rows (stereo1d.py:478-489): rows resampled at y + dy in float32 (dy == 0: plain float copy) */
void xo_shift_rows(const u8* Rr, int H, int W, double dy, float* Rs)
{
    for (int y = 0; y < H; ++y) {
        if (dy == 0.0) {
            for (int x = 0; x < W; ++x) Rs[(size_t)y * W + x] = (float)Rr[(size_t)y * W + x];
            continue;
        }
        double yy = (double)y + dy;
        double y0d = floor(yy);
        float f = (float)(yy - y0d);
        i64 y0 = (i64)y0d;
        i64 ya = y0 < 0 ? 0 : (y0 > H - 1 ? H - 1 : y0);
        i64 yb = y0 + 1 < 0 ? 0 : (y0 + 1 > H - 1 ? H - 1 : y0 + 1);
        for (int x = 0; x < W; ++x) {
            float a = (float)Rr[(size_t)ya * W + x], b = (float)Rr[(size_t)yb * W + x];
            Rs[(size_t)y * W + x] = a + f * (b - a);
        }
    }
}

/* OpenBLAS getf2 (left-looking: per column the earlier interchanges, dot products accumulated from zero by fused
   multiply-adds and then subtracted, first-max pivot, row swap of the finished columns, scale by the reciprocal) */
void xo_getf2(double a[3][3], int piv[3])
{
    for (int j = 0; j < 3; ++j) {
        for (int i = 0; i < j; ++i) {
            int ip = piv[i];
            if (ip != i) { double t = a[i][j]; a[i][j] = a[ip][j]; a[ip][j] = t; }
        }
        for (int i = 1; i < j; ++i) {
            double s = 0.0;
            for (int k = 0; k < i; ++k) s = fma(a[i][k], a[k][j], s);
            a[i][j] = a[i][j] - s;
        }
        if (j > 0)
            for (int i = j; i < 3; ++i) {
                double s = 0.0;
                for (int k = 0; k < j; ++k) s = fma(a[i][k], a[k][j], s);
                a[i][j] = a[i][j] - s;
            }
        int jp = j;
        double mx = fabs(a[j][j]);
        for (int i = j + 1; i < 3; ++i)
            if (fabs(a[i][j]) > mx) { mx = fabs(a[i][j]); jp = i; }
        piv[j] = jp;
        double t = a[jp][j];
        if (t != 0.0) {
            t = 1.0 / t;
            if (jp != j)
                for (int k = 0; k <= j; ++k) { double u = a[j][k]; a[j][k] = a[jp][k]; a[jp][k] = u; }
            for (int i = j + 1; i < 3; ++i) a[i][j] = a[i][j] * t;
        }
    }
}

/* getrs: interchanges, unit-lower then upper triangular solves with fused axpy updates */
void xo_getrs(double a[3][3], const int piv[3], double y[3])
{
    for (int j = 0; j < 3; ++j) { int p = piv[j]; if (p != j) { double t = y[j]; y[j] = y[p]; y[p] = t; } }
    for (int j = 0; j < 3; ++j)
        for (int i = j + 1; i < 3; ++i) y[i] = fma(-y[j], a[i][j], y[i]);
    for (int j = 2; j >= 0; --j) {
        y[j] = y[j] / a[j][j];
        for (int i = 0; i < j; ++i) y[i] = fma(-y[j], a[i][j], y[i]);
    }
}

/* getri from the getf2 factors: trti2 (upper, non-unit: trmv as axpy-then-scale, scaled by -1/a_jj), then the
   unblocked dgetri column sweep (gemv accumulated from zero by fused multiply-adds, then subtracted), then the column
   interchanges in reverse order */
void xo_getri(double a[3][3], const int piv[3])
{
    for (int j = 0; j < 3; ++j) {
        double ajj = 1.0 / a[j][j];
        a[j][j] = ajj;
        double x[3];
        for (int i = 0; i < j; ++i) x[i] = a[i][j];
        for (int i = 0; i < j; ++i) {
            for (int q = 0; q < i; ++q) x[q] = fma(x[i], a[q][i], x[q]);
            x[i] = x[i] * a[i][i];
        }
        for (int i = 0; i < j; ++i) a[i][j] = x[i] * -ajj;
    }
    double work[3] = {0.0, 0.0, 0.0};
    for (int j = 2; j >= 0; --j) {
        for (int i = j + 1; i < 3; ++i) { work[i] = a[i][j]; a[i][j] = 0.0; }
        if (j < 2)
            for (int r = 0; r < 3; ++r) {
                double s = 0.0;
                for (int k = j + 1; k < 3; ++k) s = fma(a[r][k], work[k], s);
                a[r][j] = a[r][j] - s;
            }
    }
    for (int j = 1; j >= 0; --j) {
        int jp = piv[j];
        if (jp != j)
            for (int r = 0; r < 3; ++r) { double t = a[r][j]; a[r][j] = a[r][jp]; a[r][jp] = t; }
    }
}

/* solve + inverse of n row-major 3x3 systems (the LK solver self-check) */
void xo_lk_solve_inv(const double* As, const double* gs, int n, double* X, double* Inv)
{
    for (int k = 0; k < n; ++k) {
        double a[3][3], b[3][3];
        int piv[3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) a[i][j] = b[i][j] = As[9 * k + 3 * i + j];
        xo_getf2(a, piv);
        double y[3] = {gs[3 * k], gs[3 * k + 1], gs[3 * k + 2]};
        xo_getrs(a, piv, y);
        for (int i = 0; i < 3; ++i) X[3 * k + i] = y[i];
        int piv2[3];
        xo_getf2(b, piv2);
        xo_getri(b, piv2);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) Inv[9 * k + 3 * i + j] = b[i][j];
    }
}

typedef struct { int half, pw, npix; } Geo;

static void patch_stats_u8(const u8* img, int W, int u, int v, Geo g, double* m, double* sd)
{
    double s = 0.0, s2 = 0.0;
    for (int dy = -g.half; dy <= g.half; ++dy)
        for (int dx = -g.half; dx <= g.half; ++dx) {
            double x = (double)img[(size_t)(v + dy) * W + u + dx];
            s = s + x;
            s2 = s2 + x * x;
        }
    double mm = s / g.npix;
    double var = s2 / g.npix - mm * mm;
    *m = mm;
    *sd = sqrt(var > 0.0 ? var : 0.0);
}

/* float32 image: numba keeps float(float32) in float32, so x * x is a float32 product */
static void patch_stats_f(const float* img, int W, int u, int v, Geo g, double* m, double* sd)
{
    double s = 0.0, s2 = 0.0;
    for (int dy = -g.half; dy <= g.half; ++dy)
        for (int dx = -g.half; dx <= g.half; ++dx) {
            float x = img[(size_t)(v + dy) * W + u + dx];
            s = s + (double)x;
            s2 = s2 + (double)(x * x);
        }
    double mm = s / g.npix;
    double var = s2 / g.npix - mm * mm;
    *m = mm;
    *sd = sqrt(var > 0.0 ? var : 0.0);
}

static double zncc_f(const double* T, double tm, double ts, const float* img, int W, int x, int v, Geo g)
{
    double s = 0.0, s2 = 0.0, sx = 0.0;
    int k = 0;
    for (int dy = -g.half; dy <= g.half; ++dy)
        for (int dx = -g.half; dx <= g.half; ++dx) {
            float rf = img[(size_t)(v + dy) * W + x + dx];
            double r = (double)rf;
            s = s + r;
            s2 = s2 + (double)(rf * rf);
            sx = sx + r * (T[k] - tm);
            ++k;
        }
    double m = s / g.npix;
    double var = s2 / g.npix - m * m;
    double sd = sqrt(var > 0.0 ? var : 0.0);
    double den = (ts * sd) * g.npix;
    return den > 1e-6 ? sx / den : -2.0;
}

static double zncc_u8(const double* T, double tm, double ts, const u8* img, int W, int x, int v, Geo g)
{
    double s = 0.0, s2 = 0.0, sx = 0.0;
    int k = 0;
    for (int dy = -g.half; dy <= g.half; ++dy)
        for (int dx = -g.half; dx <= g.half; ++dx) {
            double r = (double)img[(size_t)(v + dy) * W + x + dx];
            s = s + r;
            s2 = s2 + r * r;
            sx = sx + r * (T[k] - tm);
            ++k;
        }
    double m = s / g.npix;
    double var = s2 / g.npix - m * m;
    double sd = sqrt(var > 0.0 ? var : 0.0);
    double den = (ts * sd) * g.npix;
    return den > 1e-6 ? sx / den : -2.0;
}

static void bil_u8(const u8* img, int H, int W, double x, double y, double* val, double* gx)
{
    int x0 = (int)floor(x), y0 = (int)floor(y);
    double ax = x - x0, ay = y - y0;
    if (x0 < 0) x0 = 0;
    if (x0 > W - 2) x0 = W - 2;
    if (y0 < 0) y0 = 0;
    if (y0 > H - 2) y0 = H - 2;
    double a = img[(size_t)y0 * W + x0], b = img[(size_t)y0 * W + x0 + 1];
    double c = img[(size_t)(y0 + 1) * W + x0], d = img[(size_t)(y0 + 1) * W + x0 + 1];
    double top = a + ax * (b - a);
    double bot = c + ax * (d - c);
    *val = top + ay * (bot - top);
    *gx = (b - a) * (1.0 - ay) + (d - c) * ay;
}

static void bil_f(const float* img, int H, int W, double x, double y, double* val, double* gx)
{
    int x0 = (int)floor(x), y0 = (int)floor(y);
    double ax = x - x0, ay = y - y0;
    if (x0 < 0) x0 = 0;
    if (x0 > W - 2) x0 = W - 2;
    if (y0 < 0) y0 = 0;
    if (y0 > H - 2) y0 = H - 2;
    float fa = img[(size_t)y0 * W + x0], fb = img[(size_t)y0 * W + x0 + 1];
    float fc = img[(size_t)(y0 + 1) * W + x0], fd = img[(size_t)(y0 + 1) * W + x0 + 1];
    double a = fa, c = fc;
    double ba = (double)(fb - fa), dc = (double)(fd - fc);
    double top = a + ax * ba;
    double bot = c + ax * dc;
    *val = top + ay * (bot - top);
    *gx = ba * (1.0 - ay) + dc * ay;
}

#define LK_ITERS 6
#define MAXD 128

/* _lk_v: affine 1-D LK on (d, gain, offset), sums over the patch pixels in row-major order -> (d, a, sigma, ok) */
static int lk_v(const u8* L, const float* R, int H, int W, double u, double v, double d0, double voff, Geo g,
                double* d_out, double* sig_out)
{
    double T[256], px[256], py[256];
    int k = 0;
    for (int gy = -g.half; gy <= g.half; ++gy)
        for (int gx = -g.half; gx <= g.half; ++gx) {
            px[k] = u + gx;
            py[k] = v + gy;
            double gg;
            bil_u8(L, H, W, px[k], py[k], &T[k], &gg);
            ++k;
        }
    double d = d0, a = 1.0, b = 0.0;
    for (int it = 0; it < LK_ITERS; ++it) {
        double A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, gv[3] = {0, 0, 0};
        for (k = 0; k < g.npix; ++k) {
            double rv, rg;
            bil_f(R, H, W, px[k] - d, py[k] + voff, &rv, &rg);
            double r = T[k] - (a * rv + b);
            double J[3] = {-a * rg, rv, 1.0};
            for (int i = 0; i < 3; ++i) {
                gv[i] = gv[i] + J[i] * r;
                for (int j = 0; j < 3; ++j) A[i][j] = A[i][j] + J[i] * J[j];
            }
        }
        for (int i = 0; i < 3; ++i) A[i][i] = A[i][i] + 1e-9;
        int piv[3];
        xo_getf2(A, piv);
        xo_getrs(A, piv, gv);
        d = d + gv[0];
        a = a + gv[1];
        b = b + gv[2];
        if (!(isfinite(d) && isfinite(a))) { *d_out = d; *sig_out = INFINITY; return 0; }
    }
    double A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    double s2 = 0.0;
    for (k = 0; k < g.npix; ++k) {
        double rv, rg;
        bil_f(R, H, W, px[k] - d, py[k] + voff, &rv, &rg);
        double r = T[k] - (a * rv + b);
        s2 = s2 + r * r;
        double J[3] = {-a * rg, rv, 1.0};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) A[i][j] = A[i][j] + J[i] * J[j];
    }
    for (int i = 0; i < 3; ++i) A[i][i] = A[i][i] + 1e-9;
    s2 = s2 / (g.npix - 3);
    int piv[3];
    xo_getf2(A, piv);
    xo_getri(A, piv);
    double var = s2 * A[0][0];
    double sig = var > 0.0 ? sqrt(var) : 0.0;
    *d_out = d;
    *sig_out = sig;
    return isfinite(d) && fabs(d - d0) <= 1.0 && a > 0.5 && a < 2.0;
}

/* stereo_points_band over N points; Rs = shifted float32 right image.  Outputs as stereo1d (d 0 / sig inf / ok 0 /
   zn -2 / dy NaN unless set). */
void xo_stereo(const u8* L, const float* Rs, int H, int W, const double* kp, const i64* dlo, const i64* dhi, int N,
               int band, int half, double* out_d, double* out_sig, u8* out_ok, double* out_zn, double* out_dy)
{
    Geo g = {half, 2 * half + 1, (2 * half + 1) * (2 * half + 1)};
    const double ZMIN = 0.5, UNIQ1 = 1.0 + 0.05, LRT = 1.0;
    double T[256], T2[256], sc[MAXD], col[64];
    int jb[MAXD];
    for (int n = 0; n < N; ++n) {
        out_ok[n] = 0; out_d[n] = 0.0; out_sig[n] = INFINITY; out_zn[n] = -2.0; out_dy[n] = NAN;
        double u = kp[2 * n], v = kp[2 * n + 1];
        int ui = (int)floor(u + 0.5), vi = (int)floor(v + 0.5);
        if (ui - half - 2 < 0 || ui + half + 2 >= W || vi - half - 2 - band < 0 || vi + half + 2 + band >= H) continue;
        i64 lo = dlo[n], hi = dhi[n];
        if (lo < 0) lo = 0;
        if (hi > MAXD - 1) hi = MAXD - 1;
        if (hi > ui - half - 2) hi = ui - half - 2;
        if (hi < lo) continue;
        int k = 0;
        for (int dy = -half; dy <= half; ++dy)
            for (int dx = -half; dx <= half; ++dx) T[k++] = (double)L[(size_t)(vi + dy) * W + ui + dx];
        double tm, ts;
        patch_stats_u8(L, W, ui, vi, g, &tm, &ts);
        if (ts <= 1e-6) continue;
        int best = -1;
        double bs = -2.0;
        for (int d = (int)lo; d <= (int)hi; ++d) {
            double s = zncc_f(T, tm, ts, Rs, W, ui - d, vi, g);
            int jj = 0;
            for (int j = 1; j <= band; ++j) {
                double s1 = zncc_f(T, tm, ts, Rs, W, ui - d, vi - j, g);
                if (s1 > s) { s = s1; jj = -j; }
                s1 = zncc_f(T, tm, ts, Rs, W, ui - d, vi + j, g);
                if (s1 > s) { s = s1; jj = j; }
            }
            sc[d] = s;
            jb[d] = jj;
            if (s > bs) { bs = s; best = d; }
        }
        out_zn[n] = bs;
        if (best < 0 || bs < ZMIN) continue;
        double sec = -2.0;
        for (int d = (int)lo; d <= (int)hi; ++d)
            if (abs(d - best) > 1 && sc[d] > sec) sec = sc[d];
        if (!((1.0 - sec) > (1.0 - bs) * UNIQ1)) continue;
        int js = jb[best];
        int xr = ui - best;
        k = 0;
        for (int dy = -half; dy <= half; ++dy)
            for (int dx = -half; dx <= half; ++dx) T2[k++] = (double)Rs[(size_t)(vi + js + dy) * W + xr + dx];
        double rm, rs;
        patch_stats_f(Rs, W, xr, vi + js, g, &rm, &rs);
        if (rs <= 1e-6) continue;
        int bb = -1;
        double bbs = -2.0;
        int dmax = MAXD - 1;
        if (xr + dmax + half >= W) dmax = W - 1 - half - xr;
        for (int d = 0; d <= dmax; ++d) {
            double s = zncc_u8(T2, rm, rs, L, W, xr + d, vi, g);
            if (s > bbs) { bbs = s; bb = d; }
        }
        if (bb < 0 || fabs((double)(bb - best)) > LRT) continue;
        double off = 0.0;
        if (best > lo && best < hi) {
            double y0 = sc[best - 1], y2 = sc[best + 1];
            double den = (y0 - 2.0 * bs) + y2;
            if (den < -1e-9) {
                off = (0.5 * (y0 - y2)) / den;
                if (off > 0.5) off = 0.5;
                if (off < -0.5) off = -0.5;
            }
        }
        double seed = ((double)best + off) + (u - (double)ui);
        double dl, sig;
        int conv = lk_v(L, Rs, H, W, u, v, seed, (double)js, g, &dl, &sig);
        if (!conv || dl < 0.5) continue;
        out_d[n] = dl;
        out_sig[n] = sig;
        out_ok[n] = 1;
        if (vi - 2 * half - 1 >= 0 && vi + 2 * half + 1 < H) {
            int jp = 0;
            double cs = -2.0;
            for (int j = -half; j <= half; ++j) {
                col[j + half] = zncc_f(T, tm, ts, Rs, W, xr, vi + j, g);
                if (col[j + half] > cs) { cs = col[j + half]; jp = j; }
            }
            double offy = 0.0;
            if (jp > -half && jp < half) {
                double y0 = col[jp - 1 + half], y2 = col[jp + 1 + half];
                double den = (y0 - 2.0 * cs) + y2;
                if (den < -1e-9) {
                    offy = (0.5 * (y0 - y2)) / den;
                    if (offy > 0.5) offy = 0.5;
                    if (offy < -0.5) offy = -0.5;
                }
            }
            out_dy[n] = (double)jp + offy;
        }
    }
}

/* ======================================================= hamming ======================================================= */
void xo_hamming(const u64* A, int L, const u64* B, int N, int* o1, int* o2, int* oi, int* ci)
{
    int* cb = (int*)malloc(sizeof(int) * (size_t)(N > 0 ? N : 1));
    for (int j = 0; j < N; ++j) { cb[j] = 1 << 30; ci[j] = -1; }
    for (int i = 0; i < L; ++i) {
        int r1 = 1 << 30, r2 = 1 << 30, ri = -1;
        for (int j = 0; j < N; ++j) {
            int d = __builtin_popcountll(A[4 * i] ^ B[4 * j]) + __builtin_popcountll(A[4 * i + 1] ^ B[4 * j + 1])
                    + __builtin_popcountll(A[4 * i + 2] ^ B[4 * j + 2]) + __builtin_popcountll(A[4 * i + 3] ^ B[4 * j + 3]);
            if (d < r1) { r2 = r1; r1 = d; ri = j; }
            else if (d < r2) r2 = d;
            if (d < cb[j]) { cb[j] = d; ci[j] = i; }
        }
        o1[i] = r1; o2[i] = r2; oi[i] = ri;
    }
    free(cb);
}

/* mutual NN + ratio + chance bound -> matches in query order; returns count */
int xo_match(const u64* A, int L, const u64* B, int N, int ham_max, double ratio, i64* m0, i64* m1)
{
    if (L < 2 || N < 2) return 0;
    int* o1 = (int*)malloc(sizeof(int) * L);
    int* o2 = (int*)malloc(sizeof(int) * L);
    int* oi = (int*)malloc(sizeof(int) * L);
    int* ci = (int*)malloc(sizeof(int) * N);
    xo_hamming(A, L, B, N, o1, o2, oi, ci);
    int m = 0;
    for (int i = 0; i < L; ++i) {
        int j = oi[i];
        if (j < 0) continue;
        if (o1[i] > ham_max || !((double)o1[i] < ratio * (double)o2[i])) continue;
        if (ci[j] != i) continue;
        m0[m] = i; m1[m] = j; ++m;
    }
    free(o1); free(o2); free(oi); free(ci);
    return m;
}

/* ============================================= one frame, end to end (CPU baseline) ============================================= */
/* detect + describe + stereo (+ match against a previous frame's descriptors when prev != NULL) for one stereo pair.
   kp (cap x 2 f32), desc (cap x 32), stereo outputs (cap each), matches m0/m1 (cap each).  -> keypoint count;
   *nmatch = match count. */
int xo_frame(const u8* left, const u8* right, int H, int W, int budget, int cap, double Q, int dy_vend, int dx_vend,
             const float* kf, int vr, int vc, const int8_t* pat, int half, int dlo, int dhi, const u8* prev_desc,
             int nprev, float* kp, u8* desc, double* d, double* sig, u8* ok, double* zn, double* dy, i64* m0, i64* m1,
             int* nmatch)
{
    size_t npx = (size_t)H * W;
    float* R = (float*)malloc(sizeof(float) * npx);
    xo_response(left, H, W, dy_vend, dx_vend, R);
    float ff;
    xo_noise_floor(left, H, W, Q, &ff);
    int nc;
    int cnt = xo_detect(R, H, W, budget, ff, cap, kp, &nc);
    u8* Bl = (u8*)malloc((size_t)(H + 64) * (W + 64));
    xo_blur(left, H, W, kf, vr, vc, Bl);
    xo_orb(Bl, W + 64, kp, cnt, pat, desc);
    float* Rs = (float*)malloc(sizeof(float) * npx);
    xo_shift_rows(right, H, W, 0.0, Rs);
    double* kpd = (double*)malloc(sizeof(double) * 2 * (size_t)(cnt > 0 ? cnt : 1));
    i64* lo = (i64*)malloc(sizeof(i64) * (size_t)(cnt > 0 ? cnt : 1));
    i64* hi = (i64*)malloc(sizeof(i64) * (size_t)(cnt > 0 ? cnt : 1));
    for (int i = 0; i < cnt; ++i) { kpd[2 * i] = kp[2 * i]; kpd[2 * i + 1] = kp[2 * i + 1]; lo[i] = dlo; hi[i] = dhi; }
    xo_stereo(left, Rs, H, W, kpd, lo, hi, cnt, 0, half, d, sig, ok, zn, dy);
    *nmatch = 0;
    if (prev_desc)
        *nmatch = xo_match((const u64*)prev_desc, nprev, (const u64*)desc, cnt, 104, 0.8, m0, m1);
    free(R); free(Bl); free(Rs); free(kpd); free(lo); free(hi);
    return cnt;
}

/* F frames in parallel (OpenMP over frames; frame f matches against frame f-1 of the same batch, frame 0 against
   prev0 when given).  Arrays are frame-major with per-frame capacity cap.  -> total keypoints. */
long xo_frames(const u8* left, const u8* right, int F, int H, int W, int budget, int cap, double Q, int dy_vend,
               int dx_vend, const float* kf, int vr, int vc, const int8_t* pat, int half, int dlo, int dhi,
               int nthreads, int* counts, float* kp, u8* desc, double* d, double* sig, u8* ok, double* zn, double* dy,
               i64* m0, i64* m1, int* nmatch)
{
    size_t npx = (size_t)H * W;
    /* pass 1: detection + description (independent frames) */
    long tot = 0;
    #pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1) reduction(+ : tot)
    for (int f = 0; f < F; ++f) {
        int mm;
        counts[f] = xo_frame(left + f * npx, right + f * npx, H, W, budget, cap, Q, dy_vend, dx_vend, kf, vr, vc, pat,
                             half, dlo, dhi, NULL, 0, kp + (size_t)f * cap * 2, desc + (size_t)f * cap * 32,
                             d + (size_t)f * cap, sig + (size_t)f * cap, ok + (size_t)f * cap, zn + (size_t)f * cap,
                             dy + (size_t)f * cap, NULL, NULL, &mm);
        tot += counts[f];
    }
    /* pass 2: match frame f against frame f-1 */
    #pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
    for (int f = 1; f < F; ++f)
        nmatch[f] = xo_match((const u64*)(desc + (size_t)(f - 1) * cap * 32), counts[f - 1],
                             (const u64*)(desc + (size_t)f * cap * 32), counts[f], 104, 0.8, m0 + (size_t)f * cap,
                             m1 + (size_t)f * cap);
    if (F > 0) nmatch[0] = 0;
    return tot;
}

/* ================================================== gated map matching ================================================== */
/* float64 -> int64 as x86-64 converts it (numpy astype(np.int64) and numba int() both compile to cvttsd2si there):
   NaN and values outside the int64 range give INT64_MIN ("integer indefinite") */
static i64 xo_f2i64(double v)
{
    if (!(v >= -9223372036854775808.0 && v < 9223372036854775808.0)) return INT64_MIN;
    return (i64)v;
}

static int xo_ham4(const u64* a, const u64* b)
{
    return __builtin_popcountll(a[0] ^ b[0]) + __builtin_popcountll(a[1] ^ b[1]) + __builtin_popcountll(a[2] ^ b[2])
           + __builtin_popcountll(a[3] ^ b[3]);
}

/* MapMatcher.match for one frame (the caller has already returned the defaults for L == 0 or N == 0).
   kp (N x 2) float64, kd (N x 4 words), uvp (L x 2), S (L x 2 x 2), ld (L x D x 4 words), lnd (L).
   Preamble (mapmatch.py:158-166): det, Sinv, half = sqrt(max(chi2 S_ii, 0)) with NaN kept, nd = lnd where det > 0.
   Grid (mapmatch.py:141-146): cell = clip(x // 16) + gw clip(y // 16), stable counting sort.
   Gated search (mapmatch.py:52-112): visit the cells of the gate's bounding box row by row, a cell's keypoints in
   index order; keep the best (Hamming, then Mahalanobis d2) and the second-best distance; chance bound and ratio.
   Mutual step (mapmatch.py:113-131): landmarks in index order claim their keypoint; a later claimant takes it only
   with a smaller distance, or an equal distance and a smaller d2. */
void xo_mapmatch(const double* kp, int N, const u64* kd, const double* uvp, const double* S, const u64* ld, int D,
                 const i64* lnd, int L, int gw, int gh, double chi2, double ratio, int ham_max, i64* out_kp, i64* out_d,
                 double* out_d2)
{
    const int grid = 16;
    double* Sinv = (double*)calloc((size_t)L * 4 + 1, sizeof(double));
    double* half = (double*)malloc(sizeof(double) * ((size_t)L * 2 + 1));
    i64* nd = (i64*)calloc((size_t)L + 1, sizeof(i64));
    for (int l = 0; l < L; ++l) {
        const double* s = S + 4 * (size_t)l;
        double det = s[0] * s[3] - s[1] * s[2];
        if (det > 0) {
            Sinv[4 * l + 0] = s[3] / det;
            Sinv[4 * l + 3] = s[0] / det;
            Sinv[4 * l + 1] = -s[1] / det;
            Sinv[4 * l + 2] = -s[2] / det;
            nd[l] = lnd[l];
        }
        for (int a = 0; a < 2; ++a) {
            double h = chi2 * s[3 * a];
            half[2 * l + a] = sqrt((h >= 0.0 || isnan(h)) ? h : 0.0);
        }
    }
    const int ncell = gw * gh;
    i64* cstart = (i64*)calloc((size_t)ncell + 1, sizeof(i64));
    i64* cur = (i64*)malloc(sizeof(i64) * (size_t)ncell);
    int* cell = (int*)malloc(sizeof(int) * (size_t)N);
    int* cidx = (int*)malloc(sizeof(int) * (size_t)N);
    for (int k = 0; k < N; ++k) {
        i64 cx = xo_f2i64(floor(kp[2 * k] / grid)), cy = xo_f2i64(floor(kp[2 * k + 1] / grid));
        cx = cx < 0 ? 0 : (cx > gw - 1 ? gw - 1 : cx);
        cy = cy < 0 ? 0 : (cy > gh - 1 ? gh - 1 : cy);
        cell[k] = (int)(cy * gw + cx);
        cstart[cell[k] + 1] += 1;
    }
    for (int c = 0; c < ncell; ++c) cstart[c + 1] += cstart[c];
    for (int c = 0; c < ncell; ++c) cur[c] = cstart[c];
    for (int k = 0; k < N; ++k) cidx[cur[cell[k]]++] = k;
    for (int l = 0; l < L; ++l) {
        out_kp[l] = -1;
        out_d[l] = 9999;
        out_d2[l] = INFINITY;
        const double u = uvp[2 * l], v = uvp[2 * l + 1];
        if (nd[l] <= 0 || !(isfinite(u) && isfinite(v))) continue;
        i64 x0 = xo_f2i64(floor((u - half[2 * l]) / grid)), x1 = xo_f2i64(floor((u + half[2 * l]) / grid));
        i64 y0 = xo_f2i64(floor((v - half[2 * l + 1]) / grid)), y1 = xo_f2i64(floor((v + half[2 * l + 1]) / grid));
        if (x0 < 0) x0 = 0;
        if (y0 < 0) y0 = 0;
        if (x1 > gw - 1) x1 = gw - 1;
        if (y1 > gh - 1) y1 = gh - 1;
        const double* si = Sinv + 4 * (size_t)l;
        int best = 9999, second = 9999;
        i64 bk = -1;
        double bd2 = INFINITY;
        for (i64 cy = y0; cy <= y1; ++cy)
            for (i64 cx = x0; cx <= x1; ++cx) {
                const i64 c = cy * gw + cx;
                for (i64 t = cstart[c]; t < cstart[c + 1]; ++t) {
                    const int k = cidx[t];
                    const double dx = kp[2 * k] - u, dy = kp[2 * k + 1] - v;
                    const double d2 = dx * (si[0] * dx + si[1] * dy) + dy * (si[2] * dx + si[3] * dy);
                    if (d2 > chi2) continue;
                    int h = 9999;
                    for (i64 j = 0; j < nd[l]; ++j) {
                        int hj = xo_ham4(kd + 4 * (size_t)k, ld + 4 * ((size_t)l * D + j));
                        if (hj < h) h = hj;
                    }
                    if (h < best || (h == best && d2 < bd2)) {
                        second = best;
                        best = h;
                        bk = k;
                        bd2 = d2;
                    } else if (h < second) {
                        second = h;
                    }
                }
            }
        if (bk < 0 || best > ham_max) continue;
        if (second < 9999 && !((double)best < ratio * (double)second)) continue;
        out_kp[l] = bk;
        out_d[l] = best;
        out_d2[l] = bd2;
    }
    i64* owner = (i64*)malloc(sizeof(i64) * ((size_t)N + 1));
    for (int k = 0; k < N; ++k) owner[k] = -1;
    for (int l = 0; l < L; ++l) {
        const i64 k = out_kp[l];
        if (k < 0) continue;
        const i64 o = owner[k];
        if (o < 0) { owner[k] = l; continue; }
        if (out_d[l] < out_d[o] || (out_d[l] == out_d[o] && out_d2[l] < out_d2[o])) {
            owner[k] = l;
            out_kp[o] = -1;
        } else {
            out_kp[l] = -1;
        }
    }
    free(owner); free(cidx); free(cell); free(cur); free(cstart); free(nd); free(half); free(Sinv);
}

/* F frames of MapMatcher.match (frame f: counts_kp[f] keypoints of kp_stride, counts_lm[f] landmarks of lm_stride),
   OpenMP over frames with nthreads threads; float32 keypoints as the frontend stores them (widened to float64 as
   MapMatcher.match does). */
void xo_mapmatch_frames(const float* kp32, const int* counts_kp, int kp_stride, const u8* desc, const double* uvp,
                        const double* S, const u8* ld, int D, const i64* lnd, const int* counts_lm, int lm_stride, int F,
                        int gw, int gh, double chi2, int nthreads, i64* out_kp, i64* out_d, double* out_d2)
{
    #pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
    for (int f = 0; f < F; ++f) {
        const int N = counts_kp[f], L = counts_lm[f];
        i64* ok = out_kp + (size_t)f * lm_stride;
        i64* od = out_d + (size_t)f * lm_stride;
        double* od2 = out_d2 + (size_t)f * lm_stride;
        for (int l = 0; l < L; ++l) { ok[l] = -1; od[l] = 9999; od2[l] = INFINITY; }
        if (L == 0 || N == 0) continue;
        double* kp = (double*)malloc(sizeof(double) * 2 * (size_t)N);
        for (int i = 0; i < 2 * N; ++i) kp[i] = (double)kp32[(size_t)f * kp_stride * 2 + i];
        xo_mapmatch(kp, N, (const u64*)(desc + (size_t)f * kp_stride * 32), uvp + (size_t)f * lm_stride * 2,
                    S + (size_t)f * lm_stride * 4, (const u64*)(ld + (size_t)f * lm_stride * D * 32), D,
                    lnd + (size_t)f * lm_stride, L, gw, gh, chi2, 0.8, 104, ok, od, od2);
        free(kp);
    }
}

/* ================================================ gating prediction ================================================ */
/* window.predict_projection (src/xclean/vio/window.py:1032-1144): every landmark (host camera Rwc_h / pwc_h, inverse-
   depth state a, b, rho) projected into the predicted body pose (Rwb_t, pwb_t) through the body-to-camera extrinsic
   (Rbc, pbc); S = Jp Spose Jp^T + Jl Sl Jl^T + sig_px^2 I.  Writes ok for every landmark, uv and depth where the point
   is in front (q2 > 1e-9, rho > 0), S where it also projects inside the image; other entries are left as they are.
   Row-major 3x3 / 6x6 arrays; every sum in the reference's order. */
static void xo_mm3(const double* A, const double* B, double* out)
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) out[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}

void xo_predict_projection(const double* Rwb_t, const double* pwb_t, const double* Rbc, const double* pbc,
                           const double* Rwc_h, const double* pwc_h, const double* lmp, const double* Spose,
                           const double* Sl, double sig_px, double fx, double fy, double cx, double cy, double W,
                           double H, int L, double* uv, double* S, u8* ok, double* depth)
{
    double Rwc_t[9], pwc_t[3], Rcb[9], Px[9] = {0}, Wt[9], Rct[9], RctWt[9];
    xo_mm3(Rwb_t, Rbc, Rwc_t);
    for (int i = 0; i < 3; ++i) pwc_t[i] = pwb_t[i] + Rwb_t[3 * i] * pbc[0] + Rwb_t[3 * i + 1] * pbc[1] + Rwb_t[3 * i + 2] * pbc[2];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Rcb[3 * i + j] = Rbc[3 * j + i];
    Px[1] = -pbc[2]; Px[2] = pbc[1]; Px[3] = pbc[2]; Px[5] = -pbc[0]; Px[6] = -pbc[1]; Px[7] = pbc[0];
    xo_mm3(Rwb_t, Px, Wt);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Rct[3 * i + j] = Rwc_t[3 * j + i];
    xo_mm3(Rct, Wt, RctWt);
    double Qx[9] = {0}, QR[9], Jp[12], Jl[6], RcR[9], Dp[6], t6[12], t3[6];
    for (int l = 0; l < L; ++l) {
        ok[l] = 0;
        const double* R = Rwc_h + 9 * (size_t)l;
        const double a = lmp[3 * l], b = lmp[3 * l + 1], rho = lmp[3 * l + 2];
        const double d0 = pwc_h[3 * l] - pwc_t[0], d1 = pwc_h[3 * l + 1] - pwc_t[1], d2 = pwc_h[3 * l + 2] - pwc_t[2];
        const double Y0 = R[0] * a + R[1] * b + R[2] + rho * d0;
        const double Y1 = R[3] * a + R[4] * b + R[5] + rho * d1;
        const double Y2 = R[6] * a + R[7] * b + R[8] + rho * d2;
        const double q0 = Rct[0] * Y0 + Rct[1] * Y1 + Rct[2] * Y2;
        const double q1 = Rct[3] * Y0 + Rct[4] * Y1 + Rct[5] * Y2;
        const double q2 = Rct[6] * Y0 + Rct[7] * Y1 + Rct[8] * Y2;
        if (q2 <= 1e-9 || rho <= 0.0) continue;
        depth[l] = q2 / rho;
        const double iq = 1.0 / q2;
        const double u = fx * q0 * iq + cx, v = fy * q1 * iq + cy;
        uv[2 * l] = u;
        uv[2 * l + 1] = v;
        if (u < 0.0 || u >= W || v < 0.0 || v >= H) continue;
        Dp[0] = fx * iq; Dp[1] = 0.0; Dp[2] = -fx * q0 * iq * iq;
        Dp[3] = 0.0; Dp[4] = fy * iq; Dp[5] = -fy * q1 * iq * iq;
        Qx[1] = -q2; Qx[2] = q1; Qx[3] = q2; Qx[5] = -q0; Qx[6] = -q1; Qx[7] = q0;
        xo_mm3(Qx, Rcb, QR);
        for (int r = 0; r < 2; ++r)
            for (int j = 0; j < 3; ++j) {
                Jp[6 * r + j] = Dp[3 * r] * (QR[j] + rho * RctWt[j]) + Dp[3 * r + 1] * (QR[3 + j] + rho * RctWt[3 + j])
                                + Dp[3 * r + 2] * (QR[6 + j] + rho * RctWt[6 + j]);
                Jp[6 * r + 3 + j] = -rho * (Dp[3 * r] * Rct[j] + Dp[3 * r + 1] * Rct[3 + j] + Dp[3 * r + 2] * Rct[6 + j]);
            }
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) RcR[3 * i + j] = Rct[3 * i] * R[j] + Rct[3 * i + 1] * R[3 + j] + Rct[3 * i + 2] * R[6 + j];
        const double e0 = Rct[0] * d0 + Rct[1] * d1 + Rct[2] * d2;
        const double e1 = Rct[3] * d0 + Rct[4] * d1 + Rct[5] * d2;
        const double e2 = Rct[6] * d0 + Rct[7] * d1 + Rct[8] * d2;
        for (int r = 0; r < 2; ++r) {
            Jl[3 * r] = Dp[3 * r] * RcR[0] + Dp[3 * r + 1] * RcR[3] + Dp[3 * r + 2] * RcR[6];
            Jl[3 * r + 1] = Dp[3 * r] * RcR[1] + Dp[3 * r + 1] * RcR[4] + Dp[3 * r + 2] * RcR[7];
            Jl[3 * r + 2] = Dp[3 * r] * e0 + Dp[3 * r + 1] * e1 + Dp[3 * r + 2] * e2;
        }
        const double* sl = Sl + 9 * (size_t)l;
        for (int r = 0; r < 2; ++r) {
            for (int j = 0; j < 6; ++j) {
                double acc = 0.0;
                for (int k = 0; k < 6; ++k) acc += Jp[6 * r + k] * Spose[6 * k + j];
                t6[6 * r + j] = acc;
            }
            for (int j = 0; j < 3; ++j) {
                double acc = 0.0;
                for (int k = 0; k < 3; ++k) acc += Jl[3 * r + k] * sl[3 * k + j];
                t3[3 * r + j] = acc;
            }
        }
        for (int r = 0; r < 2; ++r)
            for (int c = 0; c < 2; ++c) {
                double acc = 0.0;
                for (int k = 0; k < 6; ++k) acc += t6[6 * r + k] * Jp[6 * c + k];
                for (int k = 0; k < 3; ++k) acc += t3[3 * r + k] * Jl[3 * c + k];
                S[4 * (size_t)l + 2 * r + c] = acc + (r == c ? sig_px * sig_px : 0.0);
            }
        ok[l] = 1;
    }
}
