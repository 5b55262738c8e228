/* ext_oracle.c -- CPU restatement of the frontend's multi-scale, oriented extras (test infrastructure: the checker of
 * the device FAST / pyramid / orientation / steered rBRIEF, never the product path).
 *
 * These go beyond the reference (its frontend is single-scale Shi-Tomasi with unoriented ORB,
 * src/xclean/stages/features.py:27-28, :102-103; src/xclean/front/gpu_front.py:1712-1717).  The definitions follow
 * OpenCV where OpenCV defines them, and the tests pin them to cv2 itself:
 *   FAST       cv2.FastFeatureDetector TYPE_9_16: a pixel at least 3 px inside is a corner at threshold t when 9
 *              contiguous pixels of its 16-pixel radius-3 circle are all brighter than p + t or all darker than p - t;
 *              its score is the largest t at which it is still a corner (found here by bisection over t with the
 *              segment test itself); non-maximum suppression keeps a corner whose score beats all 8 neighbours'
 *              (a non-corner counts 0).  Row-major order.
 *   pyramid    cv2.resize INTER_LINEAR_EXACT: source coordinate (d + 1/2) ns / nd - 1/2, exact; an 8-bit weight
 *              rounded half to even; clamped at both ends; the two passes in 8.8 fixed point, rounded at the end.
 *   steering   the rBRIEF of the reference's describe stage at KeyPoint.angle = 12 k (the rotated tables are inputs).
 * Own definitions (no cv2 counterpart): the top-quota selection (score descending, ties in row-major order) and the
 * orientation bins (the intensity centroid over u^2 + v^2 <= 240, bin k of 30 centred on 12 k degrees, decided by sign
 * tests against the directions at 12 k - 6 and 12 k + 6 degrees).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static const int circ16[16][2] = {{0, -3}, {1, -3}, {2, -2}, {3, -1}, {3, 0}, {3, 1}, {2, 2}, {1, 3},
                                  {0, 3}, {-1, 3}, {-2, 2}, {-3, 1}, {-3, 0}, {-3, -1}, {-2, -2}, {-1, -3}};

/* the segment test at threshold t */
static int fast_corner_at(const uint8_t* img, int W, int x, int y, int t)
{
    const int p = img[y * W + x];
    int st[16];
    for (int k = 0; k < 16; ++k) {
        const int v = img[(y + circ16[k][1]) * W + x + circ16[k][0]];
        st[k] = v > p + t ? 1 : (v < p - t ? -1 : 0);
    }
    for (int s = 0; s < 16; ++s) {
        int bright = 1, dark = 1;
        for (int j = 0; j < 9; ++j) {
            bright &= st[(s + j) % 16] == 1;
            dark &= st[(s + j) % 16] == -1;
        }
        if (bright || dark) return 1;
    }
    return 0;
}

/* -> the score map (-1 = no corner at thr) */
static void fast_scores(const uint8_t* img, int H, int W, int thr, int* sc)
{
    for (int i = 0; i < H * W; ++i) sc[i] = -1;
    for (int y = 3; y < H - 3; ++y)
        for (int x = 3; x < W - 3; ++x) {
            if (!fast_corner_at(img, W, x, y, thr)) continue;
            int lo = thr, hi = 255;               /* corner at lo, not at hi (no pixel differs by more than 255) */
            while (hi - lo > 1) {
                const int mid = (lo + hi) / 2;
                if (fast_corner_at(img, W, x, y, mid)) lo = mid;
                else hi = mid;
            }
            sc[y * W + x] = lo;
        }
}

long xo_fast(const uint8_t* img, int H, int W, int thr, int nms, long cap, float* kp, float* resp)
{
    int* sc = (int*)malloc(sizeof(int) * (size_t)H * W);
    fast_scores(img, H, W, thr, sc);
    long n = 0;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const int s = sc[y * W + x];
            if (s < 0) continue;
            int keep = 1;
            if (nms)
                for (int dy = -1; dy <= 1 && keep; ++dy)
                    for (int dx = -1; dx <= 1 && keep; ++dx) {
                        if (!dx && !dy) continue;
                        const int yy = y + dy, xx = x + dx;
                        int t = 0;
                        if (yy >= 0 && yy < H && xx >= 0 && xx < W && sc[yy * W + xx] > 0) t = sc[yy * W + xx];
                        if (!(s > t)) keep = 0;
                    }
            if (!keep) continue;
            if (n < cap) {
                kp[2 * n] = (float)x;
                kp[2 * n + 1] = (float)y;
                resp[n] = (float)s;
            }
            ++n;
        }
    free(sc);
    return n;
}

typedef struct {
    float s;
    long i;
} XoSel;

static int sel_cmp(const void* a, const void* b)
{
    const XoSel *p = (const XoSel*)a, *q = (const XoSel*)b;
    if (p->s != q->s) return p->s > q->s ? -1 : 1;
    return p->i < q->i ? -1 : (p->i > q->i ? 1 : 0);
}

static int idx_cmp(const void* a, const void* b)
{
    const long p = *(const long*)a, q = *(const long*)b;
    return p < q ? -1 : (p > q ? 1 : 0);
}

/* of n keypoints, those at least `edge` inside: the quota best by score, ties by input order; written in input order */
long xo_fast_select(const float* kp, const float* resp, long n, int W, int H, int edge, long quota, float* kpo,
                    float* respo)
{
    XoSel* v = (XoSel*)malloc(sizeof(XoSel) * (size_t)(n + 1));
    long m = 0;
    for (long i = 0; i < n; ++i) {
        const float x = kp[2 * i], y = kp[2 * i + 1];
        if (x >= edge && x < W - edge && y >= edge && y < H - edge) {
            v[m].s = resp[i];
            v[m].i = i;
            ++m;
        }
    }
    qsort(v, (size_t)m, sizeof(XoSel), sel_cmp);
    const long k = m < quota ? m : quota;
    long* id = (long*)malloc(sizeof(long) * (size_t)(k + 1));
    for (long j = 0; j < k; ++j) id[j] = v[j].i;
    qsort(id, (size_t)k, sizeof(long), idx_cmp);
    for (long j = 0; j < k; ++j) {
        kpo[2 * j] = kp[2 * id[j]];
        kpo[2 * j + 1] = kp[2 * id[j] + 1];
        respo[j] = resp[id[j]];
    }
    free(v);
    free(id);
    return k;
}

/* source index and 8-bit weight along one axis */
static void lin_exact(int ns, int nd, int d, int* i0, int* w)
{
    /* src = ((2 d + 1) ns - nd) / (2 nd) */
    const long long num = (2LL * d + 1) * ns - nd, den = 2LL * nd;
    long long fl = num / den;
    if (num % den != 0 && num < 0) fl -= 1;       /* floor */
    const long long rem = num - fl * den;         /* [0, den) */
    /* round half to even of rem * 256 / den */
    const long long t = rem * 256, q = t / den, r2 = 2 * (t - q * den);
    long long wt = q;
    if (r2 > den || (r2 == den && (q % 2 == 1))) wt = q + 1;
    if (fl < 0) {
        fl = 0;
        wt = 0;
    }
    if (fl >= ns - 1) {
        fl = ns - 1;
        wt = 0;
    }
    *i0 = (int)fl;
    *w = (int)wt;
}

void xo_pyr_down(const uint8_t* src, int Hs, int Ws, uint8_t* dst, int Hd, int Wd)
{
    for (int y = 0; y < Hd; ++y) {
        int ya, wy;
        lin_exact(Hs, Hd, y, &ya, &wy);
        const int yb = ya + 1 < Hs ? ya + 1 : Hs - 1;
        for (int x = 0; x < Wd; ++x) {
            int xa, wx;
            lin_exact(Ws, Wd, x, &xa, &wx);
            const int xb = xa + 1 < Ws ? xa + 1 : Ws - 1;
            const long r0 = (long)src[ya * Ws + xa] * (256 - wx) + (long)src[ya * Ws + xb] * wx;
            const long r1 = (long)src[yb * Ws + xa] * (256 - wx) + (long)src[yb * Ws + xb] * wx;
            dst[y * Wd + x] = (uint8_t)((r0 * (256 - wy) + r1 * wy + (1L << 15)) >> 16);
        }
    }
}

/* orientation bins (and the moments) of n keypoints on img */
void xo_ic_bins(const uint8_t* img, int H, int W, const float* kp, long n, int32_t* bins, int64_t* mom)
{
    double bd[30][2], cd[30][2];
    const double d2r = M_PI / 180.0;
    for (int k = 0; k < 30; ++k) {
        bd[k][0] = cos((double)(12 * k - 6) * d2r);
        bd[k][1] = sin((double)(12 * k - 6) * d2r);
        cd[k][0] = cos((double)(12 * k) * d2r);
        cd[k][1] = sin((double)(12 * k) * d2r);
    }
    for (long i = 0; i < n; ++i) {
        const int cx = (int)lrintf(kp[2 * i]), cy = (int)lrintf(kp[2 * i + 1]);
        int64_t m10 = 0, m01 = 0;
        for (int v = -15; v <= 15; ++v)
            for (int u = -15; u <= 15; ++u) {
                if (u * u + v * v > 240) continue;
                const int x = cx + u, y = cy + v;
                const int I = (x >= 0 && x < W && y >= 0 && y < H) ? img[y * W + x] : 0;
                m10 += (int64_t)u * I;
                m01 += (int64_t)v * I;
            }
        int bin = 0;
        if (m10 || m01) {
            const double X = (double)m10, Y = (double)m01;
            for (int k = 0; k < 30; ++k) {
                const int k1 = (k + 1) % 30;
                const double a = bd[k][0] * Y - bd[k][1] * X;
                const double b = bd[k1][0] * Y - bd[k1][1] * X;
                const double c = cd[k][0] * X + cd[k][1] * Y;
                if (a >= 0.0 && b < 0.0 && c > 0.0) {
                    bin = k;
                    break;
                }
            }
        }
        bins[i] = bin;
        if (mom) {
            mom[2 * i] = m10;
            mom[2 * i + 1] = m01;
        }
    }
}

/* steered rBRIEF: pats [30][256][4]; a point outside the padded image reads 0 */
void xo_orb_steer(const uint8_t* blur, int Hp, int Wp, int pad, const float* kp, long n, const int32_t* bins,
                  const int8_t* pats, uint8_t* desc)
{
    for (long i = 0; i < n; ++i) {
        const int cx = (int)lrintf(kp[2 * i] + (float)pad), cy = (int)lrintf(kp[2 * i + 1] + (float)pad);
        const int8_t* t = pats + (size_t)bins[i] * 1024;
        for (int j = 0; j < 32; ++j) {
            int byte = 0;
            for (int b = 0; b < 8; ++b) {
                const int8_t* q = t + 4 * (8 * j + b);
                const int x1 = cx + q[0], y1 = cy + q[1], x2 = cx + q[2], y2 = cy + q[3];
                const int v1 = (x1 >= 0 && x1 < Wp && y1 >= 0 && y1 < Hp) ? blur[y1 * Wp + x1] : 0;
                const int v2 = (x2 >= 0 && x2 < Wp && y2 >= 0 && y2 < Hp) ? blur[y2 * Wp + x2] : 0;
                if (v1 < v2) byte |= 1 << b;
            }
            desc[i * 32 + j] = (uint8_t)byte;
        }
    }
}
