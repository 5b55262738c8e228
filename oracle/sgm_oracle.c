/* sgm_oracle.c -- CPU restatement of the reference's dense 32-direction SGM (test infrastructure: the checker of the
 * device SGM, never the product path).
 *
 * src/xclean/stereo/sgm32.py (its module notes and its kernel string, :105-266): census 9x9 (80 comparisons, the
 * centre skipped without taking a bit, bits 0..63 in one word and 64..79 in a second; a neighbour outside the image
 * reads as the centre), Hamming cost volume over d = 0..127 (the census maximum 80 where x - d < 0), one aggregation
 * of Hirschmueller's recursion along 32 directed paths (sgm32.py:84-93 directions, :96-102 path starts, penalties
 * P1 * num / den, P2 * num / den per family) summed into one uint16 volume, the left winner with the uniqueness test
 * against the best non-adjacent disparity and the parabola, the right winner read off the same volume's diagonal,
 * the left-right check.  float32 arithmetic in the reference's order (no contraction).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define SGM_D 128
#define SGM_BITS 80
#define SGM_INF (1 << 28)

static void census9(const uint8_t* img, int H, int W, uint64_t* w0, uint16_t* w1)
{
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const uint8_t c = img[y * W + x];
            uint64_t a = 0;
            unsigned b = 0;
            int bit = 0;
            for (int dy = -4; dy <= 4; ++dy)
                for (int dx = -4; dx <= 4; ++dx) {
                    if (!dx && !dy) continue;
                    const int nx = x + dx, ny = y + dy;
                    const uint8_t v = (nx >= 0 && nx < W && ny >= 0 && ny < H) ? img[ny * W + nx] : c;
                    const unsigned s = v < c;
                    if (bit < 64) a |= (uint64_t)s << bit;
                    else b |= s << (bit - 64);
                    ++bit;
                }
            w0[y * W + x] = a;
            w1[y * W + x] = (uint16_t)b;
        }
}

/* the 32 directions: 4 axis paths, then the 7 oblique families with every sign combination */
static int directions(int* dx, int* dy, int* num, int* den)
{
    static const int fam[7][4] = {{1, 1, 1, 1}, {1, 2, 9, 4}, {2, 1, 9, 4}, {1, 3, 19, 6},
                                  {3, 1, 19, 6}, {2, 3, 18, 5}, {3, 2, 18, 5}};
    int k = 0;
    const int ax[4][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}};
    for (int i = 0; i < 4; ++i) { dx[k] = ax[i][0]; dy[k] = ax[i][1]; num[k] = 1; den[k] = 1; ++k; }
    for (int f = 0; f < 7; ++f)
        for (int sx = 1; sx >= -1; sx -= 2)
            for (int sy = 1; sy >= -1; sy -= 2) {
                dx[k] = sx * fam[f][0]; dy[k] = sy * fam[f][1]; num[k] = fam[f][2]; den[k] = fam[f][3]; ++k;
            }
    return k;
}

static inline int imin(int a, int b) { return a < b ? a : b; }

/* S (H x W x 128 uint16) += the aggregation of every path of every direction */
static void aggregate(const uint8_t* C, int H, int W, int p1b, int p2b, uint16_t* S)
{
    int dx[32], dy[32], num[32], den[32];
    const int nd = directions(dx, dy, num, den);
    int* Lc = (int*)malloc(SGM_D * sizeof(int));
    int* Ln = (int*)malloc(SGM_D * sizeof(int));
    for (int k = 0; k < nd; ++k) {
        const int p1 = p1b * num[k] / den[k], p2 = p2b * num[k] / den[k];
        for (int y0 = 0; y0 < H; ++y0)
            for (int x0 = 0; x0 < W; ++x0) {
                const int px = x0 - dx[k], py = y0 - dy[k];
                if (px >= 0 && px < W && py >= 0 && py < H) continue;      /* not a path start */
                int x = x0, y = y0;
                const uint8_t* c = C + ((size_t)y * W + x) * SGM_D;
                int mprev = SGM_INF;
                for (int d = 0; d < SGM_D; ++d) {
                    Lc[d] = c[d];
                    S[((size_t)y * W + x) * SGM_D + d] += (uint16_t)Lc[d];
                    mprev = imin(mprev, Lc[d]);
                }
                x += dx[k]; y += dy[k];
                while (x >= 0 && x < W && y >= 0 && y < H) {
                    c = C + ((size_t)y * W + x) * SGM_D;
                    const int mp2 = mprev + p2;
                    int mn = SGM_INF;
                    for (int d = 0; d < SGM_D; ++d) {
                        const int left = d > 0 ? Lc[d - 1] : SGM_INF, right = d < SGM_D - 1 ? Lc[d + 1] : SGM_INF;
                        Ln[d] = (int)c[d] + imin(imin(Lc[d], mp2), imin(left, right) + p1) - mprev;
                    }
                    for (int d = 0; d < SGM_D; ++d) {
                        Lc[d] = Ln[d];
                        S[((size_t)y * W + x) * SGM_D + d] += (uint16_t)Ln[d];
                        mn = imin(mn, Ln[d]);
                    }
                    mprev = mn;
                    x += dx[k]; y += dy[k];
                }
            }
    }
    free(Lc);
    free(Ln);
}

/* the whole SGM of a rectified pair: disp (0 = invalid) and conf; optional C (H x W x 128) and S outputs */
void xo_sgm(const uint8_t* L, const uint8_t* R, int H, int W, int p1, int p2, float uniq, float lr_thr, float dmin,
            float* disp, float* conf, uint8_t* C_out, uint16_t* S_out)
{
    const size_t n = (size_t)H * W;
    uint64_t* l0 = (uint64_t*)malloc(n * 8);
    uint64_t* r0 = (uint64_t*)malloc(n * 8);
    uint16_t* l1 = (uint16_t*)malloc(n * 2);
    uint16_t* r1 = (uint16_t*)malloc(n * 2);
    census9(L, H, W, l0, l1);
    census9(R, H, W, r0, r1);
    uint8_t* C = C_out ? C_out : (uint8_t*)malloc(n * SGM_D);
    uint16_t* S = S_out ? S_out : (uint16_t*)malloc(n * SGM_D * 2);
    for (size_t p = 0; p < n; ++p) {
        const int x = (int)(p % (size_t)W);
        for (int d = 0; d < SGM_D; ++d) {
            if (x - d < 0) { C[p * SGM_D + d] = SGM_BITS; continue; }
            const size_t q = p - (size_t)d;
            C[p * SGM_D + d] = (uint8_t)(__builtin_popcountll(l0[p] ^ r0[q]) + __builtin_popcount((unsigned)(l1[p] ^ r1[q])));
        }
    }
    memset(S, 0, n * SGM_D * 2);
    aggregate(C, H, W, p1, p2, S);
    float* dr = (float*)malloc(n * sizeof(float));
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            /* the right winner of right pixel x: S(y, x + d, d) */
            const int nd = imin(SGM_D, W - x);
            unsigned best = 0xFFFFFFFFu;
            int bd = 0;
            for (int d = 0; d < nd; ++d) {
                const unsigned c = S[((size_t)y * W + x + d) * SGM_D + d];
                if (c < best) { best = c; bd = d; }
            }
            float sd = (float)bd;
            if (bd > 0 && bd < nd - 1) {
                const int cv = (int)S[((size_t)y * W + x + bd - 1) * SGM_D + bd - 1];
                const int cn = (int)S[((size_t)y * W + x + bd + 1) * SGM_D + bd + 1];
                const int dn = cv - 2 * (int)best + cn;
                if (dn > 0) {
                    const float off = (float)(cv - cn) / (float)(2 * dn);
                    sd = (float)bd + fmaxf(-1.0f, fminf(1.0f, off));
                }
            }
            dr[(size_t)y * W + x] = sd;
        }
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const size_t p = (size_t)y * W + x;
            const uint16_t* s = S + p * SGM_D;
            const int nd = imin(SGM_D, x + 1);
            unsigned best = 0xFFFFFFFFu, sec = 0xFFFFFFFFu;
            int bd = 0;
            for (int d = 0; d < nd; ++d)
                if (s[d] < best) { best = s[d]; bd = d; }
            for (int d = 0; d < nd; ++d)
                if (abs(d - bd) > 1 && s[d] < sec) sec = s[d];
            if (sec != 0xFFFFFFFFu && (float)sec <= (float)best * (1.0f + uniq)) { disp[p] = 0.0f; conf[p] = 0.0f; continue; }
            float sd = (float)bd;
            if (bd > 0 && bd < nd - 1) {
                const int cv = (int)s[bd - 1], cc = (int)best, cn = (int)s[bd + 1];
                const int dn = cv - 2 * cc + cn;
                if (dn > 0) {
                    const float off = (float)(cv - cn) / (float)(2 * dn);
                    sd = (float)bd + fmaxf(-1.0f, fminf(1.0f, off));
                }
            }
            const float cval = (sec != 0xFFFFFFFFu && sec > 0) ? 1.0f - (float)best / (float)sec : 0.5f;
            disp[p] = sd >= dmin ? sd : 0.0f;
            conf[p] = sd >= dmin ? fmaxf(0.0f, fminf(1.0f, cval)) : 0.0f;
        }
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const size_t i = (size_t)y * W + x;
            const float d = disp[i];
            if (d <= 0.0f) continue;
            const int xr = x - (int)(d + 0.5f);
            if (xr < 0 || xr >= W || fabsf(d - dr[(size_t)y * W + xr]) > lr_thr) { disp[i] = 0.0f; conf[i] = 0.0f; }
        }
    free(dr);
    if (!C_out) free(C);
    if (!S_out) free(S);
    free(l0); free(r0); free(l1); free(r1);
}
