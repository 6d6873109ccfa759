/*
 * tcoracle.c — CPU restatement of the TCodec v2 pixel-pipeline kernels.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the sm_100a kernels, never part
 * of the product.  Parity pinned against the reference library built from
 * the reference sources (tests/test_oracle.py) wherever the reference
 * exports the function; the encoder-internal helpers (RDOQ, bit model,
 * MV predictor, global-motion walk) are pinned through end-to-end
 * bitstream equality of the GPU encoder with the reference encoder.
 */
#include "tcoracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static int clipi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static int iabs(int v) { return v < 0 ? -v : v; }

/* ------------------------------------------------------------------ */
/* Quantiser tables (reference src/quantize.c:30-85, 286-293).         */
/* ------------------------------------------------------------------ */
static const int QSCALE[64] = {
    1, 1, 1, 1, 1, 2, 2, 2, 3, 3, 4, 4, 5, 6, 7, 8,
    9, 10, 12, 14, 16, 18, 21, 24, 28, 32, 37, 42, 49, 56, 64, 74,
    85, 98, 112, 128, 149, 171, 197, 226, 256, 299, 343, 394, 453, 512, 598, 686,
    788, 907, 1024, 1196, 1373, 1576, 1814, 2048, 2392, 2745, 3153, 3629, 4096, 4784, 5490, 6305};
static const int JND[4] = {6, 7, 8, 10};

int or_qscale(int qp) { return QSCALE[clipi(qp, 0, 63)]; }
int or_eff_scale(int qp, int band) {
    int e = (or_qscale(qp) * JND[clipi(band, 0, 3)] + 4) >> 3;
    return e < 1 ? 1 : e;
}
int or_lambda(int qp) {
    long long s = or_qscale(qp), l = (s * s * 200) >> 10;
    if (l < 1) l = 1;
    if (l > (1LL << 30)) l = 1LL << 30;
    return (int)l;
}
/* Band of a raster coefficient index (reference src/entropy.c:72-79). */
int or_freq_band(int pos, int n) {
    if (pos == 0) return 0;
    if (pos < n / 4) return 1;
    if (pos < n / 2) return 2;
    return 3;
}
/* Dead-zone quantiser / centroid dequantiser (tcodec_common.h:232-246). */
int or_quant(int c, int eff) {
    int off = eff / 3;
    if (c > 0) return (c + off) / eff;
    if (c < 0) return -((-c + off) / eff);
    return 0;
}
int or_dequant(int q, int eff) {
    int b = eff / 6;
    if (q > 0) return q * eff + b;
    if (q < 0) return q * eff - b;
    return 0;
}

/* ------------------------------------------------------------------ */
/* Transforms (reference src/transform.c:313-439, 502-636).            */
/* ------------------------------------------------------------------ */
void or_dct_matrix(int n, int *m) {
    const double pi = 3.14159265358979323846;
    for (int k = 0; k < n; k++)
        for (int j = 0; j < n; j++) {
            double s = k == 0 ? sqrt(1.0 / n) : sqrt(2.0 / n);
            m[k * n + j] = (int)lround(16384.0 * s * cos((2 * j + 1) * k * pi / (2.0 * n)));
        }
}

/* One rounded 14-bit pass: out[k] = (sum_j M(k,j) in[j] + 2^13) >> 14,
 * M = C (forward) or C^T (inverse), 64-bit accumulation. */
static void dct_pass(int n, const int *m, const long long *in, long long *out, int inverse) {
    for (int k = 0; k < n; k++) {
        long long acc = 0;
        for (int j = 0; j < n; j++) acc += (long long)(inverse ? m[j * n + k] : m[k * n + j]) * in[j];
        out[k] = (acc + (1 << 13)) >> 14;
    }
}

static void dct2d(int n, const int16_t *in, int is, int16_t *out, int os, int inverse) {
    int m[64];
    long long tmp[8][8], t2[8][8], v[8];
    or_dct_matrix(n, m);
    for (int i = 0; i < n; i++) {
        for (int j = 0; j < n; j++) v[j] = in[i * is + j];
        dct_pass(n, m, v, tmp[i], inverse);
    }
    for (int j = 0; j < n; j++) {
        for (int i = 0; i < n; i++) v[i] = tmp[i][j];
        dct_pass(n, m, v, t2[j], inverse);
    }
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) out[i * os + j] = (int16_t)(int)t2[j][i];
}

void or_fdct(int n, const int16_t *in, int is, int16_t *out) { dct2d(n, in, is, out, n, 0); }
void or_idct(int n, const int16_t *in, int16_t *out, int os) { dct2d(n, in, n, out, os, 1); }

/* Walsh-Hadamard: H4 butterfly s=a+c, t=b+d, u=a-c, v=b-d -> (s+t, s-t,
 * u+v, u-v); H8 = H4 on the sum and difference halves; the column pass
 * rounds by n (reference src/transform.c:526-636). */
static void had(int n, const int *x, int *y) {
    if (n == 4) {
        int s = x[0] + x[2], t = x[1] + x[3], u = x[0] - x[2], v = x[1] - x[3];
        y[0] = s + t; y[1] = s - t; y[2] = u + v; y[3] = u - v;
    } else {
        int a[4], b[4];
        for (int i = 0; i < 4; i++) { a[i] = x[i] + x[i + 4]; b[i] = x[i] - x[i + 4]; }
        had(4, a, y);
        had(4, b, y + 4);
    }
}
static void wht2d(int n, const int16_t *in, int is, int16_t *out, int os) {
    int tmp[8][8], v[8], r[8];
    int sh = n == 4 ? 2 : 3;
    for (int i = 0; i < n; i++) {
        for (int j = 0; j < n; j++) v[j] = in[i * is + j];
        had(n, v, tmp[i]);
    }
    for (int j = 0; j < n; j++) {
        for (int i = 0; i < n; i++) v[i] = tmp[i][j];
        had(n, v, r);
        for (int i = 0; i < n; i++) out[i * os + j] = (int16_t)((r[i] + (1 << (sh - 1))) >> sh);
    }
}
void or_fwht(int n, const int16_t *in, int is, int16_t *out) { wht2d(n, in, is, out, n); }
void or_iwht(int n, const int16_t *in, int16_t *out, int os) { wht2d(n, in, n, out, os); }

/* ------------------------------------------------------------------ */
/* Fused residual coding of one TU (reference src/encoder.c:488-536).  */
/* ------------------------------------------------------------------ */
static int bitlen_u(unsigned v) { int b = 0; while (v) { b++; v >>= 1; } return b; }

long long or_code_tu(int n, const uint8_t *org, int os, const uint8_t *pred, int ps, int qp,
                     long long lambda, int16_t *lv, uint8_t *rec, int rs, int *bits) {
    int16_t res[64] = {0}, co[64], dq[64], rr[64];
    const int nn = n * n;
    for (int y = 0; y < n; y++)
        for (int x = 0; x < n; x++)
            res[y * n + x] = (int16_t)clipi((int)org[y * os + x] - (int)pred[y * ps + x], -512, 511);
    or_fdct(n, res, n, co);
    int nz = 0, last = -1;
    for (int i = 0; i < nn; i++) {
        int eff = or_eff_scale(qp, or_freq_band(i, nn));
        int q = (int16_t)or_quant(co[i], eff);
        /* RDOQ-lite keep-vs-zero for |level| == 1 (src/encoder.c:333-355). */
        if (q == 1 || q == -1) {
            int d = or_dequant(q, eff), c = co[i];
            long long dz = (long long)c * c + lambda;
            long long dk = (long long)(c - d) * (c - d) + 2 * lambda;
            if (dz < dk) q = 0;
        }
        lv[i] = (int16_t)q;
    }
    for (int i = 0; i < nn; i++) if (lv[i]) { nz++; last = i; }
    /* Bit model 1 + 2 nz + sig/level terms + last-position cost
     * (src/encoder.c:360-385). */
    int b = 1 + 2 * nz;
    for (int i = 0; i <= last; i++) b += lv[i] ? 2 + 2 * bitlen_u((unsigned)iabs(lv[i])) : 1;
    if (last < 0) b += 1;
    else if (last < 4) b += 1 + (last + 1) + 1;
    else b += 1 + 5 + (2 * bitlen_u((unsigned)(last - 4) + 1) - 1);
    *bits = b;
    for (int i = 0; i < nn; i++) dq[i] = (int16_t)or_dequant(lv[i], or_eff_scale(qp, or_freq_band(i, nn)));
    or_idct(n, dq, rr, n);
    long long sse = 0;
    for (int y = 0; y < n; y++)
        for (int x = 0; x < n; x++) {
            int v = clipi((int)pred[y * ps + x] + rr[y * n + x], 0, 255);
            int d = (int)org[y * os + x] - v;
            rec[y * rs + x] = (uint8_t)v;
            sse += d * d;
        }
    return sse;
}

/* ------------------------------------------------------------------ */
/* Motion (reference src/motion.c:40-632).                              */
/* ------------------------------------------------------------------ */
int or_sad(const uint8_t *a, int sa, const uint8_t *b, int sb, int n) {
    int s = 0;
    for (int y = 0; y < n; y++)
        for (int x = 0; x < n; x++) s += iabs((int)a[y * sa + x] - (int)b[y * sb + x]);
    return s;
}

static int tap6(int a, int b, int c, int d, int e, int f) {
    return (a - 5 * b + 20 * c + 20 * d - 5 * e + f + 16) >> 5;
}
static int hh(const uint8_t *r, int s, int x, int y) {
    const uint8_t *p = r + y * s + x;
    return tap6(p[-2], p[-1], p[0], p[1], p[2], p[3]);
}
static int vv(const uint8_t *r, int s, int x, int y) {
    const uint8_t *p = r + y * s + x;
    return tap6(p[-2 * s], p[-s], p[0], p[s], p[2 * s], p[3 * s]);
}
static int dd(const uint8_t *r, int s, int x, int y) {
    return tap6(hh(r, s, x, y - 2), hh(r, s, x, y - 1), hh(r, s, x, y), hh(r, s, x, y + 1),
                hh(r, s, x, y + 2), hh(r, s, x, y + 3));
}
/* Horizontal / vertical quarter-pel: integer, (int + half + 1)/2, half,
 * (half + next + 1)/2, clipped (src/motion.c:133-188). */
static int qh(const uint8_t *r, int s, int x, int y, int f) {
    int a = r[y * s + x];
    if (f == 0) return a;
    int h = hh(r, s, x, y);
    if (f == 2) return clipi(h, 0, 255);
    if (f == 1) return clipi((a + h + 1) / 2, 0, 255);
    return clipi((h + r[y * s + x + 1] + 1) / 2, 0, 255);
}
static int qv(const uint8_t *r, int s, int x, int y, int f) {
    int a = r[y * s + x];
    if (f == 0) return a;
    int v = vv(r, s, x, y);
    if (f == 2) return clipi(v, 0, 255);
    if (f == 1) return clipi((a + v + 1) / 2, 0, 255);
    return clipi((v + r[(y + 1) * s + x] + 1) / 2, 0, 255);
}
/* Diagonal: horizontal blend on rows y, y+1/2, y+1 then vertical blend
 * (src/motion.c:190-260). */
static int qhv(const uint8_t *r, int s, int x, int y, int fx, int fy) {
    int a00 = r[y * s + x], a10 = r[y * s + x + 1], a01 = r[(y + 1) * s + x], a11 = r[(y + 1) * s + x + 1];
    int b = hh(r, s, x, y), e = hh(r, s, x, y + 1), c = vv(r, s, x, y), f = vv(r, s, x + 1, y);
    int d = dd(r, s, x, y);
    int row[3];
    const int A[3] = {a00, c, a01}, H[3] = {b, d, e}, B[3] = {a10, f, a11};
    for (int k = 0; k < 3; k++) {
        if (fx == 0) row[k] = A[k];
        else if (fx == 1) row[k] = (A[k] + H[k] + 1) >> 1;
        else if (fx == 2) row[k] = H[k];
        else row[k] = (H[k] + B[k] + 1) >> 1;
    }
    int v;
    if (fy == 0) v = row[0];
    else if (fy == 1) v = (row[0] + row[1] + 1) >> 1;
    else if (fy == 2) v = row[1];
    else v = (row[1] + row[2] + 1) >> 1;
    return clipi(v, 0, 255);
}
static int blend4(int a, int b, int f) { return clipi((a * (4 - f) + b * f + 2) / 4, 0, 255); }

static int luma_sample(const uint8_t *r, int s, int w, int h, int x, int y, int fx, int fy) {
    if (x >= 2 && x + 3 < w && y >= 2 && y + 3 < h) {
        if (!fx && !fy) return r[y * s + x];
        if (!fy) return qh(r, s, x, y, fx);
        if (!fx) return qv(r, s, x, y, fy);
        return qhv(r, s, x, y, fx, fy);
    }
    if (x >= 0 && y >= 0 && x + 1 < w && y + 1 < h) {
        int t = blend4(r[y * s + x], r[y * s + x + 1], fx);
        int u = blend4(r[(y + 1) * s + x], r[(y + 1) * s + x + 1], fx);
        return blend4(t, u, fy);
    }
    return r[clipi(y + (fy >= 2), 0, h - 1) * s + clipi(x + (fx >= 2), 0, w - 1)];
}

void or_pred_luma(const uint8_t *r, int s, int w, int h, int mvx, int mvy, uint8_t *dst, int ds, int n) {
    int x0 = mvx >> 2, y0 = mvy >> 2, fx = mvx & 3, fy = mvy & 3;
    int inside = x0 >= 0 && y0 >= 0 && x0 + n <= w && y0 + n <= h;
    int full6 = x0 >= 2 && x0 + n + 2 < w && y0 >= 2 && y0 + n + 2 < h;
    for (int y = 0; y < n; y++)
        for (int x = 0; x < n; x++) {
            int v;
            if (!fx && !fy && inside) v = r[(y0 + y) * s + x0 + x];
            else if ((fx || fy) && full6)
                v = !fy ? qh(r, s, x0 + x, y0 + y, fx)
                        : (!fx ? qv(r, s, x0 + x, y0 + y, fy) : qhv(r, s, x0 + x, y0 + y, fx, fy));
            else v = luma_sample(r, s, w, h, x0 + x, y0 + y, fx, fy);
            dst[y * ds + x] = (uint8_t)v;
        }
}

void or_pred_chroma(const uint8_t *r, int s, int w, int h, int mvx, int mvy, uint8_t *dst, int ds, int n) {
    int xi = mvx >> 3, yi = mvy >> 3, fx = mvx & 7, fy = mvy & 7;
    for (int y = 0; y < n; y++)
        for (int x = 0; x < n; x++) {
            int y0 = clipi(yi + y, 0, h - 1), y1 = clipi(yi + y + 1, 0, h - 1);
            int xa = clipi(xi + x, 0, w - 1), xb = clipi(xi + x + 1, 0, w - 1);
            int v = ((8 - fx) * (8 - fy) * r[y0 * s + xa] + fx * (8 - fy) * r[y0 * s + xb] +
                     (8 - fx) * fy * r[y1 * s + xa] + fx * fy * r[y1 * s + xb] + 32) >> 6;
            dst[y * ds + x] = (uint8_t)v;
        }
}

static int sad_at(const uint8_t *r, int rs, int w, int h, const uint8_t *o, int os, int n, int x, int y) {
    if (x < 0 || y < 0 || x + n > w || y + n > h) return 0x7FFFFFFF;
    return or_sad(r + y * rs + x, rs, o, os, n);
}

/* Hexagon -> small hexagon -> diamond integer search with in-pass commit,
 * then eight quarter-pel neighbours (src/motion.c:384-485). */
void or_motion_est(const uint8_t *r, int rs, int w, int h, const uint8_t *o, int os, int cx, int cy,
                   int n, int sr, int *mvx, int *mvy, int *sadout) {
    static const int L[7][2] = {{0, 0}, {-2, -4}, {2, -4}, {-4, 0}, {4, 0}, {-2, 4}, {2, 4}};
    static const int S[7][2] = {{0, 0}, {-1, -2}, {1, -2}, {-2, 0}, {2, 0}, {-1, 2}, {1, 2}};
    static const int D[5][2] = {{0, 0}, {0, -1}, {-1, 0}, {1, 0}, {0, 1}};
    static const int Q[9][2] = {{0, 0}, {1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {-1, 1}, {1, -1}, {-1, -1}};
    int bx = clipi(cx, 0, w - n), by = clipi(cy, 0, h - n);
    int best = sad_at(r, rs, w, h, o, os, n, bx, by);
    int scale = sr / 4 < 1 ? 1 : sr / 4;
    const int (*pat[3])[2] = {L, S, D};
    const int npts[3] = {6, 6, 4}, iters[3] = {2, 3, 4}, sc[3] = {scale, 1, 1};
    for (int st = 0; st < 3; st++)
        for (int it = 0; it < iters[st]; it++) {
            int improved = 0;
            for (int p = 1; p <= npts[st]; p++) {
                int x = bx + pat[st][p][0] * sc[st], y = by + pat[st][p][1] * sc[st];
                int s = sad_at(r, rs, w, h, o, os, n, x, y);
                if (s < best) { best = s; bx = x; by = y; improved = 1; }
            }
            if (!improved) break;
        }
    int qx = bx * 4, qy = by * 4;
    for (int p = 1; p < 9; p++) {
        int cxq = qx + Q[p][0], cyq = qy + Q[p][1], fx = cxq >> 2, fy = cyq >> 2, dx = cxq & 3, dy = cyq & 3;
        if (fx < 0 || fy < 0 || fx + n + 1 > w || fy + n + 1 > h) continue;
        int s = 0;
        int six = fx >= 2 && fy >= 2 && fx + n + 2 < w && fy + n + 2 < h;
        for (int y = 0; y < n; y++)
            for (int x = 0; x < n; x++) {
                int pv;
                if (six) pv = qhv(r, rs, fx + x, fy + y, dx, dy);
                else {
                    const uint8_t *q = r + (fy + y) * rs + fx + x;
                    pv = blend4(blend4(q[0], q[1], dx), blend4(q[rs], q[rs + 1], dx), dy);
                }
                s += iabs((int)o[y * os + x] - pv);
            }
        if (s < best) { best = s; qx = cxq; qy = cyq; }
    }
    *mvx = qx; *mvy = qy;
    if (sadout) *sadout = best;
}

/* Minimum-magnitude predictor over left / above / above-right cells
 * (src/encoder.c:405-427). */
void or_mvp(const or_mvcell_t *g, int cx, int cy, int *mx, int *my) {
    int v[3][2] = {{0, 0}, {0, 0}, {0, 0}}, has[3] = {0, 0, 0};
    const int pos[3][2] = {{cx - 1, cy}, {cx, cy - 1}, {cx + 1, cy - 1}};
    const int ok[3] = {cx > 0, cy > 0, cy > 0 && cx < 7};
    for (int k = 0; k < 3; k++)
        if (ok[k]) {
            const or_mvcell_t *c = &g[pos[k][1] * 8 + pos[k][0]];
            if (!c->intra) { v[k][0] = c->dx; v[k][1] = c->dy; has[k] = 1; }
        }
    if (!has[0] && !has[1] && !has[2]) { *mx = 0; *my = 0; return; }
    if (!has[0]) { v[0][0] = has[1] ? v[1][0] : v[2][0]; v[0][1] = has[1] ? v[1][1] : v[2][1]; }
    if (!has[1]) { v[1][0] = has[0] ? v[0][0] : v[2][0]; v[1][1] = has[0] ? v[0][1] : v[2][1]; }
    if (!has[2]) { v[2][0] = has[0] ? v[0][0] : v[1][0]; v[2][1] = has[0] ? v[0][1] : v[1][1]; }
    long long q[3];
    for (int k = 0; k < 3; k++) q[k] = (long long)v[k][0] * v[k][0] + (long long)v[k][1] * v[k][1];
    int pick = 0;
    if (q[1] < q[0] && q[1] <= q[2]) pick = 1;
    else if (q[2] < q[0] && q[2] < q[1]) pick = 2;
    *mx = v[pick][0]; *my = v[pick][1];
}

/* ------------------------------------------------------------------ */
/* Intra (reference src/predict.c:117-520).                             */
/* ------------------------------------------------------------------ */
void or_intra_refs(const uint8_t *rec, int s, int x, int y, int n, int w, int h, uint8_t *ra, uint8_t *rl) {
    int up = y > 0, left = x > 0;
    int tl = up && left ? rec[(y - 1) * s + x - 1] : (up ? rec[(y - 1) * s + x] : (left ? rec[y * s + x - 1] : 128));
    for (int i = 0; i < n; i++) {
        ra[1 + i] = up ? rec[(y - 1) * s + (x + i < w ? x + i : w - 1)] : (left ? rec[y * s + x - 1] : 128);
    }
    for (int i = 0; i < n; i++) {
        rl[1 + i] = left ? rec[(y + i < h ? y + i : h - 1) * s + x - 1] : (up ? ra[1] : 128);
    }
    for (int i = n; i <= 2 * n; i++) { ra[1 + i] = ra[n]; rl[1 + i] = rl[n]; }
    ra[0] = rl[0] = (uint8_t)tl;
}

void or_intra_pred(uint8_t *dst, int ds, const uint8_t *ra0, const uint8_t *rl0, int n, int mode) {
    const uint8_t *A = ra0 + 1, *Lf = rl0 + 1;   /* A[-1] = corner */
    static const int DV[7] = {32, 16, 6, 0, -6, -16, -32};
    static const int DH[9] = {32, 16, 6, 0, -6, -16, -32, -48, 48};
    int dc = 0;
    for (int i = 0; i < n; i++) dc += A[i + 1] + Lf[i + 1];
    dc = (dc + n) / (2 * n);
    for (int y = 0; y < n; y++)
        for (int x = 0; x < n; x++) {
            int v;
            if (mode == 0) {
                v = clipi((A[x + 1] * (n - 1 - y) + Lf[y + 1] * (n - 1 - x) + A[0] * (x + y) + n) / (2 * n), 0, 255);
            } else if (mode == 1 || mode < 0 || mode > 17) {
                v = dc;
            } else {
                int vert = mode < 9, disp = vert ? DV[mode - 2] : DH[mode - 9];
                int pos = vert ? (x << 5) + y * disp : (y << 5) + x * disp;
                const uint8_t *src = vert ? A : Lf;
                if (!(disp >= 0 || pos >= 0)) { src = vert ? Lf : A; pos = -pos; }
                int i0 = (pos >> 5) + 1, fr = pos & 31;
                int p0 = src[clipi(i0, 0, 2 * n)], p1 = src[clipi(i0 + 1, 0, 2 * n)];
                v = clipi(p0 + (((p1 - p0) * fr + 16) >> 5), 0, 255);
            }
            dst[y * ds + x] = (uint8_t)v;
        }
}

void or_chroma_dc(const uint8_t *rec, int s, int cx, int cy, int cs, uint8_t *dst, int ds) {
    int sum = 0, n = 0;
    if (cy > 0) for (int i = 0; i < cs; i++) { sum += rec[(cy - 1) * s + cx + i]; n++; }
    if (cx > 0) for (int i = 0; i < cs; i++) { sum += rec[(cy + i) * s + cx - 1]; n++; }
    int dc = n ? (sum + n / 2) / n : 128;
    for (int y = 0; y < cs; y++) memset(dst + y * ds, dc, (size_t)cs);
}

/* CfL: sign and shift from neighbour covariance, per-4x4-tile luma mean
 * (src/predict.c:390-462). */
void or_cfl_blend(uint8_t *dst, int ds, const uint8_t *Y, int sy, const uint8_t *C, int sc,
                  int lx, int ly, int cx, int cy, int cw, int ch) {
    long long sl = 0, sm = 0, slc = 0, sl2 = 0, n = 0;
    if (ly > 0 && cy > 0)
        for (int x = 0; x < cw; x++) {
            int la = (Y[(ly - 1) * sy + lx + 2 * x] + Y[(ly - 1) * sy + lx + 2 * x + 1] + 1) >> 1;
            int c = C[(cy - 1) * sc + cx + x];
            sl += la; sm += c; slc += (long long)la * c; sl2 += (long long)la * la; n++;
        }
    if (lx > 0 && cx > 0)
        for (int y = 0; y < ch; y++) {
            const uint8_t *r0 = Y + (ly + 2 * y) * sy, *r1 = r0 + sy;
            int la = (r0[lx - 2] + r0[lx - 1] + r1[lx - 2] + r1[lx - 1] + 2) >> 2;
            int c = C[(cy + y) * sc + cx - 1];
            sl += la; sm += c; slc += (long long)la * c; sl2 += (long long)la * la; n++;
        }
    int sign = (n == 0 || n * slc >= sl * sm) ? 1 : -1;
    int sh = 3;
    long long cov = n * slc - sl * sm, vl = n * sl2 - sl * sl;
    if (n > 0 && vl > 0 && cov != 0) {
        unsigned long long q = (unsigned long long)vl / (unsigned long long)(cov < 0 ? -cov : cov);
        int s = q < 1 ? 2 : (q > 0xFFFFFFFFull ? 5 : bitlen_u((unsigned)q) - 1);
        sh = s < 2 ? 2 : (s > 5 ? 5 : s);
    }
    for (int ty = 0; ty < ch; ty += 4)
        for (int tx = 0; tx < cw; tx += 4) {
            int ye = ty + 4 < ch ? ty + 4 : ch, xe = tx + 4 < cw ? tx + 4 : cw, sum = 0, m = 0;
            int la[4][4];
            for (int y = ty; y < ye; y++)
                for (int x = tx; x < xe; x++) {
                    const uint8_t *r0 = Y + (ly + 2 * y) * sy + lx + 2 * x, *r1 = r0 + sy;
                    la[y - ty][x - tx] = (r0[0] + r0[1] + r1[0] + r1[1] + 2) >> 2;
                    sum += la[y - ty][x - tx]; m++;
                }
            int avg = m ? (sum + m / 2) / m : 128;
            for (int y = ty; y < ye; y++)
                for (int x = tx; x < xe; x++) {
                    int v = (int)dst[y * ds + x] + sign * ((la[y - ty][x - tx] - avg) >> sh);
                    dst[y * ds + x] = (uint8_t)clipi(v, 0, 255);
                }
        }
}

/* ------------------------------------------------------------------ */
/* In-loop filters (reference src/filter.c:23-319).                     */
/* ------------------------------------------------------------------ */
static int strength(int p0, int q0, int qp) {
    int d = iabs(p0 - q0);
    if (d < clipi(qp / 4, 2, 16)) return 2;
    if (d < clipi(qp / 2, 4, 32)) return 1;
    if (d < clipi(qp, 8, 48)) return 1;
    return 0;
}
static int weak(int p1, int p0, int q0, int q1, int tc) {
    int d = clipi((9 * (q0 - p0) - 3 * (q1 - p1) + 8) >> 4, -tc, tc);
    return clipi(p0 + d, 0, 255);
}

void or_deblock_ctu(uint8_t *Y, int sy, uint8_t *cb, int scb, uint8_t *cr, int scr, int x0, int y0, int qp) {
    int tc = clipi(qp / 3, 1, 10);
    for (int e = 1; e < 16; e++)
        for (int r = 0; r < 64; r++) {
            uint8_t *p = Y + (y0 + r) * sy + x0 + 4 * e;
            int p1 = p[-2], p0 = p[-1], q0 = p[0], q1 = p[1];
            if (strength(p0, q0, qp)) { p[-1] = (uint8_t)weak(p1, p0, q0, q1, tc); p[0] = (uint8_t)weak(q1, q0, p0, p1, tc); }
        }
    for (int e = 1; e < 16; e++)
        for (int c = 0; c < 64; c++) {
            uint8_t *p = Y + (y0 + 4 * e) * sy + x0 + c;
            int p1 = p[-2 * sy], p0 = p[-sy], q0 = p[0], q1 = p[sy];
            if (strength(p0, q0, qp)) { p[-sy] = (uint8_t)weak(p1, p0, q0, q1, tc); p[0] = (uint8_t)weak(q1, q0, p0, p1, tc); }
        }
    int cq = clipi(qp - 1, 0, 63), ctc = clipi(cq / 4, 1, 6);
    for (int e = 1; e < 8; e++)
        for (int r = 0; r < 32; r++) {
            uint8_t *p = cb + (y0 / 2 + r) * scb + x0 / 2 + 4 * e;
            int p0 = p[-1], q0 = p[0];
            if (strength(p0, q0, cq)) {
                int d = clipi((q0 - p0 + 1) >> 1, -ctc, ctc);
                p[-1] = (uint8_t)clipi(p0 + d, 0, 255); p[0] = (uint8_t)clipi(q0 - d, 0, 255);
            }
        }
    for (int e = 1; e < 8; e++)
        for (int c = 0; c < 32; c++) {
            uint8_t *pr = cr + (y0 / 2 + 4 * e) * scr + x0 / 2 + c, *pb = cb + (y0 / 2 + 4 * e) * scb + x0 / 2 + c;
            int p0 = pr[0], q0 = pr[scr], b0 = pb[0], b1 = pb[scb];
            if (strength(p0, q0, cq)) {
                int d = clipi((q0 - p0 + 1) >> 1, -ctc, ctc);
                pr[0] = (uint8_t)clipi(p0 + d, 0, 255); pr[scr] = (uint8_t)clipi(q0 - d, 0, 255);
                d = clipi((b1 - b0 + 1) >> 1, -ctc, ctc);
                pb[0] = (uint8_t)clipi(b0 + d, 0, 255); pb[scb] = (uint8_t)clipi(b1 - d, 0, 255);
            }
        }
}

int or_sao_choose(const uint8_t *org, int os, const uint8_t *rec, int rs, int x, int y, int w, int h,
                  int *band, int *offset) {
    int x1 = x + 64 < w ? x + 64 : w, y1 = y + 64 < h ? y + 64 : h;
    long long sum[32] = {0}, cnt[32] = {0}, base = 0;
    for (int r = y; r < y1; r++)
        for (int c = x; c < x1; c++) {
            int d = (int)org[r * os + c] - (int)rec[r * rs + c];
            base += (long long)d * d;
            sum[rec[r * rs + c] >> 3] += d;
            cnt[rec[r * rs + c] >> 3]++;
        }
    long long best = base;
    int bb = 0, bo = 0;
    for (int b = 0; b < 32; b++) {
        if (!cnt[b]) continue;
        int cand = clipi((int)((sum[b] + (sum[b] >= 0 ? cnt[b] / 2 : -cnt[b] / 2)) / cnt[b]), -7, 7);
        if (!cand) continue;
        long long sse = 0;
        for (int r = y; r < y1; r++)
            for (int c = x; c < x1; c++) {
                int v = rec[r * rs + c];
                if ((v >> 3) == b) v = clipi(v + cand, 0, 255);
                int d = (int)org[r * os + c] - v;
                sse += (long long)d * d;
            }
        if (sse < best) { best = sse; bb = b; bo = cand; }
    }
    if (best >= base) return 0;
    *band = bb; *offset = bo;
    return 1;
}

void or_sao_apply(uint8_t *Y, int s, int x, int y0, int w, int h, int band, int offset) {
    int x1 = x + 64 < w ? x + 64 : w, y1 = y0 + 64 < h ? y0 + 64 : h;
    band = clipi(band, 0, 31); offset = clipi(offset, -7, 7);
    for (int r = y0; r < y1; r++)
        for (int c = x; c < x1; c++) {
            uint8_t *p = Y + r * s + c;
            if ((*p >> 3) == band) *p = (uint8_t)clipi(*p + offset, 0, 255);
        }
}

/* SAO decision of one CTU as the v2 encoder makes it (src/encoder.c:
 * 1463-1493): tc_sao_choose_bo, then keep the offset only if its SSE plus
 * 6 * tc_lambda(qp) is below the unfiltered SSE.  Returns present. */
int or_sao_decide(const uint8_t *org, int os, const uint8_t *rec, int rs, int x, int y, int w, int h,
                  int qp, int *band, int *offset) {
    int b = 0, o = 0;
    int has = or_sao_choose(org, os, rec, rs, x, y, w, h, &b, &o);
    if (has) {
        int x1 = x + 64 < w ? x + 64 : w, y1 = y + 64 < h ? y + 64 : h;
        long long base = 0, cost = 0;
        for (int r = y; r < y1; r++)
            for (int c = x; c < x1; c++) {
                int ov = org[r * os + c], rv = rec[r * rs + c];
                int r1 = (rv >> 3) == b ? clipi(rv + o, 0, 255) : rv;
                base += (long long)(ov - rv) * (ov - rv);
                cost += (long long)(ov - r1) * (ov - r1);
            }
        if (cost + (long long)or_lambda(qp) * 6 >= base) has = 0;
    }
    *band = has ? b : 0;
    *offset = has ? o : 0;
    return has;
}

/* Two-pass greedy walk over a 4x-decimated SAD, committing each
 * improvement in scan order (src/encoder.c:171-202). */
void or_global_mv(const uint8_t *cur, const uint8_t *ref, int w, int h, int s, int *gx, int *gy) {
    int cw = w / 4, ch = h / 4, bdx = 0, bdy = 0;
    long long best = 1LL << 60;
    for (int pass = 0; pass < 2; pass++) {
        int step = pass ? 1 : 2, range = pass ? 1 : 8;
        for (int dy = -range; dy <= range; dy += step)
            for (int dx = -range; dx <= range; dx += step) {
                long long sad = 0;
                for (int yy = 0; yy < ch; yy += 2)
                    for (int xx = 0; xx < cw; xx += 2) {
                        int rx = xx * 4 + bdx + dx * 4, ry = yy * 4 + bdy + dy * 4;
                        if (rx < 0 || ry < 0 || rx >= w || ry >= h) { sad += 255 * 4; continue; }
                        sad += iabs((int)cur[yy * 4 * s + xx * 4] - (int)ref[ry * s + rx]);
                    }
                if (sad < best) { best = sad; bdx += dx * 4; bdy += dy * 4; }
            }
    }
    *gx = bdx * 4; *gy = bdy * 4;
}
