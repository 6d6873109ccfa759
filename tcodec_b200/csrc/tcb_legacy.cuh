// tcb_legacy.cuh — the legacy (v0 / v1) block path: one CTU of fixed 8x8
// blocks coded in raster order (reference src/encoder.c:1526-2269
// encode_block, src/decoder.c:260-650 decode_block).
//
// Each CTU is worked by one warp.  A block's 64 samples are spread over the
// lanes (two each); decisions that depend on a whole block (SADs, SSEs,
// non-zero counts) are warp reductions, and every lane then takes the same
// branch, so the sequential order of the reference (search candidates
// committed one at a time, blocks in raster order) is kept exactly.
//
// The functions are written against a small "team" interface (lane index,
// lane count, sum, sync) so that the same source also compiles as plain C++
// with a team of one lane: the CPU tests run it that way against the
// reference library (tests/legacy_emu.cpp).  The including translation unit
// provides ldct4(k, n) / ldct8(k, n), the DCT-II matrices.
#pragma once
#include <stdint.h>
#include "tcb_common.cuh"
#include "tcb_pixel.cuh"
#include "tcb_legacy_types.h"

namespace tcb {
namespace legacy {

#ifdef __CUDACC__
#define LG_FN __device__ __forceinline__
#define LG_TABLE static __constant__
#define LG_NOINL __device__ __noinline__
constexpr int NL = 32;
LG_FN int lane_id() { return threadIdx.x & 31; }
LG_FN int team_sum(int v) { return (int)__reduce_add_sync(0xffffffffu, (unsigned)v); }
LG_FN void team_sync() { __syncwarp(); }
LG_FN int popc(unsigned v) { return __popc(v); }
#else
#define LG_FN inline
#define LG_NOINL inline
#define LG_TABLE static const
constexpr int NL = 1;
inline int lane_id() { return 0; }
inline int team_sum(int v) { return v; }
inline void team_sync() {}
inline int popc(unsigned v) { return __builtin_popcount(v); }
#endif

constexpr int SAD_MAX = 0x7FFFFFFF;

// Per-CTU working state (shared memory on the device).
struct LState {
    uint8_t orig[64], pred[64], tpred[64], cpred[16];
    uint8_t rec[2][64];                 // candidate reconstructions per transform type
    uint8_t ra[20], rl[20];             // [0] corner, [1 + i] sample i (i = 0..16)
    int16_t resid[64];
    int16_t cand[2][64];                // quantized levels per transform type (8x8 raster)
    int16_t dq[64], inv[64];
    int32_t t32[64];
    int16_t cres[16];
    uint8_t blk_inter[64];              // block info of this CTU: 1 = not intra
    int32_t blk_mvx[64], blk_mvy[64];
};

// Normative tables (reference src/quantize.c:30-39, 72-77) and the search
// patterns of tc_motion_est (src/motion.c:346-369), centre points dropped.
LG_TABLE int lg_qscale[64] = TCB_QSCALE_INIT;
LG_TABLE int8_t lg_hexl[6][2] = {{-2, -4}, {2, -4}, {-4, 0}, {4, 0}, {-2, 4}, {2, 4}};
LG_TABLE int8_t lg_hexs[6][2] = {{-1, -2}, {1, -2}, {-2, 0}, {2, 0}, {-1, 2}, {1, 2}};
LG_TABLE int8_t lg_dia[4][2] = {{0, -1}, {-1, 0}, {1, 0}, {0, 1}};
LG_TABLE int8_t lg_qpel[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {-1, 1}, {1, -1}, {-1, -1}};
// Intra modes tried first (reference src/encoder.c:1563-1565).
LG_TABLE int8_t lg_fast_modes[8] = {0, 1, 2, 5, 8, 9, 13, 17};

LG_FN int qscale_of(int qp) { return lg_qscale[clampi(qp, 0, 63)]; }
LG_FN int jnd_of(int band) {
    return band <= 0 ? 6 : band == 1 ? 7 : band == 2 ? 8 : 10;
}
LG_FN int eff_of(int scale, int band) {
    const int e = (scale * jnd_of(band) + 4) >> 3;
    return e < 1 ? 1 : e;
}
// Legacy dead-zone quantizer and mid-point dequantizer
// (reference src/quantize.c:101-147, src/encoder.c:1858-1873).
LG_FN int lq_quant(int c, int eff) {
    const int off = eff / 3;
    return c > 0 ? (c + off) / eff : (c < 0 ? -((-c + off) / eff) : 0);
}
LG_FN int lq_dequant(int q, int eff) {
    return q > 0 ? q * eff + (eff >> 1) : (q < 0 ? q * eff - (eff >> 1) : 0);
}

// Element e (0..63) of an 8x8 area split into N x N transform blocks:
// transform block b, row r, column c within it, and the raster index of
// the sample in the 8x8 area.
LG_FN void elem_pos(int N, int e, int &b, int &r, int &c, int &ras) {
    if (N == 8) { b = 0; r = e >> 3; c = e & 7; ras = e; return; }
    b = e >> 4; r = (e >> 2) & 3; c = e & 3;
    ras = (((b >> 1) << 2) + r) * 8 + ((b & 1) << 2) + c;
}

// Transform matrix entry: kind 0 Walsh-Hadamard in the reference's
// butterfly order, (-1)^popcount(k & n) (reference src/transform.c:502-636);
// kind 1 the DCT-II matrix (src/transform.c:313-329).
LG_FN int tmat(int kind, int N, int k, int n) {
    if (kind == 0) return (popc((unsigned)(k & n)) & 1) ? -1 : 1;
    return N == 4 ? ldct4(k, n) : ldct8(k, n);
}

LG_FN int round14(long long acc) { return (int)((acc + (1 << 13)) >> 14); }

// Separable 2-D transform of the 8x8 area `in` (raster) into `out`, for
// every N x N block of it: rows first, then columns, each with the
// reference's rounding (WHT: exact rows, (x + N/2) >> log2 N on columns;
// DCT: 14-bit rounding after both passes).  `inverse` uses the transposed
// DCT matrix (the WHT is its own inverse).  Results are stored as the
// reference's int16 coefficients.
LG_FN void transform8(LState &S, const int16_t *in, int16_t *out, int N, int kind, bool inverse) {
    const int L = lane_id();
    for (int e = L; e < 64; e += NL) {
        int b, r, c, ras;
        elem_pos(N, e, b, r, c, ras);
        const int row0 = ras - c;                   // raster index of (r, 0) in this block
        long long acc = 0;
        for (int n = 0; n < N; ++n) {
            const int m = inverse && kind ? tmat(kind, N, n, c) : tmat(kind, N, c, n);
            acc += (long long)m * in[row0 + n];
        }
        S.t32[ras] = kind ? round14(acc) : (int)acc;   // t[r][k = c]
    }
    team_sync();
    for (int e = L; e < 64; e += NL) {
        int b, r, c, ras;
        elem_pos(N, e, b, r, c, ras);               // output (k = r, j = c)
        const int col0 = ras - r * 8;               // raster index of (0, c) in this block
        long long acc = 0;
        for (int i = 0; i < N; ++i) {
            const int m = inverse && kind ? tmat(kind, N, i, r) : tmat(kind, N, r, i);
            acc += (long long)m * S.t32[col0 + i * 8];
        }
        int v;
        if (kind) v = round14(acc);
        else v = N == 4 ? (int)((acc + 2) >> 2) : (int)((acc + 4) >> 3);
        out[ras] = (int16_t)v;
    }
    team_sync();
}

// Reference samples of an 8x8 block at (x, y) from the reconstruction
// (reference src/predict.c:23-110 tc_intra_get_ref, called with ra + 1 /
// rl + 1 as at src/encoder.c:1555-1558).
LG_FN void build_refs(LState &S, const uint8_t *rec, int s, int x, int y, int W, int H) {
    const int L = lane_id();
    const bool ha = y > 0, hl = x > 0;
    for (int j = L; j < 18; j += NL) {
        // ra[j]: j = 0 corner, 1..16 samples 0..15, 17 the guard
        int a, l;
        if (!ha && !hl) { a = 128; l = 128; }
        else {
            const uint8_t *arow = ha ? rec + (size_t)(y - 1) * s : rec;
            if (ha) {
                if (j == 0) a = hl ? arow[x - 1] : arow[x < W ? x : W - 1];
                else { const int i = j == 17 ? 15 : j - 1; const int px = x + i; a = arow[px < W ? px : W - 1]; }
            } else a = 128;
            if (hl) {
                if (j == 0) l = ha ? arow[x - 1] : rec[(size_t)(y < H ? y : H - 1) * s + x - 1];
                else { const int i = j == 17 ? 15 : j - 1; const int py = y + i; l = rec[(size_t)(py < H ? py : H - 1) * s + x - 1]; }
            } else l = 128;
        }
        S.ra[j] = (uint8_t)a;
        S.rl[j] = (uint8_t)l;
    }
    team_sync();
}

// DC value of the predictor (reference src/predict.c:140-165).
LG_FN int intra_dc_value(const LState &S) {
    int sum = 0;
    for (int i = 0; i < 8; ++i) sum += S.ra[2 + i] + S.rl[2 + i];
    return (sum + 8) / 16;
}

// SAD of the block against intra mode m.
LG_FN int intra_sad(const LState &S, int m, int dc) {
    const int L = lane_id();
    int s = 0;
    for (int i = L; i < 64; i += NL) s += absi((int)S.orig[i] - intra_at(S.ra + 1, S.rl + 1, 8, m, dc, i & 7, i >> 3));
    return team_sum(s);
}

// Integer SAD at (mx, my) with the reference's frame bounds check
// (reference src/motion.c:371-380).
LG_FN int sad_at(const LState &S, const uint8_t *ref, int s, int W, int H, int mx, int my) {
    if (mx < 0 || my < 0 || mx + 8 > W || my + 8 > H) return SAD_MAX;
    const int L = lane_id();
    int a = 0;
    for (int i = L; i < 64; i += NL) a += absi((int)S.orig[i] - (int)ref[(size_t)(my + (i >> 3)) * s + mx + (i & 7)]);
    return team_sum(a);
}

// Quarter-sample SAD of the refinement stage: six-tap where the margins
// allow, bilinear otherwise (reference src/motion.c:465-480, 308-341).
LG_FN int qpel_sad(const LState &S, const uint8_t *ref, int s, int W, int H, int qx, int qy) {
    const int fx = qx >> 2, fy = qy >> 2, dx = qx & 3, dy = qy & 3;
    const int L = lane_id();
    int a = 0;
    if (fx >= 2 && fy >= 2 && fx + 8 + 2 < W && fy + 8 + 2 < H) {
        for (int i = L; i < 64; i += NL) a += absi((int)S.orig[i] - luma_hv(ref, s, fx + (i & 7), fy + (i >> 3), dx, dy));
    } else {
        for (int i = L; i < 64; i += NL) {
            const uint8_t *p = ref + (size_t)(fy + (i >> 3)) * s + fx + (i & 7);
            const int top = interp_qpel(p[0], p[1], dx), bot = interp_qpel(p[s], p[s + 1], dx);
            a += absi((int)S.orig[i] - interp_qpel(top, bot, dy));
        }
    }
    return team_sum(a);
}

// Hexagonal search with sequential commit inside every pass, then the
// quarter-sample refinement (reference src/motion.c:384-485 tc_motion_est).
LG_FN void motion_est(const LState &S, const uint8_t *ref, int s, int W, int H, int cx, int cy, int range,
                      int &mvx, int &mvy, int &sad_out) {
    cx = clampi(cx, 0, W - 8);
    cy = clampi(cy, 0, H - 8);
    int bx = cx * 4, by = cy * 4;
    int best = sad_at(S, ref, s, W, H, cx, cy);
    const int step = maxi(1, range / 4);
    for (int it = 0; it < 2; ++it) {
        bool imp = false;
        for (int p = 0; p < 6; ++p) {
            const int mx = bx / 4 + lg_hexl[p][0] * step, my = by / 4 + lg_hexl[p][1] * step;
            const int v = sad_at(S, ref, s, W, H, mx, my);
            if (v < best) { best = v; bx = mx * 4; by = my * 4; imp = true; }
        }
        if (!imp) break;
    }
    for (int it = 0; it < 3; ++it) {
        bool imp = false;
        for (int p = 0; p < 6; ++p) {
            const int mx = bx / 4 + lg_hexs[p][0], my = by / 4 + lg_hexs[p][1];
            const int v = sad_at(S, ref, s, W, H, mx, my);
            if (v < best) { best = v; bx = mx * 4; by = my * 4; imp = true; }
        }
        if (!imp) break;
    }
    for (int it = 0; it < 4; ++it) {
        bool imp = false;
        for (int p = 0; p < 4; ++p) {
            const int mx = bx / 4 + lg_dia[p][0], my = by / 4 + lg_dia[p][1];
            const int v = sad_at(S, ref, s, W, H, mx, my);
            if (v < best) { best = v; bx = mx * 4; by = my * 4; imp = true; }
        }
        if (!imp) break;
    }
    for (int p = 0; p < 8; ++p) {
        const int qx = bx + lg_qpel[p][0], qy = by + lg_qpel[p][1];
        const int fx = qx >> 2, fy = qy >> 2;
        if (fx < 0 || fy < 0 || fx + 9 > W || fy + 9 > H) continue;
        const int v = qpel_sad(S, ref, s, W, H, qx, qy);
        if (v < best) { best = v; bx = qx; by = qy; }
    }
    mvx = bx; mvy = by; sad_out = best;
}

// Luma motion compensation of the block into dst (reference
// src/motion.c:493-584 tc_inter_predict).
LG_FN void inter_pred(uint8_t *dst, const uint8_t *ref, int s, int W, int H, int mvx, int mvy) {
    LumaMC mc;
    mc.init(ref, s, W, H, mvx, mvy, 8);
    for (int i = lane_id(); i < 64; i += NL) dst[i] = (uint8_t)mc.at(i & 7, i >> 3);
}

// Average of the forward prediction at mv and the backward one at -mv
// into dst (reference src/encoder.c:1688-1706).
LG_FN void bi_pred(uint8_t *dst, const uint8_t *fwd, const uint8_t *bwd, int s, int W, int H, int mvx, int mvy) {
    LumaMC a, b;
    a.init(fwd, s, W, H, mvx, mvy, 8);
    b.init(bwd, s, W, H, -mvx, -mvy, 8);
    for (int i = lane_id(); i < 64; i += NL) dst[i] = (uint8_t)((a.at(i & 7, i >> 3) + b.at(i & 7, i >> 3) + 1) >> 1);
}

LG_FN int sad_buf(const LState &S, const uint8_t *p) {
    int a = 0;
    for (int i = lane_id(); i < 64; i += NL) a += absi((int)S.orig[i] - (int)p[i]);
    return team_sum(a);
}

// Median motion predictor of block `bi` from its left, above and
// above-right neighbours inside the CTU (reference src/encoder.c:1619-1645,
// src/decoder.c:346-372).  Returns whether one of them is inter.
LG_FN bool median_mv(const LState &S, int bi, int &px, int &py) {
    const int bx = bi & 7, by = bi >> 3;
    int ax = 0, ay = 0, bxv = 0, byv = 0, cxv = 0, cyv = 0;
    bool ha = false, hb = false, hc = false;
    if (bx > 0 && S.blk_inter[bi - 1]) { ax = S.blk_mvx[bi - 1]; ay = S.blk_mvy[bi - 1]; ha = true; }
    if (by > 0 && S.blk_inter[bi - 8]) { bxv = S.blk_mvx[bi - 8]; byv = S.blk_mvy[bi - 8]; hb = true; }
    if (by > 0 && bx < 7 && S.blk_inter[bi - 7]) { cxv = S.blk_mvx[bi - 7]; cyv = S.blk_mvy[bi - 7]; hc = true; }
    if (!(ha || hb || hc)) return false;
    if (!ha) { ax = hb ? bxv : cxv; ay = hb ? byv : cyv; }
    if (!hb) { bxv = ha ? ax : cxv; byv = ha ? ay : cyv; }
    if (!hc) { cxv = ha ? ax : bxv; cyv = ha ? ay : byv; }
    auto med = [](int a, int b, int c) {
        if (a > b) { int t = a; a = b; b = t; }
        if (b > c) { int t = b; b = c; c = t; }
        if (a > b) { int t = a; a = b; b = t; }
        return b;
    };
    px = med(ax, bxv, cxv);
    py = med(ay, byv, cyv);
    return true;
}

// Chroma of one block (reference src/encoder.c:2192-2268, decoder.c:553-638):
// CfL blend of the chroma DC with the reconstructed luma for intra blocks,
// 128 otherwise; 4x4 WHT residual quantized at QP + 1 with the DC band's
// weight for every coefficient.  Encoder (enc = true) quantizes the
// residual of `orig` into `lv`; the decoder reads `lv`.  Writes the
// reconstruction.
LG_FN void chroma_block(LState &S, const LFrame &F, bool enc, const uint8_t *orig_c, uint8_t *rec_c,
                        int fx, int fy, bool intra, int16_t *lv) {
    const int cx = fx / 2, cy = fy / 2, s = F.sc;
    const int L = lane_id();
    if (intra) {
        int lsum = 0;
        for (int i = 0; i < 16; ++i) lsum += F.rec_y[(size_t)(fy + (i >> 2)) * F.sy + fx + (i & 3)];
        const int lavg = lsum / 16;
        int csum = 0, cnt = 0;
        if (cy > 0) for (int c = 0; c < 4; ++c) { csum += rec_c[(size_t)(cy - 1) * s + cx + c]; ++cnt; }
        if (cx > 0) for (int r = 0; r < 4; ++r) { csum += rec_c[(size_t)(cy + r) * s + cx - 1]; ++cnt; }
        const int cdc = cnt > 0 ? (csum + cnt / 2) / cnt : 128;
        for (int i = L; i < 16; i += NL) {
            const int lv_ = F.rec_y[(size_t)(fy + (i >> 2)) * F.sy + fx + (i & 3)];
            S.cpred[i] = (uint8_t)clampi(cdc + ((lv_ - lavg) >> 3), 0, 255);
        }
    } else {
        for (int i = L; i < 16; i += NL) S.cpred[i] = 128;
    }
    team_sync();
    const int eff = eff_of(qscale_of(clampi(F.qp + 1, 0, 63)), 0);
    // 4x4 WHT as the 8x8-area helper's first block: the area is padded with
    // zeros, and only block 0 (raster rows 0..3, columns 0..3) is used.
    for (int e = L; e < 64; e += NL) {
        const int r = e >> 3, c = e & 7;
        int16_t v = 0;
        if (enc && r < 4 && c < 4) v = (int16_t)((int)orig_c[(size_t)(cy + r) * s + cx + c] - (int)S.cpred[r * 4 + c]);
        S.resid[e] = v;
    }
    team_sync();
    if (enc) {
        transform8(S, S.resid, S.inv, 4, 0, false);
        for (int i = L; i < 16; i += NL) lv[i] = (int16_t)lq_quant(S.inv[(i >> 2) * 8 + (i & 3)], eff);
        team_sync();
    }
    for (int e = L; e < 64; e += NL) {
        const int r = e >> 3, c = e & 7;
        S.dq[e] = (r < 4 && c < 4) ? (int16_t)lq_dequant(lv[r * 4 + c], eff) : (int16_t)0;
    }
    team_sync();
    transform8(S, S.dq, S.inv, 4, 0, true);
    const int cw = F.W / 2, ch = F.H / 2;
    for (int i = L; i < 16; i += NL) {
        const int r = i >> 2, c = i & 3;
        if (cx + c < cw && cy + r < ch)
            rec_c[(size_t)(cy + r) * s + cx + c] = (uint8_t)clampi((int)S.cpred[i] + S.inv[r * 8 + c], 0, 255);
    }
    team_sync();
}

// Deblocking of a whole CTU's internal edges (reference src/filter.c:175-237
// tc_deblock_ctu).  Every filtered edge only moves p0 / q0 (the strength is
// never above 2), and the samples one edge writes are never read by another
// edge of the same pass, so each pass runs all its edges at once.
LG_FN void deblock_ctu(const LFrame &F, int ox, int oy) {
    const int L = lane_id(), qp = F.qp, s = F.sy;
    const int tcl = clampi(qp / 3, 1, 10);
    for (int it = L; it < 64 * 15; it += NL) {           // vertical luma edges: row x edge
        const int row = it / 15, x = ox + (it % 15 + 1) * 4;
        uint8_t *p = F.rec_y + (size_t)(oy + row) * s + x;
        const int p1 = p[-2], p0 = p[-1], q0 = p[0], q1 = p[1];
        if (edge_strength(p0, q0, qp) == 0) continue;
        p[-1] = (uint8_t)weak_filter(p1, p0, q0, q1, tcl);
        p[0] = (uint8_t)weak_filter(q1, q0, p0, p1, tcl);
    }
    team_sync();
    for (int it = L; it < 64 * 15; it += NL) {           // horizontal luma edges: column x edge
        const int col = it / 15, y = oy + (it % 15 + 1) * 4;
        uint8_t *p = F.rec_y + (size_t)y * s + ox + col;
        const int p1 = p[-2 * s], p0 = p[-s], q0 = p[0], q1 = p[s];
        if (edge_strength(p0, q0, qp) == 0) continue;
        p[-s] = (uint8_t)weak_filter(p1, p0, q0, q1, tcl);
        p[0] = (uint8_t)weak_filter(q1, q0, p0, p1, tcl);
    }
    team_sync();
    const int cqp = clampi(qp - 1, 0, 63), tcc = clampi(cqp / 4, 1, 6), sc = F.sc;
    for (int it = L; it < 32 * 7; it += NL) {            // vertical chroma edges (Cb only)
        const int row = it / 7, x = ox / 2 + (it % 7 + 1) * 4;
        uint8_t *p = F.rec_cb + (size_t)(oy / 2 + row) * sc + x;
        const int p0 = p[-1], q0 = p[0];
        if (edge_strength(p0, q0, cqp) == 0) continue;
        const int d = clampi((q0 - p0 + 1) >> 1, -tcc, tcc);
        p[-1] = (uint8_t)clampi(p0 + d, 0, 255);
        p[0] = (uint8_t)clampi(q0 - d, 0, 255);
    }
    team_sync();
    for (int it = L; it < 32 * 7; it += NL) {            // horizontal chroma edges (Cr's strength for both)
        const int col = it / 7, y = oy / 2 + (it % 7 + 1) * 4, x = ox / 2 + col;
        uint8_t *r = F.rec_cr + (size_t)y * sc + x, *b = F.rec_cb + (size_t)y * sc + x;
        const int p0 = r[0], q0 = r[sc], pb = b[0], qb = b[sc];
        if (edge_strength(p0, q0, cqp) == 0) continue;
        int d = clampi((q0 - p0 + 1) >> 1, -tcc, tcc);
        r[0] = (uint8_t)clampi(p0 + d, 0, 255);
        r[sc] = (uint8_t)clampi(q0 - d, 0, 255);
        d = clampi((qb - pb + 1) >> 1, -tcc, tcc);
        b[0] = (uint8_t)clampi(pb + d, 0, 255);
        b[sc] = (uint8_t)clampi(qb - d, 0, 255);
    }
    team_sync();
}

// Evaluate one transform type for the residual: forward transform,
// quantization with the JND band weights, dequantization, inverse, pixel
// SSE (reference src/encoder.c:1843-1925).  Leaves levels in S.cand[t] and
// the reconstruction in S.rec[t]; returns the non-zero count and adds the SSE.
LG_FN int eval_transform(LState &S, int N, int t, int scale, int &dist) {
    const int L = lane_id();
    transform8(S, S.resid, S.inv, N, t, false);
    int nz = 0;
    for (int e = L; e < 64; e += NL) {
        int b, r, c, ras;
        elem_pos(N, e, b, r, c, ras);
        const int eff = eff_of(scale, freq_band(r * N + c, N * N));
        const int q = (int16_t)lq_quant(S.inv[ras], eff);
        S.cand[t][ras] = (int16_t)q;
        nz += q != 0;
        S.dq[ras] = (int16_t)lq_dequant(q, eff);
    }
    team_sync();
    transform8(S, S.dq, S.inv, N, t, true);
    int d = 0;
    for (int i = L; i < 64; i += NL) {
        const int v = clampi((int)S.pred[i] + S.inv[i], 0, 255);
        S.rec[t][i] = (uint8_t)v;
        const int e = (int)S.orig[i] - v;
        d += e * e;
    }
    dist = team_sum(d);
    return team_sum(nz);
}

// Encode one 8x8 block (reference src/encoder.c:1526-2269 encode_block).
LG_NOINL void encode_block(LState &S, const LFrame &F, int bi, int fx, int fy, LBlock &out) {
    const int L = lane_id(), sy = F.sy, W = F.W, H = F.H;
    const int ftype = F.frame_type, qp = F.qp;
    for (int i = L; i < 64; i += NL) S.orig[i] = F.cur_y[(size_t)(fy + (i >> 3)) * sy + fx + (i & 7)];
    build_refs(S, F.rec_y, sy, fx, fy, W, H);   // syncs (orig visible too)
    // ---- intra search: eight fast modes, the rest when none is good
    const int dc = intra_dc_value(S);
    int best_intra = 1, best_isad = SAD_MAX;
    for (int k = 0; k < 8; ++k) {
        const int v = intra_sad(S, lg_fast_modes[k], dc);
        if (v < best_isad) { best_isad = v; best_intra = lg_fast_modes[k]; }
    }
    if (best_isad > 256)
        for (int m = 0; m < 18; ++m) {
            if (m == 0 || m == 1 || m == 2 || m == 5 || m == 8 || m == 9 || m == 13 || m == 17) continue;
            const int v = intra_sad(S, m, dc);
            if (v < best_isad) { best_isad = v; best_intra = m; }
        }
    for (int i = L; i < 64; i += NL) S.pred[i] = (uint8_t)intra_at(S.ra + 1, S.rl + 1, 8, best_intra, dc, i & 7, i >> 3);
    bool is_intra = true;
    int mvx = 0, mvy = 0, ref_idx = 0;
    // ---- inter search
    int best_sad = SAD_MAX, bmx = 0, bmy = 0, bref = 0;
    int mgx = fx * 4, mgy = fy * 4, merge_sad = SAD_MAX, merge_sel = 0;
    bool merge_ok = false;
    if (ftype != 0 && best_isad > 32) {
        if (bi > 0) merge_ok = median_mv(S, bi, mgx, mgy);
        for (int ci = 0; ci < F.n_cand; ++ci) {
            int mx, my, sd;
            motion_est(S, F.cand_y[ci], sy, W, H, mgx / 4, mgy / 4, F.search_range, mx, my, sd);
            if (sd < best_sad) { best_sad = sd; bmx = mx; bmy = my; bref = F.cand_sel[ci]; }
        }
        if (ftype == 2 && F.n_cand == 2) {
            bi_pred(S.tpred, F.cand_y[0], F.cand_y[1], sy, W, H, bmx, bmy);
            team_sync();
            const int v = sad_buf(S, S.tpred);
            if (v < best_sad) { best_sad = v; bref = 2; }
        }
        team_sync();
        if (best_sad < best_isad) {
            const uint8_t *src = nullptr;
            bool bi_avg = false;
            if (ftype == 2 && bref == 2) bi_avg = F.fwd_y && F.bwd_y;
            else if (ftype == 2) src = bref ? F.bwd_y : F.fwd_y;
            else src = F.dpb_y[bref];
            if (bi_avg || src || (ftype == 2 && bref == 2)) {
                if (bi_avg) bi_pred(S.pred, F.fwd_y, F.bwd_y, sy, W, H, bmx, bmy);
                else if (src) inter_pred(S.pred, src, sy, W, H, bmx, bmy);
                // (B, ref_sel 2 without both references keeps the intra samples)
                is_intra = false; mvx = bmx; mvy = bmy; ref_idx = bref;
            }
        }
        team_sync();
        if (merge_ok) {
            for (int ci = 0; ci < F.n_cand; ++ci) {
                const int v = sad_at(S, F.cand_y[ci], sy, W, H, mgx >> 2, mgy >> 2);
                if (v < merge_sad) { merge_sad = v; merge_sel = F.cand_sel[ci]; }
            }
            if (ftype == 2 && F.n_cand == 2) {
                bi_pred(S.tpred, F.cand_y[0], F.cand_y[1], sy, W, H, mgx, mgy);
                team_sync();
                const int v = sad_buf(S, S.tpred);
                if (v < merge_sad) { merge_sad = v; merge_sel = 2; }
                team_sync();
            }
        }
    }
    // ---- residual, transform size by variance, WHT vs DCT by RD-lite cost
    int sum = 0, sq = 0;
    for (int i = L; i < 64; i += NL) {
        const int o = S.orig[i];
        S.resid[i] = (int16_t)(o - (int)S.pred[i]);
        sum += o; sq += o * o;
    }
    sum = team_sum(sum); sq = team_sum(sq);
    team_sync();
    const int mean = sum / 64, var = sq / 64 - mean * mean;
    const int N = var > 512 ? 4 : 8;
    const int scale = qscale_of(qp);
    int d0, d1;
    const int nz0 = eval_transform(S, N, 0, scale, d0);
    const int nz1 = eval_transform(S, N, 1, scale, d1);
    const long long c0 = (long long)d0 + F.lambda * (4LL * nz0 + 2);
    const long long c1 = (long long)d1 + F.lambda * (4LL * nz1 + 2);
    const int tt = c1 < c0 ? 1 : 0;
    const int best_nz = tt ? nz1 : nz0;
    const bool all_zero = best_nz == 0;
    const int tid = (N == 8 ? 2 : 0) | tt;
    // ---- mode decision: merge > skip > inter > intra
    bool is_merge = false, is_skip = false;
    if (!is_intra && ftype != 0) {
        if (all_zero && merge_ok && merge_sad < qp * qp) is_merge = true;
        else if (all_zero) is_skip = true;
        else if (best_sad < qp * qp / 2) is_skip = true;
    }
    if (is_merge) {
        if (ftype == 2 && merge_sel == 2) {
            if (F.fwd_y && F.bwd_y) bi_pred(S.pred, F.fwd_y, F.bwd_y, sy, W, H, mgx, mgy);
            else for (int i = L; i < 64; i += NL) S.pred[i] = 128;
        } else {
            const uint8_t *src = ftype == 2 ? (merge_sel ? F.bwd_y : F.fwd_y) : F.dpb_y[0];
            if (src) inter_pred(S.pred, src, sy, W, H, mgx, mgy);
            else for (int i = L; i < 64; i += NL) S.pred[i] = 128;
        }
        is_intra = false; mvx = mgx; mvy = mgy; ref_idx = merge_sel;
        team_sync();
    }
    // ---- record
    if (L == 0) {
        out.coded = 1;
        out.mode = is_merge ? 3 : is_skip ? 0 : is_intra ? 2 : 1;
        out.intra_mode = (uint8_t)best_intra;
        out.ref = (uint8_t)ref_idx;
        out.tid = (uint8_t)tid;
        out.mvd_x = mvx - mgx;
        out.mvd_y = mvy - mgy;
    }
    const bool zero_res = is_merge || is_skip;
    for (int e = L; e < 64; e += NL) {
        int b, r, c, ras;
        elem_pos(N, e, b, r, c, ras);
        out.luma[e] = zero_res ? (int16_t)0 : S.cand[tt][ras];   // write order: block-major
    }
    // ---- reconstruction
    for (int i = L; i < 64; i += NL)
        F.rec_y[(size_t)(fy + (i >> 3)) * sy + fx + (i & 7)] = zero_res ? S.pred[i] : S.rec[tt][i];
    team_sync();
    // ---- chroma
    chroma_block(S, F, true, F.cur_cb, F.rec_cb, fx, fy, is_intra, out.chroma);
    chroma_block(S, F, true, F.cur_cr, F.rec_cr, fx, fy, is_intra, out.chroma + 16);
    if (L == 0) {
        S.blk_inter[bi] = is_intra ? 0 : 1;
        S.blk_mvx[bi] = mvx;
        S.blk_mvy[bi] = mvy;
    }
    team_sync();
}

// Reconstruct one 8x8 block from its parsed record (reference
// src/decoder.c:260-650 decode_block, after parsing).
LG_NOINL void decode_block(LState &S, const LFrame &F, int fx, int fy, const LBlock &in) {
    const int L = lane_id(), sy = F.sy, W = F.W, H = F.H, ftype = F.frame_type;
    const bool intra = in.mode == 2, skip = in.mode == 0 || in.mode == 3;
    if (intra) {
        build_refs(S, F.rec_y, sy, fx, fy, W, H);
        const int dc = intra_dc_value(S);
        for (int i = L; i < 64; i += NL) S.pred[i] = (uint8_t)intra_at(S.ra + 1, S.rl + 1, 8, in.intra_mode, dc, i & 7, i >> 3);
    } else {
        const int mvx = in.mvd_x, mvy = in.mvd_y;
        if (ftype == 2 && in.ref == 2) {
            if (F.fwd_y && F.bwd_y) bi_pred(S.pred, F.fwd_y, F.bwd_y, sy, W, H, mvx, mvy);
            else for (int i = L; i < 64; i += NL) S.pred[i] = 128;
        } else {
            const uint8_t *src = ftype == 2 ? (in.ref ? F.bwd_y : F.fwd_y) : F.dpb_y[in.ref & 3];
            if (src) inter_pred(S.pred, src, sy, W, H, mvx, mvy);
            else for (int i = L; i < 64; i += NL) S.pred[i] = 128;
        }
    }
    team_sync();
    if (skip) {
        for (int i = L; i < 64; i += NL) F.rec_y[(size_t)(fy + (i >> 3)) * sy + fx + (i & 7)] = S.pred[i];
    } else {
        const int N = (in.tid & 2) ? 8 : 4, t = in.tid & 1;
        const int scale = qscale_of(F.qp);
        for (int e = L; e < 64; e += NL) {
            int b, r, c, ras;
            elem_pos(N, e, b, r, c, ras);
            S.dq[ras] = (int16_t)lq_dequant(in.luma[e], eff_of(scale, freq_band(r * N + c, N * N)));
        }
        team_sync();
        transform8(S, S.dq, S.inv, N, t, true);
        for (int i = L; i < 64; i += NL)
            F.rec_y[(size_t)(fy + (i >> 3)) * sy + fx + (i & 7)] = (uint8_t)clampi((int)S.pred[i] + S.inv[i], 0, 255);
    }
    team_sync();
    const bool cfl = intra;   // intra blocks are never skip / merge
    int16_t lv[32];
    for (int i = 0; i < 32; ++i) lv[i] = in.chroma[i];
    chroma_block(S, F, false, nullptr, F.rec_cb, fx, fy, cfl, lv);
    chroma_block(S, F, false, nullptr, F.rec_cr, fx, fy, cfl, lv + 16);
}

// One CTU: its blocks in raster order, then deblocking when the CTU lies
// wholly inside the frame (reference src/encoder.c:2323-2346,
// src/decoder.c:656-683).
LG_FN void code_ctu(LState &S, const LFrame &F, int row, int col, bool enc) {
    const int L = lane_id();
    const int ox = col * 64, oy = row * 64;
    LBlock *blk = F.blocks + (size_t)(row * F.ctu_cols + col) * BLOCKS;
    if (enc) {
        // Blocks outside the frame keep the reference's zeroed block info:
        // not intra, motion vector (0, 0).
        for (int i = L; i < 64; i += NL) { S.blk_inter[i] = 1; S.blk_mvx[i] = 0; S.blk_mvy[i] = 0; }
        for (int i = L; i < 64; i += NL) blk[i].coded = 0;
        team_sync();
    }
    for (int b = 0; b < BLOCKS; ++b) {
        const int fx = ox + (b & 7) * 8, fy = oy + (b >> 3) * 8;
        if (fx + 8 > F.W || fy + 8 > F.H) continue;
        if (enc) encode_block(S, F, b, fx, fy, blk[b]);
        else if (blk[b].coded) decode_block(S, F, fx, fy, blk[b]);
    }
    if (ox + 64 <= F.W && oy + 64 <= F.H) deblock_ctu(F, ox, oy);
}

}  // namespace legacy
}  // namespace tcb
