// tcb_deblock_pairs.cuh — the v2 in-loop deblocking of one 64x64 CTU
// (reference src/filter.c:23-237 tc_deblock_ctu, scalar path) on packed
// sample pairs (tcb_pair16.cuh), for the standalone frame kernel.
//
// The CTU is a shared-memory tile: luma rows of 64 bytes, Cb and Cr rows of
// 32.  Filtering an edge changes only p0 and q0, and the edges of one
// direction are 4 samples apart while a filter reads p1..q1, so all edges of
// one direction are independent; the kernel runs them as work items in any
// order, vertical before horizontal, luma and chroma side by side.  Every
// filter call handles two edge positions at once, one per lane:
//
//   luma / Cb vertical  (edges 2j+1 and 2j+2 of a row): the four bytes
//                       around each edge come from the words at columns 8j,
//                       8j+4, 8j+8; the pair rewrites word 8j+4 whole and
//                       one byte of each of the other two.  The kernels take
//                       a whole row per item (deblock_vert_row: 16-byte
//                       loads and stores, the bytes merged in registers);
//                       deblock_vert keeps the single-pair items, which the
//                       CPU check runs against the rows
//   luma horizontal     (edge, 4 WPI columns): WPI words from each of the
//                       rows y-2 .. y+1, two pairs per word; the kernels
//                       use WPI = 4 (16-byte rows)
//   chroma horizontal   (edge, four columns): rows 4e and 4e+1 of Cr decide
//                       and filter Cr and Cb (the reference filters across
//                       the row pair 4e / 4e+1 for both planes)
//
// All functions are __host__ __device__ so the item order and the packed
// arithmetic can be checked against the oracle on the CPU.
#pragma once
#include <cstdint>

#include "tcb_pair16.cuh"

namespace tcb {

// 0xFFFF in the lanes where |p0 - q0| >= t (edge strength 0: the
// reference leaves the samples), 0 where the edge is filtered
// (reference src/filter.c:23-38: strength > 0 iff the difference is below
// the third threshold).  Lanes 0..255, t in 8..48.
__host__ __device__ __forceinline__ uint32_t deblock_keep(uint32_t p0, uint32_t q0, uint32_t t) {
    // |p0 - q0| per lane: the lanes' high bytes are 0 in both, so the
    // byte-wise absolute difference is the lane-wise one
#ifdef __CUDA_ARCH__
    const uint32_t diff = __vabsdiffu4(p0, q0);
#else
    const uint32_t diff = pair_max(p0, q0) - pair_min(p0, q0);
#endif
    const uint32_t ge = diff + (0x8000u - t) * 0x00010001u;   // bit 15 of a lane set iff diff >= t
    return pair_prmt(ge, 0, 0xBB99);                           // sign of each lane's high byte, replicated
}

// Luma weak filter (reference src/filter.c:49-57) of both sides of an edge:
// with A = 9 (q0 - p0) - 3 (q1 - p1), p0 + clamp((A + 8) >> 4, +-tc) and
// q0 - clamp((A + 7) >> 4, +-tc) (the reference's (8 - A) >> 4 for the q
// side, negated), both clamped to 0..255, in the lanes not kept.
// A is carried with a bias of 4096 (lanes 1044..7164) and the deltas and
// results with 256: a result clamped to 256..511 holds the sample in its
// low byte, and only the low bytes of p0 and q0 are used afterwards (bit 8
// of a filtered lane stays set).
__host__ __device__ __forceinline__ void deblock_luma_pair(uint32_t p1, uint32_t &p0, uint32_t &q0, uint32_t q1,
                                                         uint32_t t3, uint32_t tc) {
    const uint32_t one = 0x00010001u;
    const uint32_t s1 = q0 * 9u + p1 * 3u + (4096u + 8u) * one;
    const uint32_t s2 = p0 * 9u + q1 * 3u;
    const uint32_t a8 = s1 - s2;                                 // A + 8 + 4096
    const uint32_t lo = (256u - tc) * one, hi = (256u + tc) * one;
    const uint32_t dp = pair_min(pair_max((a8 >> 4) & 0x0FFF0FFFu, lo), hi);
    const uint32_t dq = pair_min(pair_max(((a8 - one) >> 4) & 0x0FFF0FFFu, lo), hi);
    const uint32_t b0 = 256u * one, b255 = 511u * one;
    const uint32_t np = pair_min(pair_max(p0 + dp, b0), b255);
    const uint32_t nq = pair_min(pair_max(q0 + 2u * b0 - dq, b0), b255);
    const uint32_t keep = deblock_keep(p0, q0, t3);
    p0 = (p0 & keep) | (np & ~keep);
    q0 = (q0 & keep) | (nq & ~keep);
}

// Chroma filter (reference src/filter.c:196-234): delta =
// clamp((q0 - p0 + 1) >> 1, +-tc), p0 + delta and q0 - delta clamped to
// 0..255, in the lanes not kept.  The delta and the results carry a bias of
// 256 as in the luma filter (sample in the low byte).
__host__ __device__ __forceinline__ void deblock_chroma_pair(uint32_t &p0, uint32_t &q0, uint32_t keep, uint32_t tc) {
    const uint32_t one = 0x00010001u, b0 = 256u * one, b255 = 511u * one;
    const uint32_t d = ((q0 + 513u * one - p0) >> 1) & 0x7FFF7FFFu;
    const uint32_t dc = pair_min(pair_max(d, (256u - tc) * one), (256u + tc) * one);
    const uint32_t np = pair_min(pair_max(p0 + dc, b0), b255);
    const uint32_t nq = pair_min(pair_max(q0 + 2u * b0 - dc, b0), b255);
    p0 = (p0 & keep) | (np & ~keep);
    q0 = (q0 & keep) | (nq & ~keep);
}

struct DeblockQp {
    uint32_t t3, tc, ct3, ctc;      // luma / chroma strength threshold and clip
    __host__ __device__ __forceinline__ void init(int qp) {
        const int cqp = qp < 1 ? 0 : (qp - 1 > 63 ? 63 : qp - 1);
        auto clamp = [](int v, int a, int b) { return v < a ? a : (v > b ? b : v); };
        t3 = (uint32_t)clamp(qp, 8, 48);
        tc = (uint32_t)clamp(qp / 3, 1, 10);
        ct3 = (uint32_t)clamp(cqp, 8, 48);
        ctc = (uint32_t)clamp(cqp / 4, 1, 6);
    }
};

// Vertical edges 2j+1 and 2j+2 (x = 8j+4, 8j+8) of one row of `row_bytes`
// (64 luma, 32 Cb); edge 2j+2 exists when 8j+8 < row_bytes.
__host__ __device__ __forceinline__ void deblock_vert_item(uint8_t *row, int row_bytes, int j, bool luma,
                                                         DeblockQp q) {
    const bool two = 8 * j + 8 < row_bytes;
    uint32_t *w = (uint32_t *)(row + 8 * j);
    const uint32_t wa = w[0], wb = w[1], wc = two ? w[2] : wb;
    const uint32_t lp = pair_prmt(wa, wb, 0x7632);            // (p1, p0) of both edges, interleaved
    const uint32_t lq = pair_prmt(wb, wc, 0x5410);            // (q0, q1)
    uint32_t p1 = lp & 0x00FF00FFu, p0 = (lp >> 8) & 0x00FF00FFu;
    uint32_t q0 = lq & 0x00FF00FFu, q1 = (lq >> 8) & 0x00FF00FFu;
    if (luma) deblock_luma_pair(p1, p0, q0, q1, q.t3, q.tc);
    else deblock_chroma_pair(p0, q0, deblock_keep(p0, q0, q.ct3), q.ctc);
    // p0 of edge 2j+1 -> byte 3 of word 8j; q0 of edge 2j+1 and p0 of edge
    // 2j+2 -> bytes 0 and 3 of word 8j+4; q0 of edge 2j+2 -> byte 0 of 8j+8.
    row[8 * j + 3] = (uint8_t)p0;
    if (two) {
        w[1] = pair_prmt(wb, pair_prmt(q0, p0, 0x6000), 0x7214);
        row[8 * j + 8] = (uint8_t)(q0 >> 16);
    } else {
        w[1] = pair_prmt(wb, q0, 0x3214);
    }
}

// Every vertical edge of one row of NW words (16: luma, 8: Cb), in
// registers: the row is read and written with 16-byte accesses, and the
// filtered bytes are merged into the words by byte permutes.  The inputs
// of every edge are taken from the unfiltered words (no edge reads a byte
// another edge writes), so this equals the items of the row in any order.
template <int NW>
__host__ __device__ __forceinline__ void deblock_vert_row(uint8_t *row, bool luma, DeblockQp q) {
    uint32_t w[NW], o[NW];
#pragma unroll
    for (int i = 0; i < NW / 4; ++i) {
        const uint4 v = ((const uint4 *)row)[i];
        w[4 * i] = v.x; w[4 * i + 1] = v.y; w[4 * i + 2] = v.z; w[4 * i + 3] = v.w;
    }
#pragma unroll
    for (int i = 0; i < NW; ++i) o[i] = w[i];
#pragma unroll
    for (int j = 0; j < NW / 2; ++j) {
        const bool two = 2 * j + 2 < NW;
        const uint32_t wa = w[2 * j], wb = w[2 * j + 1], wc = two ? w[2 * j + 2] : wb;
        const uint32_t lp = pair_prmt(wa, wb, 0x7632), lq = pair_prmt(wb, wc, 0x5410);
        uint32_t p1 = lp & 0x00FF00FFu, p0 = (lp >> 8) & 0x00FF00FFu;
        uint32_t q0 = lq & 0x00FF00FFu, q1 = (lq >> 8) & 0x00FF00FFu;
        if (luma) deblock_luma_pair(p1, p0, q0, q1, q.t3, q.tc);
        else deblock_chroma_pair(p0, q0, deblock_keep(p0, q0, q.ct3), q.ctc);
        o[2 * j] = pair_prmt(o[2 * j], p0, 0x4210);                       // byte 3 <- p0 of edge 2j+1
        if (two) {
            o[2 * j + 1] = pair_prmt(wb, pair_prmt(q0, p0, 0x6000), 0x7214);
            o[2 * j + 2] = pair_prmt(o[2 * j + 2], q0, 0x3216);           // byte 0 <- q0 of edge 2j+2
        } else {
            o[2 * j + 1] = pair_prmt(wb, q0, 0x3214);
        }
    }
#pragma unroll
    for (int i = 0; i < NW / 4; ++i) ((uint4 *)row)[i] = make_uint4(o[4 * i], o[4 * i + 1], o[4 * i + 2], o[4 * i + 3]);
}

// Rows of the vertical phase: 64 luma rows, then 32 Cb rows.
constexpr int DEBLOCK_VERT_ROWS = 64 + 32;
__host__ __device__ __forceinline__ void deblock_vert_rows(uint8_t *ty, uint8_t *tcb, int i, DeblockQp q) {
    if (i < 64) deblock_vert_row<16>(ty + i * 64, true, q);
    else deblock_vert_row<8>(tcb + (i - 64) * 32, false, q);
}

// Horizontal luma edge e, columns 4 WPI c .. 4 WPI c + 4 WPI - 1: the
// four rows around the edge read and the two filtered rows written as
// WPI-word vectors.
template <int WPI>
__host__ __device__ __forceinline__ void deblock_luma_horiz_wide(uint8_t *tile, int e, int c, DeblockQp q) {
    uint32_t r[4][WPI];
    uint8_t *base = tile + (4 * e - 2) * 64 + 4 * WPI * c;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if constexpr (WPI == 4) {
            const uint4 v = *(const uint4 *)(base + k * 64);
            r[k][0] = v.x; r[k][1] = v.y; r[k][2] = v.z; r[k][3] = v.w;
        } else if constexpr (WPI == 2) {
            const uint2 v = *(const uint2 *)(base + k * 64);
            r[k][0] = v.x; r[k][1] = v.y;
        } else {
            r[k][0] = *(const uint32_t *)(base + k * 64);
        }
    }
    uint32_t np[WPI], nq[WPI];
#pragma unroll
    for (int i = 0; i < WPI; ++i) {
        uint32_t p0a = pair_lo(r[1][i]), q0a = pair_lo(r[2][i]), p0b = pair_hi(r[1][i]), q0b = pair_hi(r[2][i]);
        deblock_luma_pair(pair_lo(r[0][i]), p0a, q0a, pair_lo(r[3][i]), q.t3, q.tc);
        deblock_luma_pair(pair_hi(r[0][i]), p0b, q0b, pair_hi(r[3][i]), q.t3, q.tc);
        np[i] = pair_pack(p0a, p0b);
        nq[i] = pair_pack(q0a, q0b);
    }
    if constexpr (WPI == 4) {
        *(uint4 *)(base + 64) = make_uint4(np[0], np[1], np[2], np[3]);
        *(uint4 *)(base + 128) = make_uint4(nq[0], nq[1], nq[2], nq[3]);
    } else if constexpr (WPI == 2) {
        *(uint2 *)(base + 64) = make_uint2(np[0], np[1]);
        *(uint2 *)(base + 128) = make_uint2(nq[0], nq[1]);
    } else {
        *(uint32_t *)(base + 64) = np[0];
        *(uint32_t *)(base + 128) = nq[0];
    }
}

// Horizontal chroma edge e (rows 4e and 4e + 1), columns 4c..4c+3 of both
// planes; Cr decides for both; rows 32 bytes apart.
__host__ __device__ __forceinline__ void deblock_chroma_horiz_item(uint8_t *cb, uint8_t *cr, int e, int c,
                                                                 DeblockQp q) {
    uint32_t *wr = (uint32_t *)(cr + 4 * e * 32 + 4 * c), *wb = (uint32_t *)(cb + 4 * e * 32 + 4 * c);
    const uint32_t r0 = wr[0], r1 = wr[8], b0 = wb[0], b1 = wb[8];
    uint32_t pa = pair_lo(r0), qa = pair_lo(r1), pb = pair_hi(r0), qb = pair_hi(r1);
    const uint32_t ka = deblock_keep(pa, qa, q.ct3), kb = deblock_keep(pb, qb, q.ct3);
    deblock_chroma_pair(pa, qa, ka, q.ctc);
    deblock_chroma_pair(pb, qb, kb, q.ctc);
    wr[0] = pair_pack(pa, pb);
    wr[8] = pair_pack(qa, qb);
    pa = pair_lo(b0); qa = pair_lo(b1); pb = pair_hi(b0); qb = pair_hi(b1);
    deblock_chroma_pair(pa, qa, ka, q.ctc);
    deblock_chroma_pair(pb, qb, kb, q.ctc);
    wb[0] = pair_pack(pa, pb);
    wb[8] = pair_pack(qa, qb);
}

// Items of the vertical phase: 64 luma rows x 8 + 32 Cb rows x 4.
constexpr int DEBLOCK_VERT_ITEMS = 64 * 8 + 32 * 4;

__host__ __device__ __forceinline__ void deblock_vert(uint8_t *ty, uint8_t *tcb, int i, DeblockQp q) {
    if (i < 64 * 8) deblock_vert_item(ty + (i >> 3) * 64, 64, i & 7, true, q);
    else {
        i -= 64 * 8;
        deblock_vert_item(tcb + (i >> 2) * 32, 32, i & 3, false, q);
    }
}
// The horizontal phase with luma items WPI words wide: 15 luma edges x
// 16 / WPI items, then the 7 x 8 chroma items.
template <int WPI>
constexpr int deblock_horiz_wide_items() { return 15 * (16 / WPI) + 7 * 8; }
template <int WPI>
__host__ __device__ __forceinline__ void deblock_horiz_wide(uint8_t *ty, uint8_t *tcb, uint8_t *tcr, int i,
                                                          DeblockQp q) {
    constexpr int PER = 16 / WPI;
    if (i < 15 * PER) deblock_luma_horiz_wide<WPI>(ty, i / PER + 1, i % PER, q);
    else {
        i -= 15 * PER;
        deblock_chroma_horiz_item(tcb, tcr, (i >> 3) + 1, i & 7, q);
    }
}

}  // namespace tcb
