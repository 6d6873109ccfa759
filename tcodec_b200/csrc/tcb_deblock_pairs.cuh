// tcb_deblock_pairs.cuh — the v2 in-loop deblocking of one 64x64 CTU
// (reference src/filter.c:23-237 tc_deblock_ctu, scalar path) on packed
// sample pairs (tcb_pair16.cuh), for the standalone frame kernel.
//
// The CTU is a shared-memory tile: luma rows of 64 bytes, Cb and Cr rows of
// 32.  Filtering an edge changes only p0 and q0, and the edges of one
// direction are 4 samples apart while a filter reads p1..q1, so all edges of
// one direction are independent; the kernel runs them as work items in any
// order, vertical before horizontal, luma and chroma side by side.  An item
// filters two edge positions at once, one per lane:
//
//   luma / Cb vertical  (row, edges 2j+1 and 2j+2 of the row): the four
//                       bytes around each edge come from the words at
//                       columns 8j, 8j+4, 8j+8; the item rewrites word 8j+4
//                       whole and the two bytes it owns in the other two
//                       (their other bytes belong to neighbouring items)
//   luma horizontal     (edge, four columns): one word from each of the
//                       rows y-2 .. y+1, two items per word pair of lanes
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

// Horizontal luma edge e (y = 4e), columns 4c..4c+3; rows 64 bytes apart.
__host__ __device__ __forceinline__ void deblock_luma_horiz_item(uint8_t *tile, int e, int c, DeblockQp q) {
    uint32_t *w = (uint32_t *)(tile + (4 * e - 2) * 64 + 4 * c);
    const uint32_t r0 = w[0], r1 = w[16], r2 = w[32], r3 = w[48];
    uint32_t p0a = pair_lo(r1), q0a = pair_lo(r2), p0b = pair_hi(r1), q0b = pair_hi(r2);
    deblock_luma_pair(pair_lo(r0), p0a, q0a, pair_lo(r3), q.t3, q.tc);
    deblock_luma_pair(pair_hi(r0), p0b, q0b, pair_hi(r3), q.t3, q.tc);
    w[16] = pair_pack(p0a, p0b);
    w[32] = pair_pack(q0a, q0b);
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

// Item counts of the two phases: vertical = 64 luma rows x 8 + 32 Cb rows
// x 4; horizontal = 15 luma edges x 16 + 7 chroma edges x 8.
constexpr int DEBLOCK_VERT_ITEMS = 64 * 8 + 32 * 4;
constexpr int DEBLOCK_HORIZ_ITEMS = 15 * 16 + 7 * 8;

__host__ __device__ __forceinline__ void deblock_vert(uint8_t *ty, uint8_t *tcb, int i, DeblockQp q) {
    if (i < 64 * 8) deblock_vert_item(ty + (i >> 3) * 64, 64, i & 7, true, q);
    else {
        i -= 64 * 8;
        deblock_vert_item(tcb + (i >> 2) * 32, 32, i & 3, false, q);
    }
}
__host__ __device__ __forceinline__ void deblock_horiz(uint8_t *ty, uint8_t *tcb, uint8_t *tcr, int i,
                                                     DeblockQp q) {
    if (i < 15 * 16) deblock_luma_horiz_item(ty, (i >> 4) + 1, i & 15, q);
    else {
        i -= 15 * 16;
        deblock_chroma_horiz_item(tcb, tcr, (i >> 3) + 1, i & 7, q);
    }
}

}  // namespace tcb
