// tcb_common.cuh — types and constant tables shared by the host driver and
// the sm_100a kernels of the B200 TCodec v2 pixel pipeline.
//
// Every table here is a normative constant of the TCodec v2 bitstream or of
// its encoder decisions; its values must equal the reference's (file:line
// cited per table).  The DCT matrices are generated from their closed form
// (round(2^14 * s_k * cos((2n+1)k*pi/2N))) by the host and checked against
// the reference values in the oracle tests.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define TCB_HD __host__ __device__ __forceinline__
#else
#define TCB_HD inline
#endif

namespace tcb {

constexpr int CTU = 64;
constexpr int QT_NODES = 85;          // 1 + 4 + 16 + 64 quadtree nodes
constexpr int MAX_REFS = 4;           // DPB slots
constexpr int CTU_COEF_MAX = 64 * 64 + 2 * 32 * 32;   // luma + cb + cr
constexpr int MAX_STREAMS = 256;

// Per-CU decision record (reference tcodec_common.h:283-296 qt_node_t).
struct Node {
    uint8_t split, skip, merge, intra, bi, dct_size, intra_mode, intra_cmode,
            ref_sel;
    uint8_t ch_intra;
    int16_t mvd_x, mvd_y;
};

// 8x8-cell MV predictor grid entry (reference tcodec_common.h:281
// qt_mvcell_t): displacement in quarter-pel, intra = unavailable.
struct MvCell {
    int16_t dx, dy;
    uint8_t intra, pad;
};

// Output of one CTU for the host syntax writer: the decision tree, the
// quantized coefficients of every coded TU in write order, and the SAO
// parameters chosen after deblocking.
struct CtuOut {
    Node     nodes[QT_NODES];
    int32_t  ncoef;
    int16_t  sao_has, sao_band, sao_offset, pad;
    uint64_t tu8mask;                 // bit gy*8+gx: that 8x8 luma region uses one 8x8 TU
    int16_t  coef[CTU_COEF_MAX];
};

// One frame of one stream as the CTU engine sees it.  All plane pointers
// are device pointers; every plane of a stream shares stride_y / stride_c.
struct FrameParams {
    int W, H, stride_y, stride_c;
    int ctu_cols, ctu_rows;
    int grid_w, grid_h;                        // frame MV grid, 8x8 cells
    const uint8_t *cur_y, *cur_cb, *cur_cr;    // source picture
    uint8_t *rec_y, *rec_cb, *rec_cr;          // reconstruction (output)
    const uint8_t *ref_y[MAX_REFS], *ref_cb[MAX_REFS], *ref_cr[MAX_REFS];
    int ref_valid[MAX_REFS];
    int ref_poc[MAX_REFS];
    const MvCell *prev_grid;                   // previous frame's MV grid
    MvCell *cur_grid;                          // this frame's MV grid (out)
    CtuOut *out;                               // ctu_cols*ctu_rows records
    int frame_type;                            // 0 key, 1 P, 2 B
    int poc;
    int qp, qp_c;
    int preset;
    int multiref, fresh_skip;
    int prev_valid;
    int glob_valid, glob_x, glob_y;
    long long lambda;                          // luma RDO lambda
    int lambda_c;                              // chroma RDOQ lambda
    int lambda_sao;                            // SAO gate lambda
    int eff_l[4], eff_c[4];                    // per-band quant steps
    uint32_t rcp_l[4], rcp_c[4];               // exact reciprocals of eff
    int32_t *err;                              // device error word
    int *done;                                 // per-CTU publish flags (persistent wavefront)
    int epoch;                                 // value this frame publishes in `done`
    int search_window;                         // radius (2..5) of the search's SAD tables (engine tuning)
};

// ---------------------------------------------------------------------
// Normative tables.
// ---------------------------------------------------------------------

// QP -> quantizer step (reference src/quantize.c:30-39).
#define TCB_QSCALE_INIT { \
    1, 1, 1, 1, 1, 2, 2, 2, 3, 3, 4, 4, 5, 6, 7, 8, \
    9, 10, 12, 14, 16, 18, 21, 24, 28, 32, 37, 42, 49, 56, 64, 74, \
    85, 98, 112, 128, 149, 171, 197, 226, 256, 299, 343, 394, 453, 512, 598, 686, \
    788, 907, 1024, 1196, 1373, 1576, 1814, 2048, 2392, 2745, 3153, 3629, 4096, 4784, 5490, 6305 }

// JND band weights in eighths (reference src/quantize.c:72-77).
#define TCB_JND_INIT { 6, 7, 8, 10 }

TCB_HD int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
TCB_HD int absi(int v) { return v < 0 ? -v : v; }
TCB_HD int mini(int a, int b) { return a < b ? a : b; }
TCB_HD int maxi(int a, int b) { return a > b ? a : b; }

// Frequency band of a raster coefficient index (reference src/entropy.c:72-79).
TCB_HD int freq_band(int pos, int n) {
    return pos == 0 ? 0 : (pos < n / 4 ? 1 : (pos < n / 2 ? 2 : 3));
}

// Quadtree node index (reference tcodec_common.h:266-271).
TCB_HD int qt_index(int depth, int cx, int cy) {
    const int base = depth == 0 ? 0 : depth == 1 ? 1 : depth == 2 ? 5 : 21;
    const int shift = 3 - depth;
    return base + ((cy >> shift) << depth) + (cx >> shift);
}

// Dead-zone quantizer (reference tcodec_common.h:232-238) with the divide
// replaced by an exact reciprocal: for eff in [2, 2^13] and numerators
// below 2^16, umulhi(n, floor(2^32/eff) + 1) == n / eff (checked
// exhaustively by the oracle tests).  eff == 1 is the identity.
TCB_HD uint32_t quant_rcp(int eff) {
    return eff <= 1 ? 0u : (uint32_t)(0x100000000ull / (uint32_t)eff + 1ull);
}
TCB_HD int udiv_rcp(uint32_t n, int eff, uint32_t rcp) {
#ifdef __CUDA_ARCH__
    return eff <= 1 ? (int)n : (int)__umulhi(n, rcp);
#else
    return eff <= 1 ? (int)n : (int)(((uint64_t)n * rcp) >> 32);
#endif
}
TCB_HD int quant_coeff(int c, int eff, uint32_t rcp) {
    const int off = eff / 3;
    if (c > 0) return udiv_rcp((uint32_t)(c + off), eff, rcp);
    if (c < 0) return -udiv_rcp((uint32_t)(-c + off), eff, rcp);
    return 0;
}
// Centroid dequantizer (reference tcodec_common.h:240-246).
TCB_HD int dequant_coeff(int q, int eff) {
    const int bias = eff / 6;
    return q > 0 ? q * eff + bias : (q < 0 ? q * eff - bias : 0);
}

// Bit-length of a positive value (32 - clz).
TCB_HD int bitlen(unsigned v) {
#ifdef __CUDA_ARCH__
    return 32 - __clz((int)v);
#else
    return v ? 32 - __builtin_clz(v) : 0;
#endif
}

// Signed Exp-Golomb length (reference src/bitstream.c:95-107 tc_bs_se_bits).
TCB_HD int se_bits(int v) {
    unsigned m = v > 0 ? (unsigned)(2 * v - 1) : (v < 0 ? (unsigned)(-2 * v) : 0u);
    return 2 * bitlen(m + 1) - 1;
}

// Last-position cost of the bit model (reference src/encoder.c:377-385).
TCB_HD int lastpos_cost(int last) {
    if (last < 0) return 1;
    if (last < 4) return 1 + (last + 1) + 1;
    return 1 + 5 + (2 * bitlen((unsigned)(last - 4) + 1) - 1);
}

}  // namespace tcb
