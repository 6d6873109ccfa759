// tcb_legacy_types.h — records and frame parameters of the legacy (v0 / v1)
// 8x8 block path, shared by its kernels (tcb_legacy.cuh) and the host
// syntax writer and parser.
#pragma once
#include <stdint.h>

namespace tcb {
namespace legacy {

constexpr int BLOCKS = 64;            // 8x8 blocks per 64x64 CTU

// One block's decision record.  Encoder output (host syntax input):
// `mode` is the coded block mode (0 skip, 1 inter, 2 intra, 3 merge), `ref`
// the P-frame ref_idx or B-frame ref_sel, `tid` the transform id (bit 0
// DCT, bit 1 8x8), mvd the motion vector difference; luma levels in write
// order (four 4x4 sub-blocks of 16, or one 8x8 raster), then Cb and Cr.
// Decoder input (host parse output): the same fields with mvd_x / mvd_y
// holding the absolute motion vector.
struct LBlock {
    uint8_t coded, mode, intra_mode, ref, tid, pad0, pad1, pad2;
    int32_t mvd_x, mvd_y;
    int16_t luma[64];
    int16_t chroma[32];
};

// Frame parameters of one legacy CTU launch (device pointers).
struct LFrame {
    int W, H, sy, sc, ctu_cols, ctu_rows;
    const uint8_t *cur_y, *cur_cb, *cur_cr;      // source (encoder)
    uint8_t *rec_y, *rec_cb, *rec_cr;            // reconstruction
    // Motion-search candidates (encoder): P frames the first two occupied
    // DPB slots among those the preset allows, B frames forward / backward.
    const uint8_t *cand_y[2];
    int cand_sel[2], n_cand;
    const uint8_t *dpb_y[4];                     // P-frame references by slot (null: empty)
    const uint8_t *fwd_y, *bwd_y;                // B-frame references (null: none)
    int frame_type, qp, search_range;
    long long lambda;
    LBlock *blocks;                              // ctu_cols * ctu_rows * 64
};

}  // namespace legacy
}  // namespace tcb
