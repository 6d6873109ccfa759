// tcb_entropy.h — host-side v2 syntax emission: MSB-first bit writer,
// Exp-Golomb codes, the 119-context binary range coder and the per-CTU
// syntax walk that turns the device's decision tree + coefficients into
// bytes.  Serial by design (one writer per stream or per entry-point row).
#pragma once
#include <stddef.h>
#include <stdint.h>
#include <vector>

#include "../../include/tcodec_types.h"
#include "tcb_common.cuh"
#include "tcb_legacy_types.h"

namespace tcb {

// Context indices of the v2 syntax (reference tcodec_common.h:377-405).
enum RcCtx {
    CTX_BLOCK_MODE = 0, CTX_SKIP_FLAG = 4, CTX_INTRA_MODE = 6, CTX_DCT_SIZE = 11,
    CTX_REF_IDX = 13, CTX_MVD_SIGN = 15, CTX_MVD_X = 17, CTX_MVD_Y = 19,
    CTX_SIG = 21, CTX_SIG_DC = 29, CTX_LAST = 30, CTX_LAST_DC = 34, CTX_GT1 = 35,
    CTX_GT1_DC = 41, CTX_GT2 = 42, CTX_GT2_DC = 44, CTX_SIGN = 45, CTX_SIGN_DC = 46,
    CTX_LEVEL = 47, CTX_LEVEL_DC = 53, CTX_REF_SEL = 59, CTX_MERGE_FLAG = 61,
    CTX_QT_SPLIT = 62, CTX_SAO_TYPE = 76, CTX_SAO_BAND = 77, CTX_SAO_OFFSET = 82,
    CTX_CHROMA_BASE = 86, CTX_MAX = 119
};

// Range-coder LPS probability per state and LPS state transition.
extern const uint8_t kLpsProb[64];
extern const uint8_t kNextLps[64];

// MSB-first bit writer over a caller-owned buffer (reference
// src/bitstream.c:40-136 semantics: bytes are zeroed as they are entered).
struct BitWriter {
    uint8_t *buf = nullptr;
    size_t cap = 0, byte_pos = 0;
    int bit_pos = 0;
    bool overflow = false;
    void init(uint8_t *b, size_t c) {
        buf = b; cap = c; byte_pos = 0; bit_pos = 0; overflow = false;
        if (cap) buf[0] = 0;
    }
    void put_bits(uint32_t val, int nbits);
    void put_byte(uint8_t v) {            // fast path when byte aligned
        if (bit_pos == 0) {
            if (byte_pos >= cap) { overflow = true; return; }
            buf[byte_pos++] = v;
            if (byte_pos < cap) buf[byte_pos] = 0;
        } else {
            put_bits(v, 8);
        }
    }
    void put_ue(uint32_t v);
    void put_se(int32_t v);
    void align() {
        if (bit_pos) { bit_pos = 0; ++byte_pos; if (byte_pos < cap) buf[byte_pos] = 0; }
    }
    size_t bytes() const { return byte_pos + (bit_pos ? 1 : 0); }
};

// Binary range coder with 64-state adaptive contexts, 32-bit low and
// cache/outstanding carry propagation (reference src/range_coder.c:77-220).
struct RangeEncoder {
    BitWriter *bw = nullptr;
    uint32_t low = 0, range = 0xFFFFFFFFu;
    int cache = -1, outstanding = 0;
    void init(BitWriter *w) { bw = w; low = 0; range = 0xFFFFFFFFu; cache = -1; outstanding = 0; }
    void encode(uint8_t &ctx, int bit);
    void flush();
  private:
    void shift();
};

// One v2 syntax sink: range coded (rc != nullptr) or raw bits.
struct SyntaxSink {
    BitWriter *bw;
    RangeEncoder *rc;
    uint8_t *ctx;
    void bits(int base_ctx, uint32_t val, int nbits);
    void ue(int base_ctx, uint32_t val);
    void se(int base_ctx, int32_t val);
    void coeffs(const int16_t *c, int n, bool is4x4, bool chroma);
};

struct CtuGeom {
    int ctu_x, ctu_y, W, H;
    int frame_type;   // 0 key, 1 P, 2 B
    int multiref;
};

// Emit the syntax of one CTU (reference src/encoder.c:587-653, 429-543
// write branches, 1494-1501).
void write_ctu_syntax(SyntaxSink &s, const CtuOut &o, const CtuGeom &g);

// Emit the legacy (v0 / v1) syntax of one CTU's 8x8 blocks in raster
// order (reference src/encoder.c:1996-2098 and 2186-2190): block mode,
// B-frame reference selection, intra mode, P-frame ref_idx and MVD,
// transform id and luma levels, then Cb and Cr levels.
void write_legacy_ctu(SyntaxSink &s, const legacy::LBlock *blocks, int frame_type);

// Frame-level fields of a legacy packet.
struct LegacyFrameSyntax {
    int version = 1;          // 0: 12-byte header; 1: profile / tools / extension byte
    int W = 0, H = 0, flags = 0, qp = 32, poc = 0, profile_level = 0, tools = 0;
    int ext = -1;             // frame-type code of the extension byte, -1: none
    int frame_type = 0;
    bool wpp = false, entropy = false, crc = false;
};
// Header fields of a legacy frame (reference src/encoder.c:2713-2819):
// `wpp` when the frame's rows are coded as separate byte-aligned runs.
LegacyFrameSyntax legacy_frame_syntax(const tc_config_t &cfg, int is_key, int frame_type, int qp, int poc,
                                      bool b_mode, bool wpp);
// The whole legacy packet (reference src/encoder.c:2365-2399 header,
// 2966-3067 rows: per-row byte-aligned runs behind a 16-bit entry table
// when `wpp`, else one run, range coded when `entropy`; CRC-16 when `crc`
// and the version is 1).  Returns the packet size, 0 when `cap` is too
// small.  `row_scratch` holds the per-row runs.
size_t write_legacy_frame(uint8_t *buf, size_t cap, const LegacyFrameSyntax &h, const legacy::LBlock *blocks,
                          int ctu_cols, int ctu_rows, std::vector<uint8_t> &row_scratch);

uint16_t crc16_ccitt(const uint8_t *data, size_t len);

}  // namespace tcb
