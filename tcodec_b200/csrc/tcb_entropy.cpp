// tcb_entropy.cpp — host v2 syntax emission (see tcb_entropy.h).
#include <string.h>

#include "tcb_entropy.h"

namespace tcb {

// LPS probability per state and LPS state transition (reference
// src/range_coder.c:36-61) — normative tables of the bitstream.
const uint8_t kLpsProb[64] = {
    128, 124, 120, 116, 111, 106, 101, 96, 91, 86, 81, 76, 71, 66, 62, 58,
    54, 50, 46, 43, 39, 36, 33, 30, 27, 24, 22, 20, 18, 16, 14, 12,
    10, 9, 8, 7, 6, 5, 4, 4, 3, 3, 2, 2, 2, 1, 1, 1,
    1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1};
const uint8_t kNextLps[64] = {
    0, 0, 1, 2, 2, 4, 4, 5, 6, 7, 8, 9, 9, 11, 11, 12,
    13, 14, 15, 16, 16, 18, 18, 19, 19, 21, 21, 22, 22, 23, 23, 24,
    24, 25, 26, 26, 27, 27, 28, 28, 29, 29, 30, 30, 30, 31, 32, 32,
    33, 33, 33, 34, 34, 35, 35, 35, 36, 36, 36, 37, 37, 37, 38, 38};

// Zig-zag scans of the raw Exp-Golomb coefficient path (reference
// src/entropy.c:83-97).
static const uint8_t kZz4[16] = {0, 1, 4, 8, 5, 2, 3, 6, 9, 12, 13, 10, 7, 11, 14, 15};
static const uint8_t kZz8[64] = {
    0, 1, 8, 16, 9, 2, 3, 10, 17, 24, 32, 25, 18, 11, 4, 5,
    12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6, 7, 14, 21, 28,
    35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
    58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

void BitWriter::put_bits(uint32_t val, int nbits) {
    if (nbits <= 0) return;
    if (nbits < 32) val &= (1u << nbits) - 1;
    while (nbits > 0) {
        if (byte_pos >= cap) { overflow = true; return; }
        const int avail = 8 - bit_pos;
        const int w = nbits < avail ? nbits : avail;
        buf[byte_pos] |= (uint8_t)((val >> (nbits - w)) << (avail - w));
        bit_pos += w;
        nbits -= w;
        if (bit_pos == 8) {
            bit_pos = 0;
            ++byte_pos;
            if (byte_pos < cap) buf[byte_pos] = 0;
        }
    }
}

void BitWriter::put_ue(uint32_t v) {
    const uint32_t code = v + 1;
    int nb = 0;
    for (uint32_t t = code; t; t >>= 1) ++nb;
    put_bits(0, nb - 1);
    put_bits(code, nb);
}

void BitWriter::put_se(int32_t v) {
    put_ue(v > 0 ? (uint32_t)(2 * v - 1) : (v < 0 ? (uint32_t)(-2 * v) : 0u));
}

void RangeEncoder::shift() {
    const uint8_t top = (uint8_t)(low >> 24);
    if (top == 0xFF) {
        ++outstanding;
    } else {
        if (cache >= 0) bw->put_byte((uint8_t)cache);
        for (; outstanding > 0; --outstanding) bw->put_byte(0xFF);
        cache = top;
    }
    low <<= 8;
    range <<= 8;
}

void RangeEncoder::encode(uint8_t &ctx, int bit) {
    const int state = ctx & 0x3F, mps = (ctx >> 7) & 1;
    const uint32_t rlps = (range >> 8) * kLpsProb[state];
    if (bit == mps) {
        range -= rlps;
        if (state < 63) ctx = (uint8_t)((mps << 7) | (state + 1));
    } else {
        const uint32_t before = low;
        low += range - rlps;
        range = rlps;
        const int ns = kNextLps[state];
        ctx = (uint8_t)(((state == 0 ? (mps ^ 1) : mps) << 7) | ns);
        if (low < before) {   // carry into the pending bytes
            if (cache >= 0) {
                bw->put_byte((uint8_t)(cache + 1));
                for (; outstanding > 0; --outstanding) bw->put_byte(0x00);
            }
            cache = -1;
            outstanding = 0;
        }
    }
    while (range < (1u << 24)) shift();
}

void RangeEncoder::flush() {
    if (cache >= 0) bw->put_byte((uint8_t)cache);
    for (; outstanding > 0; --outstanding) bw->put_byte(0xFF);
    cache = -1;
    for (int i = 0; i < 5; ++i) {
        bw->put_byte((uint8_t)(low >> 24));
        low <<= 8;
    }
}

static inline int ctx_clip(int c) { return c >= CTX_MAX ? 75 : c; }

void SyntaxSink::bits(int base, uint32_t val, int nbits) {
    if (rc) {
        for (int i = 0; i < nbits; ++i)
            rc->encode(ctx[ctx_clip(base + i)], (int)((val >> (nbits - 1 - i)) & 1));
    } else {
        bw->put_bits(val, nbits);
    }
}

// Context-coded Exp-Golomb (reference src/range_coder.c:176-200).
void SyntaxSink::ue(int base, uint32_t val) {
    const uint32_t code = val + 1;
    int nb = 0;
    for (uint32_t t = code; t; t >>= 1) ++nb;
    const int lz = nb - 1;
    for (int i = 0; i < lz; ++i) rc->encode(ctx[ctx_clip(base + i)], 0);
    rc->encode(ctx[ctx_clip(base + lz)], 1);
    for (int i = 0; i < lz; ++i)
        rc->encode(ctx[ctx_clip(base + lz + 1 + i)], (int)((code >> (lz - 1 - i)) & 1));
}

void SyntaxSink::se(int base, int32_t val) {
    if (rc) ue(base, val > 0 ? (uint32_t)(2 * val - 1) : (val < 0 ? (uint32_t)(-2 * val) : 0u));
    else bw->put_se(val);
}

// Coefficient coding: context-modelled in raster order with a separate
// chroma bank (reference src/range_coder.c:204-300), or raw Exp-Golomb in
// zig-zag order (reference src/entropy.c:109-142).
void SyntaxSink::coeffs(const int16_t *c, int n, bool is4x4, bool chroma) {
    if (!rc) {
        const uint8_t *zz = is4x4 ? kZz4 : kZz8;
        int last = -1;
        for (int i = n - 1; i >= 0; --i)
            if (c[zz[i]]) { last = i; break; }
        bw->put_ue((uint32_t)(last + 1));
        for (int i = last; i >= 0; --i) {
            const int v = c[zz[i]], mag = v < 0 ? -v : v;
            bw->put_ue((uint32_t)mag);
            if (mag) bw->put_bits(v < 0 ? 1u : 0u, 1);
        }
        return;
    }
    const int co = chroma ? (CTX_CHROMA_BASE - CTX_SIG) : 0;
    int last = -1;
    for (int i = n - 1; i >= 0; --i)
        if (c[i]) { last = i; break; }
    if (last < 0) { rc->encode(ctx[CTX_LAST + co], 0); return; }
    rc->encode(ctx[CTX_LAST + co], 1);
    const int prefix = last < 4 ? last : 4;
    for (int i = 0; i < prefix; ++i) rc->encode(ctx[CTX_LAST + co + (i & 3)], 0);
    if (last < 4) rc->encode(ctx[CTX_LAST + co + (prefix & 3)], 1);
    else ue(CTX_LAST + co, (uint32_t)(last - 4));
    int gt1 = 0;
    for (int i = last; i >= 0; --i) {
        const int v = c[i];
        const bool dc = i == 0;
        const int band = n == 64 ? (i >> 3) : (n == 16 ? (i >> 1) : (i * 8 / n));
        int sig = dc ? CTX_SIG_DC + co : CTX_SIG + co + band;
        if (sig >= CTX_MAX) sig = CTX_MAX - 1;
        if (v == 0) { rc->encode(ctx[sig], 0); continue; }
        rc->encode(ctx[sig], 1);
        const int mag = v < 0 ? -v : v;
        const int c1 = dc ? CTX_GT1_DC + co : CTX_GT1 + co + (gt1 < 5 ? gt1 : 5);
        rc->encode(ctx[c1], mag > 1);
        if (mag > 1) {
            const int c2 = dc ? CTX_GT2_DC + co : CTX_GT2 + co + (gt1 < 1 ? gt1 : 1);
            rc->encode(ctx[c2], mag > 2);
            if (mag > 2) ue(dc ? CTX_LEVEL_DC + co : CTX_LEVEL + co, (uint32_t)(mag - 3));
            if (++gt1 > 5) gt1 = 5;
        }
        rc->encode(ctx[dc ? CTX_SIGN_DC + co : CTX_SIGN + co], v < 0);
    }
}

namespace {

struct Walker {
    SyntaxSink &s;
    const CtuOut &o;
    const CtuGeom &g;
    int pos = 0;

    void luma(int cu, int dct) {
        const int ntu = (cu / 8) * (cu / 8);
        for (int t = 0; t < ntu; ++t) {
            const int16_t *c = o.coef + pos + t * 64;
            if (dct) {
                s.bits(CTX_DCT_SIZE, 1, 1);
                s.coeffs(c, 64, false, false);
            } else {
                s.bits(CTX_DCT_SIZE, 0, 1);
                for (int q = 0; q < 4; ++q) {
                    s.bits(CTX_DCT_SIZE, 0, 1);
                    s.coeffs(c + q * 16, 16, true, false);
                }
            }
        }
        pos += cu * cu;
    }
    void chroma(int cu) {
        const int cs = cu / 2, nt = (cs / 4) * (cs / 4);
        for (int comp = 0; comp < 2; ++comp)
            for (int t = 0; t < nt; ++t)
                s.coeffs(o.coef + pos + comp * cs * cs + t * 16, 16, true, true);
        pos += 2 * cs * cs;
    }
    void node(int d, int cx, int cy) {
        const int cu = 64 >> d;
        const int px = g.ctu_x + cx * 8, py = g.ctu_y + cy * 8;
        const bool in_frame = px + cu <= g.W && py + cu <= g.H;
        const int h = 4 >> d;
        if (!in_frame && cu > 8) {
            for (int q = 0; q < 4; ++q) node(d + 1, cx + (q & 1) * h, cy + (q >> 1) * h);
            return;
        }
        if (!in_frame) return;
        const Node &n = o.nodes[qt_index(d, cx, cy)];
        s.bits(CTX_QT_SPLIT + d, n.split, 1);
        if (n.split) {
            for (int q = 0; q < 4; ++q) node(d + 1, cx + (q & 1) * h, cy + (q >> 1) * h);
            return;
        }
        s.bits(CTX_BLOCK_MODE, n.intra, 1);
        if (n.intra) {
            s.bits(CTX_INTRA_MODE, n.intra_mode, 5);
            s.bits(CTX_BLOCK_MODE, n.ch_intra, 1);
            if (n.ch_intra) s.bits(CTX_INTRA_MODE, n.intra_cmode, 3);
            luma(cu, n.dct_size);
            chroma(cu);
            return;
        }
        if (g.frame_type == 2) {
            s.bits(CTX_REF_SEL, n.ref_sel, 1);
            s.bits(CTX_BLOCK_MODE, n.bi, 1);
        }
        if (n.skip) {
            s.bits(CTX_SKIP_FLAG, 1, 1);
        } else if (n.merge) {
            s.bits(CTX_SKIP_FLAG, 0, 1);
            s.bits(CTX_MERGE_FLAG, 1, 1);
        } else {
            s.bits(CTX_SKIP_FLAG, 0, 1);
            s.bits(CTX_MERGE_FLAG, 0, 1);
            if (g.multiref && g.frame_type == 1) s.bits(CTX_REF_SEL, n.ref_sel & 3, 2);
            s.bits(CTX_DCT_SIZE, n.dct_size, 1);
            s.se(CTX_MVD_X, n.mvd_x);
            s.se(CTX_MVD_Y, n.mvd_y);
        }
        if (!n.skip) {
            luma(cu, n.dct_size);
            chroma(cu);
        }
    }
};

}  // namespace

void write_ctu_syntax(SyntaxSink &s, const CtuOut &o, const CtuGeom &g) {
    Walker w{s, o, g};
    w.node(0, 0, 0);
    s.bits(CTX_SAO_TYPE, (uint32_t)o.sao_has, 1);
    if (o.sao_has) {
        s.bits(CTX_SAO_BAND, (uint32_t)o.sao_band, 5);
        s.bits(CTX_SAO_OFFSET, (uint32_t)(o.sao_offset + 7), 4);
    }
}

// CRC-16/CCITT, init 0xFFFF, poly 0x1021 (reference src/bitstream.c:21-36).
void write_legacy_ctu(SyntaxSink &s, const legacy::LBlock *blocks, int frame_type) {
    for (int i = 0; i < legacy::BLOCKS; ++i) {
        const legacy::LBlock &b = blocks[i];
        if (!b.coded) continue;
        const bool intra = b.mode == 2, merge = b.mode == 3, skip = b.mode == 0;
        if (frame_type != 0) s.bits(CTX_BLOCK_MODE, b.mode, 2);
        if (frame_type == 2 && !intra) s.bits(CTX_REF_SEL, (uint32_t)(b.ref & 3), 2);
        if (intra) s.bits(CTX_INTRA_MODE, b.intra_mode, 5);
        if (!intra && !merge) {
            if (frame_type == 1) s.bits(CTX_REF_IDX, b.ref, 2);
            s.se(CTX_MVD_X, b.mvd_x);
            s.se(CTX_MVD_Y, b.mvd_y);
        }
        if (!merge && !skip) {
            s.bits(CTX_DCT_SIZE, b.tid, 2);
            if (b.tid & 2) s.coeffs(b.luma, 64, false, false);
            else for (int q = 0; q < 4; ++q) s.coeffs(b.luma + 16 * q, 16, true, false);
        }
        s.coeffs(b.chroma, 16, true, false);
        s.coeffs(b.chroma + 16, 16, true, false);
    }
}

LegacyFrameSyntax legacy_frame_syntax(const tc_config_t &cfg, int is_key, int frame_type, int qp, int poc,
                                      bool b_mode, bool wpp) {
    LegacyFrameSyntax h;
    h.version = cfg.bitstream_version == TC_VERSION_V0 ? 0 : 1;
    h.W = cfg.width; h.H = cfg.height;
    h.qp = qp; h.poc = poc; h.frame_type = frame_type;
    h.wpp = wpp;
    h.entropy = cfg.enable_entropy_coded != 0;
    int flags = is_key ? TC_FLAG_KEY_FRAME : 0;
    if (wpp) flags |= TC_FLAG_WPP;
    if (h.version != 0) {
        if (is_key) flags |= TC_FLAG_RAP;
        if (cfg.enable_crc) flags |= TC_FLAG_CRC;
        int profile = cfg.profile, level = cfg.level_idx;
        if (profile > TC_PROFILE_MAX) profile = TC_PROFILE_BASELINE_MOBILE;
        if (level > TC_LEVEL_MAX) level = TC_LEVEL_AUTO;
        h.profile_level = (profile << 4) | (level & 0x0F);
        int tools = TC_TOOL_SKIP_MERGE | TC_TOOL_CFL_CHROMA | TC_TOOL_JND_WEIGHTING | TC_TOOL_MEDIAN_MV_PRED |
                    TC_TOOL_SIX_TAP_INTERP;
        if (cfg.preset == TC_PRESET_SLOW && profile >= TC_PROFILE_STREAMING_MAIN) tools |= TC_TOOL_MULTI_REF;
        if (h.entropy) tools |= TC_TOOL_ENTROPY_CODED;
        if (frame_type == 2) tools |= TC_TOOL_BIPRED;
        h.tools = tools;
        h.crc = cfg.enable_crc != 0;
        if (b_mode) {
            flags |= TC_FLAG_EXT_HEADER;
            h.ext = frame_type == 0 ? 0 : (frame_type == 2 ? 2 : 1);
        }
    }
    h.flags = flags;
    return h;
}

size_t write_legacy_frame(uint8_t *buf, size_t cap, const LegacyFrameSyntax &h, const legacy::LBlock *blocks,
                          int ctu_cols, int ctu_rows, std::vector<uint8_t> &row_scratch) {
    memset(buf, 0, cap);
    BitWriter bw;
    bw.init(buf, cap);
    bw.put_bits(TC_MAGIC_0, 8); bw.put_bits(TC_MAGIC_1, 8); bw.put_bits(TC_MAGIC_2, 8);
    bw.put_bits((uint32_t)h.version, 8);
    bw.put_bits((uint32_t)(uint16_t)h.W, 16); bw.put_bits((uint32_t)(uint16_t)h.H, 16);
    bw.put_bits((uint32_t)h.flags, 8);
    bw.put_bits((uint8_t)(int8_t)(h.qp - TC_QP_DEFAULT), 8);
    bw.put_bits((uint8_t)(h.poc & 0xFF), 8);
    if (h.version == 0) {
        bw.put_bits(0, 8);
    } else {
        bw.put_bits((uint8_t)h.profile_level, 8);
        bw.put_bits((uint16_t)h.tools, 16);
        if (h.ext >= 0) bw.put_bits((uint32_t)h.ext, 8);
    }
    bw.align();
    const int per_ctu = legacy::BLOCKS;
    if (h.wpp) {
        // Entry table: rows - 1 offsets (16 bits each, relative to row 0),
        // then every row as its own byte-aligned run of raw syntax.
        const int noff = ctu_rows - 1;
        bw.put_bits((uint32_t)noff, 16);
        const size_t table = bw.byte_pos;
        for (int i = 0; i < noff; ++i) bw.put_bits(0, 16);
        bw.align();
        const size_t start = bw.byte_pos;
        const size_t per_row = cap / (size_t)(ctu_rows > 0 ? ctu_rows : 1) + 256;
        if (row_scratch.size() < per_row) row_scratch.resize(per_row);
        size_t offs[64];
        for (int r = 0; r < ctu_rows; ++r) {
            if (r < 64) offs[r] = bw.byte_pos - start;
            BitWriter rw;
            memset(row_scratch.data(), 0, per_row);
            rw.init(row_scratch.data(), per_row);
            SyntaxSink sink{&rw, nullptr, nullptr};
            for (int c = 0; c < ctu_cols; ++c)
                write_legacy_ctu(sink, blocks + (size_t)(r * ctu_cols + c) * per_ctu, h.frame_type);
            rw.align();
            if (rw.overflow) return 0;
            const size_t n = rw.bytes();
            if (bw.byte_pos + n > cap) return 0;
            memcpy(buf + bw.byte_pos, row_scratch.data(), n);
            bw.byte_pos += n;
            if (bw.byte_pos < cap) buf[bw.byte_pos] = 0;
        }
        for (int i = 0; i < noff && i + 1 < 64; ++i) {
            const uint16_t o = (uint16_t)offs[i + 1];
            buf[table + 2 * i] = (uint8_t)(o >> 8);
            buf[table + 2 * i + 1] = (uint8_t)(o & 0xFF);
        }
    } else {
        RangeEncoder rc;
        uint8_t ctx[TC_NUM_CONTEXTS_RC];
        memset(ctx, 0, sizeof(ctx));
        rc.init(&bw);
        SyntaxSink sink{&bw, h.entropy ? &rc : nullptr, ctx};
        for (int r = 0; r < ctu_rows; ++r)
            for (int c = 0; c < ctu_cols; ++c)
                write_legacy_ctu(sink, blocks + (size_t)(r * ctu_cols + c) * per_ctu, h.frame_type);
        if (h.entropy) rc.flush();
        bw.align();
    }
    if (h.version != 0 && h.crc) {
        const uint16_t crc = crc16_ccitt(buf, bw.bytes());
        bw.put_bits(crc >> 8, 8);
        bw.put_bits(crc & 0xFF, 8);
    }
    if (bw.overflow) return 0;
    return bw.bytes();
}

uint16_t crc16_ccitt(const uint8_t *data, size_t len) {
    uint16_t crc = 0xFFFF;
    for (size_t i = 0; i < len; ++i) {
        crc ^= (uint16_t)(data[i] << 8);
        for (int b = 0; b < 8; ++b) crc = (crc & 0x8000) ? (uint16_t)((crc << 1) ^ 0x1021) : (uint16_t)(crc << 1);
    }
    return crc;
}

}  // namespace tcb
