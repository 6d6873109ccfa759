// tcb_parse.h — host-side syntax parsing of both bitstreams: the MSB-first
// bit reader, the range decoder, the v2 CTU syntax parser and the legacy
// block parser, plus the frame header.  Used by the decoder
// (tcb_decoder.cpp) and by the CPU checks of the legacy path.
#pragma once
#include <stdint.h>
#include <string.h>

#include <algorithm>

#include "../../include/tcodec_types.h"
#include "tcb_common.cuh"
#include "tcb_entropy.h"
#include "tcb_legacy_types.h"

namespace tcb {
namespace parse {

// LPS tables of the range coder (reference src/range_coder.c:36-61).
const uint8_t kLps[64] = {
    128, 124, 120, 116, 111, 106, 101, 96, 91, 86, 81, 76, 71, 66, 62, 58,
    54, 50, 46, 43, 39, 36, 33, 30, 27, 24, 22, 20, 18, 16, 14, 12,
    10, 9, 8, 7, 6, 5, 4, 4, 3, 3, 2, 2, 2, 1, 1, 1,
    1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1};
const uint8_t kNext[64] = {
    0, 0, 1, 2, 2, 4, 4, 5, 6, 7, 8, 9, 9, 11, 11, 12,
    13, 14, 15, 16, 16, 18, 18, 19, 19, 21, 21, 22, 22, 23, 23, 24,
    24, 25, 26, 26, 27, 27, 28, 28, 29, 29, 30, 30, 30, 31, 32, 32,
    33, 33, 33, 34, 34, 35, 35, 35, 36, 36, 36, 37, 37, 37, 38, 38};
const uint8_t kZz4[16] = {0, 1, 4, 8, 5, 2, 3, 6, 9, 12, 13, 10, 7, 11, 14, 15};
const uint8_t kZz8[64] = {
    0, 1, 8, 16, 9, 2, 3, 10, 17, 24, 32, 25, 18, 11, 4, 5,
    12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6, 7, 14, 21, 28,
    35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
    58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};


// MSB-first reader; reads past the end set `error` (reference
// src/bitstream.c:140-200).
struct Reader {
    const uint8_t *buf = nullptr;
    size_t size = 0, pos = 0;
    int bit = 0, error = 0;
    void init(const uint8_t *b, size_t n) { buf = b; size = n; pos = 0; bit = 0; error = 0; }
    bool eof() const { return pos >= size; }
    uint32_t bits(int n) {
        uint32_t v = 0;
        while (n > 0) {
            if (pos >= size) { error = 1; return v; }
            const int avail = 8 - bit, take = n < avail ? n : avail;
            v = (v << take) | ((buf[pos] >> (avail - take)) & ((1u << take) - 1));
            bit += take;
            n -= take;
            if (bit == 8) { bit = 0; ++pos; }
        }
        return v;
    }
    uint32_t ue() {
        int lz = 0;
        bool one = false;
        while (pos < size) {
            if (bits(1)) { one = true; break; }
            if (++lz > 31) { error = 1; return 0; }
        }
        if (!one) { error = 1; return 0; }
        const uint32_t suf = lz ? bits(lz) : 0;
        return (1u << lz) - 1 + suf;
    }
    int32_t se() {
        const uint32_t m = ue();
        if (m == 0) return 0;
        return (m & 1) ? (int32_t)((m + 1) / 2) : -(int32_t)(m / 2);
    }
    void align() { if (bit) { bit = 0; ++pos; } }
};

// Range decoder (reference src/range_coder.c:303-400).
struct RDec {
    Reader *bs = nullptr;
    uint32_t low = 0, range = 0xFFFFFFFFu;
    uint32_t byte() {
        if (bs->bit == 0) return bs->pos < bs->size ? bs->buf[bs->pos++] : 0;
        if (bs->pos >= bs->size) return 0;
        return bs->bits(8);
    }
    void init(Reader *r) {
        bs = r; low = 0; range = 0xFFFFFFFFu;
        for (int i = 0; i < 4; ++i) low = bs->eof() ? (low << 8) : ((low << 8) | byte());
    }
    int bit(uint8_t &ctx) {
        const int state = ctx & 0x3F, mps = (ctx >> 7) & 1;
        const uint32_t rlps = (range >> 8) * kLps[state];
        int b;
        if (low < range - rlps) {
            range -= rlps;
            b = mps;
            if (state < 63) ctx = (uint8_t)((mps << 7) | (state + 1));
        } else {
            low -= range - rlps;
            range = rlps;
            b = mps ^ 1;
            ctx = (uint8_t)(((state == 0 ? (mps ^ 1) : mps) << 7) | kNext[state]);
        }
        while (range < (1u << 24)) {
            low = low << 8;
            range = range == 0 ? 0xFF : (range << 8);
            if (!bs->eof()) low |= byte();
        }
        return b;
    }
};

inline int cclip(int c) { return c >= CTX_MAX ? 75 : c; }

struct Parser {
    Reader *bs;
    RDec *rc;           // nullptr: raw Exp-Golomb syntax
    uint8_t *ctx;
    int W, H, frame_type, multiref_tool, sao_tool;
    const int *dpb_valid;
    CtuOut *o;
    int ctu_x, ctu_y, ncoef;

    uint32_t bits(int base, int n) {
        if (!rc) return bs->bits(n);
        uint32_t v = 0;
        for (int i = 0; i < n; ++i) v = (v << 1) | (uint32_t)rc->bit(ctx[cclip(base + i)]);
        return v;
    }
    uint32_t ue(int base) {
        int lz = 0;
        while (true) {
            if (rc->bit(ctx[cclip(base + lz)]) == 1) break;
            if (++lz > 31) return 0;
        }
        uint32_t suf = 0;
        for (int i = 0; i < lz; ++i) suf = (suf << 1) | (uint32_t)rc->bit(ctx[cclip(base + lz + 1 + i)]);
        return (1u << lz) - 1 + suf;
    }
    int32_t se(int base) {
        if (!rc) return bs->se();
        const uint32_t m = ue(base);
        if (m == 0) return 0;
        return (m & 1) ? (int32_t)((m + 1) >> 1) : -(int32_t)(m >> 1);
    }
    // Coefficients (reference src/range_coder.c:402-488, src/entropy.c:144-183).
    void coeffs(int16_t *c, int n, bool is4x4, bool chroma) {
        memset(c, 0, sizeof(int16_t) * n);
        if (!rc) {
            const uint8_t *zz = is4x4 ? kZz4 : kZz8;
            const uint32_t lp1 = bs->ue();
            if (lp1 == 0) return;
            if (lp1 > (uint32_t)n) { bs->error = 1; return; }
            for (int i = (int)lp1 - 1; i >= 0; --i) {
                const uint32_t mag = bs->ue();
                if (mag > 0) {
                    if (mag > 32767u) { bs->error = 1; return; }
                    const uint32_t sign = bs->bits(1);
                    c[zz[i]] = (int16_t)(sign ? -(int)mag : (int)mag);
                }
            }
            return;
        }
        const int co = chroma ? (CTX_CHROMA_BASE - CTX_SIG) : 0;
        if (rc->bit(ctx[CTX_LAST + co]) == 0) return;
        int last = 0;
        bool found = false;
        for (int i = 0; i < 4; ++i)
            if (rc->bit(ctx[CTX_LAST + co + (i & 3)]) == 1) { last = i; found = true; break; }
        if (!found) {
            const uint32_t extra = ue(CTX_LAST + co);
            if (extra > (uint32_t)n) { bs->error = 1; return; }
            last = 4 + (int)extra;
        }
        if (last < 0 || last >= n) { bs->error = 1; return; }
        int gt1 = 0;
        for (int i = last; i >= 0; --i) {
            const bool dc = i == 0;
            const int band = n == 64 ? (i >> 3) : (n == 16 ? (i >> 1) : (i * 8 / n));
            int sig = dc ? CTX_SIG_DC + co : CTX_SIG + co + band;
            if (sig >= CTX_MAX) sig = CTX_MAX - 1;
            if (!rc->bit(ctx[sig])) { c[i] = 0; continue; }
            const int g1 = rc->bit(ctx[dc ? CTX_GT1_DC + co : CTX_GT1 + co + (gt1 < 5 ? gt1 : 5)]);
            int mag;
            if (!g1) {
                mag = 1;
            } else {
                const int g2 = rc->bit(ctx[dc ? CTX_GT2_DC + co : CTX_GT2 + co + (gt1 < 1 ? gt1 : 1)]);
                mag = g2 ? 3 + (int)ue(dc ? CTX_LEVEL_DC + co : CTX_LEVEL + co) : 2;
                if (++gt1 > 5) gt1 = 5;
            }
            if (mag > 32767) { bs->error = 1; return; }
            const int s = rc->bit(ctx[dc ? CTX_SIGN_DC + co : CTX_SIGN + co]);
            c[i] = (int16_t)(s ? -mag : mag);
        }
    }
    bool room(int n) {
        if (ncoef + n > CTU_COEF_MAX) { bs->error = 1; return false; }
        return true;
    }
    void luma(int cu, int cx, int cy) {
        const int ntu = cu / 8;
        for (int ty = 0; ty < ntu; ++ty)
            for (int tx = 0; tx < ntu; ++tx) {
                const uint32_t dct = bits(CTX_DCT_SIZE, 1);
                if (!room(64)) return;
                if (dct) {
                    o->tu8mask |= 1ull << ((cy + ty) * 8 + cx + tx);
                    coeffs(o->coef + ncoef, 64, false, false);
                } else {
                    for (int q = 0; q < 4; ++q) {
                        (void)bits(CTX_DCT_SIZE, 1);
                        coeffs(o->coef + ncoef + q * 16, 16, true, false);
                    }
                }
                ncoef += 64;
            }
    }
    void chroma(int cu) {
        const int cs = cu / 2, nt = (cs / 4) * (cs / 4);
        for (int comp = 0; comp < 2; ++comp)
            for (int t = 0; t < nt; ++t) {
                if (!room(16)) return;
                coeffs(o->coef + ncoef, 16, true, true);
                ncoef += 16;
            }
    }
    void leaf(int d, int cx, int cy) {
        const int cu = 64 >> d;
        Node &n = o->nodes[qt_index(d, cx, cy)];
        const uint8_t split = n.split;
        memset(&n, 0, sizeof(n));
        n.split = split;
        n.intra = (uint8_t)bits(CTX_BLOCK_MODE, 1);
        if (n.intra) {
            uint32_t im = bits(CTX_INTRA_MODE, 5);
            if (im >= 18) { bs->error = 1; im = 1; }
            n.intra_mode = (uint8_t)im;
            n.ch_intra = (uint8_t)bits(CTX_BLOCK_MODE, 1);
            if (n.ch_intra) n.intra_cmode = (uint8_t)bits(CTX_INTRA_MODE, 3);
        } else {
            if (frame_type == 2) {
                n.ref_sel = (uint8_t)bits(CTX_REF_SEL, 1);
                n.bi = (uint8_t)bits(CTX_BLOCK_MODE, 1);
            }
            n.skip = (uint8_t)bits(CTX_SKIP_FLAG, 1);
            if (!n.skip) {
                n.merge = (uint8_t)bits(CTX_MERGE_FLAG, 1);
                if (!n.merge) {
                    if (frame_type != 2 && multiref_tool) {
                        n.ref_sel = (uint8_t)bits(CTX_REF_SEL, 2);
                        if (n.ref_sel >= MAX_REFS || !dpb_valid[n.ref_sel]) bs->error = 1;
                    }
                    n.dct_size = (uint8_t)bits(CTX_DCT_SIZE, 1);
                    const int32_t mx = se(CTX_MVD_X), my = se(CTX_MVD_Y);
                    if (mx < -32768 || mx > 32767 || my < -32768 || my > 32767) bs->error = 1;
                    n.mvd_x = (int16_t)mx;
                    n.mvd_y = (int16_t)my;
                }
            }
        }
        if (n.intra || !n.skip) {
            luma(cu, cx, cy);
            chroma(cu);
        }
    }
    void node(int d, int cx, int cy) {
        if (bs->error) return;
        const int cu = 64 >> d;
        const int px = ctu_x + cx * 8, py = ctu_y + cy * 8;
        const bool in_frame = px + cu <= W && py + cu <= H;
        const int h = 4 >> d;
        if (!in_frame && cu > 8) {
            for (int q = 0; q < 4; ++q) node(d + 1, cx + (q & 1) * h, cy + (q >> 1) * h);
            return;
        }
        if (!in_frame) return;
        const uint32_t split = bits(CTX_QT_SPLIT + d, 1);
        o->nodes[qt_index(d, cx, cy)].split = (uint8_t)split;
        if (split && cu == 8) { bs->error = 1; return; }
        if (split)
            for (int q = 0; q < 4; ++q) node(d + 1, cx + (q & 1) * h, cy + (q >> 1) * h);
        else
            leaf(d, cx, cy);
    }
    void ctu(int row, int col) {
        ctu_x = col * 64; ctu_y = row * 64; ncoef = 0;
        memset(o->nodes, 0, sizeof(o->nodes));
        o->tu8mask = 0;
        o->sao_has = 0; o->sao_band = 0; o->sao_offset = 0;
        node(0, 0, 0);
        if (bs->error) return;
        if (sao_tool) {
            o->sao_has = (int16_t)bits(CTX_SAO_TYPE, 1);
            if (o->sao_has) {
                const uint32_t band = bits(CTX_SAO_BAND, 5), off = bits(CTX_SAO_OFFSET, 4);
                if (band > 31 || off > 14) { bs->error = 1; return; }
                o->sao_band = (int16_t)band;
                o->sao_offset = (int16_t)((int)off - 7);
            }
        }
        o->ncoef = ncoef;
    }
};

// Legacy (v0 / v1) block syntax of one CTU (reference src/decoder.c:260-440
// and 486-552, the parse side of decode_block): fills the records the
// reconstruction kernel reads, motion vectors made absolute with the
// median of the left, above and above-right blocks inside the CTU.  Blocks
// outside the frame are not coded and count as inter blocks with a zero
// vector (the reference's zeroed block info).  As in the reference, a read
// past the end of the data yields zero bits and the parse goes on: the
// legacy decoder does not fail a frame on it (src/decoder.c:2847
// checks the reader's error for v2 streams only).
inline void parse_legacy_ctu(Parser &p, legacy::LBlock *blk, int ox, int oy, int W, int H, int ft) {
    uint8_t inter[legacy::BLOCKS];
    int mvx[legacy::BLOCKS], mvy[legacy::BLOCKS];
    for (int i = 0; i < legacy::BLOCKS; ++i) { inter[i] = 1; mvx[i] = 0; mvy[i] = 0; }
    auto med = [](int a, int b, int c) {
        if (a > b) std::swap(a, b);
        if (b > c) std::swap(b, c);
        if (a > b) std::swap(a, b);
        return b;
    };
    for (int b = 0; b < legacy::BLOCKS; ++b) {
        legacy::LBlock &k = blk[b];
        k.coded = 0;
        const int bx = b & 7, by = b >> 3, fx = ox + bx * 8, fy = oy + by * 8;
        if (fx + 8 > W || fy + 8 > H) continue;
        k.coded = 1;
        const int mode = ft != 0 ? (int)p.bits(CTX_BLOCK_MODE, 2) : 2;
        const bool intra = mode == 2, merge = mode == 3;
        int bmx = 0, bmy = 0, ref = 0;
        k.intra_mode = 1;
        if (intra) {
            uint32_t im = p.bits(CTX_INTRA_MODE, 5);
            if (im >= 18) im = 1;
            k.intra_mode = (uint8_t)im;
        } else {
            int ref_sel = 0;
            if (ft == 2) {
                ref_sel = (int)p.bits(CTX_REF_SEL, 2);
                if (ref_sel > 2) ref_sel = 1;
            }
            int px = fx * 4, py = fy * 4;
            int ax = 0, ay = 0, bvx = 0, bvy = 0, cvx = 0, cvy = 0;
            bool ha = false, hb = false, hc = false;
            if (bx > 0 && inter[b - 1]) { ax = mvx[b - 1]; ay = mvy[b - 1]; ha = true; }
            if (by > 0 && inter[b - 8]) { bvx = mvx[b - 8]; bvy = mvy[b - 8]; hb = true; }
            if (by > 0 && bx < 7 && inter[b - 7]) { cvx = mvx[b - 7]; cvy = mvy[b - 7]; hc = true; }
            if (ha || hb || hc) {
                if (!ha) { ax = hb ? bvx : cvx; ay = hb ? bvy : cvy; }
                if (!hb) { bvx = ha ? ax : cvx; bvy = ha ? ay : cvy; }
                if (!hc) { cvx = ha ? ax : bvx; cvy = ha ? ay : bvy; }
                px = med(ax, bvx, cvx);
                py = med(ay, bvy, cvy);
            }
            if (merge) {
                bmx = px; bmy = py;
                ref = ft == 2 ? ref_sel : 0;
            } else {
                int ri = 0;
                if (ft == 1) {
                    ri = (int)p.bits(CTX_REF_IDX, 2);
                    if (ri >= TC_REF_FRAMES) ri = 0;
                } else if (ft == 2) {
                    ri = ref_sel;
                }
                const int dx = p.se(CTX_MVD_X), dy = p.se(CTX_MVD_Y);
                bmx = dx + px; bmy = dy + py;
                ref = ri;
            }
        }
        k.mode = (uint8_t)mode;
        k.ref = (uint8_t)ref;
        k.mvd_x = bmx;
        k.mvd_y = bmy;
        k.tid = 0;
        if (mode == 1 || mode == 2) {
            k.tid = (uint8_t)p.bits(CTX_DCT_SIZE, 2);
            if (k.tid & 2) p.coeffs(k.luma, 64, false, false);
            else for (int q = 0; q < 4; ++q) p.coeffs(k.luma + 16 * q, 16, true, false);
        }
        p.coeffs(k.chroma, 16, true, false);
        p.coeffs(k.chroma + 16, 16, true, false);
        inter[b] = intra ? 0 : 1;
        mvx[b] = intra ? 0 : bmx;
        mvy[b] = intra ? 0 : bmy;
    }
}

struct Header;
inline tc_error_t parse_legacy_frame(const uint8_t *data, size_t size, Reader &bs, const Header &hdr, int entropy,
                                     int W, int H, int cols, int rows, legacy::LBlock *blocks);

struct Header {
    int version = 0, W = 0, H = 0, flags = 0, qp = 0, frame_num = 0, tools = 0;
    int profile = 0, level = 0, has_crc = 0, has_ext = 0, frame_type = 0;
};

// Frame header (reference src/decoder.c:102-225).
inline tc_error_t read_header(Reader &bs, Header &h) {
    if (bs.eof()) return TC_ERR_EOF;
    if (bs.bits(8) != TC_MAGIC_0 || bs.bits(8) != TC_MAGIC_1 || bs.bits(8) != TC_MAGIC_2) return TC_ERR_BITSTREAM;
    h.version = (int)bs.bits(8);
    if (h.version > TC_VERSION_V2) return TC_ERR_BITSTREAM;
    h.W = (int)bs.bits(16);
    h.H = (int)bs.bits(16);
    if (h.W == 0 || h.H == 0 || h.W > TC_MAX_WIDTH || h.H > TC_MAX_HEIGHT) return TC_ERR_BITSTREAM;
    h.flags = (int)bs.bits(8);
    const int8_t qd = (int8_t)bs.bits(8);
    h.frame_num = (int)bs.bits(8);
    int ext_type = -1;
    if (h.version == TC_VERSION_V0) (void)bs.bits(8);   // v0: reserved byte
    else {
        const int pl = (int)bs.bits(8);
        h.tools = (int)bs.bits(16);
        if (h.tools & ~(int)TC_TOOLS_IMPLEMENTED) return TC_ERR_BITSTREAM;
        h.profile = (pl >> 4) & 0x0F;
        h.level = pl & 0x0F;
        h.has_crc = (h.flags & TC_FLAG_CRC) != 0;
        h.has_ext = (h.flags & TC_FLAG_EXT_HEADER) != 0;
        if (h.has_ext) {
            const int fc = (int)bs.bits(8);
            ext_type = fc == 0 ? 0 : (fc == 2 ? 2 : 1);
        }
        if (h.profile > TC_PROFILE_MAX) return TC_ERR_BITSTREAM;
        static const int lw[9] = {4096, 320, 640, 1280, 1280, 1920, 1920, 3840, 3840};
        static const int lh[9] = {4096, 240, 480, 720, 720, 1080, 1080, 2160, 2160};
        if (h.level > 0 && h.level <= TC_LEVEL_MAX && (h.W > lw[h.level] || h.H > lh[h.level]))
            return TC_ERR_BITSTREAM;
    }
    if (bs.error) return TC_ERR_BITSTREAM;
    if (ext_type >= 0) h.frame_type = ext_type;
    else h.frame_type = (h.flags & TC_FLAG_KEY_FRAME) ? 0 : 1;
    h.qp = clampi(TC_QP_DEFAULT + qd, TC_QP_MIN, TC_QP_MAX);
    return TC_OK;
}

// Every CTU's block records of a legacy frame, the reader positioned after
// the header: rows as per-row runs behind a 16-bit entry table when the
// header has TC_FLAG_WPP (src/decoder.c:2676-2765; raw syntax), else one
// run, range coded when `entropy` (src/decoder.c:2613-2630, 2805-2830).
// Only a malformed entry table fails the frame.
inline tc_error_t parse_legacy_frame(const uint8_t *data, size_t size, Reader &bs, const Header &hdr, int entropy,
                                     int W, int H, int cols, int rows, legacy::LBlock *blocks) {
    const int ft = hdr.frame_type;
    uint8_t ctx[TC_NUM_CONTEXTS_RC];
    memset(ctx, 0, sizeof(ctx));
    if (hdr.flags & TC_FLAG_WPP) {
        const uint32_t noff = bs.bits(16);
        if (bs.error || noff > 63 || (int)noff != rows - 1) return TC_ERR_BITSTREAM;
        size_t off[64];
        off[0] = 0;
        for (uint32_t i = 0; i < noff; ++i) off[i + 1] = bs.bits(16);
        if (bs.error) return TC_ERR_BITSTREAM;
        bs.align();
        const size_t start = bs.pos;
        for (int r = 0; r < rows; ++r)
            if (start + off[r] > size || (r > 0 && off[r] < off[r - 1])) return TC_ERR_BITSTREAM;
        for (int r = 0; r < rows; ++r) {
            const size_t b0 = start + off[r], b1 = r + 1 < rows ? start + off[r + 1] : size;
            Reader rr;
            rr.init(data + b0, b1 - b0);
            Parser p{&rr, nullptr, ctx, W, H, ft, 0, 0, nullptr, nullptr, 0, 0, 0};
            for (int c = 0; c < cols; ++c)
                parse_legacy_ctu(p, blocks + (size_t)(r * cols + c) * legacy::BLOCKS, c * 64, r * 64, W, H, ft);
        }
    } else {
        RDec rc;
        if (entropy) rc.init(&bs);
        Parser p{&bs, entropy ? &rc : nullptr, ctx, W, H, ft, 0, 0, nullptr, nullptr, 0, 0, 0};
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < cols; ++c)
                parse_legacy_ctu(p, blocks + (size_t)(r * cols + c) * legacy::BLOCKS, c * 64, r * 64, W, H, ft);
    }
    return TC_OK;
}

}  // namespace parse
}  // namespace tcb
