// tcb_decoder.cpp — tc_decoder_* (reference include/tcodec.h:64-111): the
// serial syntax parse (range decoder / Exp-Golomb) runs on the host and
// fills the same per-CTU records the encoder emits; the reconstruction
// (prediction, dequantisation, inverse transform, deblocking, SAO) runs on
// the device as the CTU wavefront of decode_kernel (v2 streams) or of the
// legacy block kernel (v0 / v1 streams, tcb_legacy.cu).
//
// Mirrors reference src/decoder.c: header checks (102-225), frame-level
// flow (2541-2925), entry-point tables (2096-2190), syntax parse
// (1302-1520), display reorder for B-frame streams (2880-2956).
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <new>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/tcodec.h"
#include "tcb_encoder.h"
#include "tcb_entropy.h"
#include "tcb_launch.h"

using namespace tcb;

namespace {

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

uint64_t now_ns() {
    timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (uint64_t)t.tv_sec * 1000000000ull + (uint64_t)t.tv_nsec;
}

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
void parse_legacy_ctu(Parser &p, legacy::LBlock *blk, int ox, int oy, int W, int H, int ft) {
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

struct Header {
    int version = 0, W = 0, H = 0, flags = 0, qp = 0, frame_num = 0, tools = 0;
    int profile = 0, level = 0, has_crc = 0, has_ext = 0, frame_type = 0;
};

// Frame header (reference src/decoder.c:102-225).
tc_error_t read_header(Reader &bs, Header &h) {
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

}  // namespace

namespace tcb {

struct DecImpl {
    int W = 0, H = 0;                 // decoder geometry (dec->width/height)
    int fw = 0, fh = 0, sy = 0, sc = 0, cols = 0, rows = 0;   // allocated frame geometry
    int device = 0;
    cudaStream_t st = nullptr;
    DevFrame cur;                     // persistent reconstruction target
    DevFrame dpb[TC_REF_FRAMES];
    int dpb_ok[TC_REF_FRAMES] = {0, 0, 0, 0};
    int dpb_poc[TC_REF_FRAMES] = {-1, -1, -1, -1};
    std::vector<DevFrame> spare;      // free device frames
    CtuOut *d_rec = nullptr, *h_rec = nullptr;
    // Legacy (v0 / v1) streams: block records and the wavefront of
    // diagonals c + 2r (see tcb_legacy.cu).
    legacy::LBlock *d_lblk = nullptr, *h_lblk = nullptr;
    int *d_litems = nullptr;
    std::vector<int> ldiag_off, ldiag_cnt;
    FrameParams *d_params = nullptr;
    int *d_items = nullptr;
    std::vector<int> diag_off, diag_cnt;
    tc_frame_buf_t *out = nullptr;    // host output (pinned)
    std::vector<tc_frame_buf_t *> disp_frames;
    std::vector<int> disp_pocs;
    int disp_active = 0, disp_next = 0;
    tc_frame_buf_t *disp_out = nullptr;
    int crc_valid = 1, entropy = 0, threads = 4, profile = 0;
    uint64_t prof[7] = {0, 0, 0, 0, 0, 0, 0};

    // All three planes or none: a partly allocated frame is freed again.
    bool alloc_frame(DevFrame &f) {
        const size_t yb = (size_t)sy * fh + 64, cb = (size_t)sc * (fh / 2) + 64;
        if (dev_alloc(&f.y, yb) != cudaSuccess || dev_alloc(&f.cb, cb) != cudaSuccess ||
            dev_alloc(&f.cr, cb) != cudaSuccess) {
            free_frame(f);
            return false;
        }
        cudaMemset(f.y, 0, yb); cudaMemset(f.cb, 0, cb); cudaMemset(f.cr, 0, cb);
        return true;
    }
    void free_frame(DevFrame &f) { cudaFree(f.y); cudaFree(f.cb); cudaFree(f.cr); f = DevFrame(); }
    void release_geometry() {
        if (st) cudaStreamSynchronize(st);
        free_frame(cur);
        for (int i = 0; i < TC_REF_FRAMES; ++i) if (dpb_ok[i]) free_frame(dpb[i]);
        for (auto &f : spare) free_frame(f);
        spare.clear();
        for (int i = 0; i < TC_REF_FRAMES; ++i) { dpb_ok[i] = 0; dpb_poc[i] = -1; }
        cudaFree(d_rec); cudaFreeHost(h_rec); cudaFree(d_items);
        d_rec = nullptr; h_rec = nullptr; d_items = nullptr;
        cudaFree(d_lblk); cudaFreeHost(h_lblk); cudaFree(d_litems);
        d_lblk = nullptr; h_lblk = nullptr; d_litems = nullptr;
        tcb_host_frame_free(out);
        out = nullptr;
    }
    // Geometry-dependent buffers for w x h.  On failure everything is
    // released and the size forgotten, so the next frame starts over
    // instead of decoding into a partly allocated set.
    bool setup(int w, int h) {
        if (setup_buffers(w, h)) return true;
        release_geometry();
        fw = fh = 0;
        return false;
    }
    bool setup_buffers(int w, int h) {
        release_geometry();
        fw = w; fh = h;
        sy = ((w + 63) / 64) * 64;
        sc = ((w / 2 + 63) / 64) * 64;
        cols = (w + 63) / 64;
        rows = (h + 63) / 64;
        if (!alloc_frame(cur)) return false;
        if (dev_alloc(&d_rec, sizeof(CtuOut) * cols * rows) != cudaSuccess) return false;
        if (pinned_alloc(&h_rec, sizeof(CtuOut) * cols * rows) != cudaSuccess) return false;
        std::vector<int> items;
        diag_off.clear(); diag_cnt.clear();
        for (int d = 0; d < rows + cols - 1; ++d) {
            diag_off.push_back((int)items.size());
            for (int r = 0; r < rows; ++r) {
                const int c = d - r;
                if (c >= 0 && c < cols) items.push_back((r << 10) | c);
            }
            diag_cnt.push_back((int)items.size() - diag_off.back());
        }
        if (dev_alloc(&d_items, sizeof(int) * items.size()) != cudaSuccess) return false;
        cudaMemcpy(d_items, items.data(), sizeof(int) * items.size(), cudaMemcpyHostToDevice);
        std::vector<int> litems;
        ldiag_off.clear(); ldiag_cnt.clear();
        for (int d = 0; d < cols + 2 * (rows - 1); ++d) {
            ldiag_off.push_back((int)litems.size());
            for (int r = 0; r < rows; ++r) {
                const int c = d - 2 * r;
                if (c >= 0 && c < cols) litems.push_back((r << 10) | c);
            }
            ldiag_cnt.push_back((int)litems.size() - ldiag_off.back());
        }
        if (dev_alloc(&d_litems, sizeof(int) * litems.size()) != cudaSuccess) return false;
        cudaMemcpy(d_litems, litems.data(), sizeof(int) * litems.size(), cudaMemcpyHostToDevice);
        const size_t nblk = (size_t)cols * rows * legacy::BLOCKS;
        if (dev_alloc(&d_lblk, sizeof(legacy::LBlock) * nblk) != cudaSuccess) return false;
        if (pinned_alloc(&h_lblk, sizeof(legacy::LBlock) * nblk) != cudaSuccess) return false;
        out = tcb_host_frame_alloc(w, h, 1);
        return out != nullptr;
    }
    DevFrame take_frame() {
        if (!spare.empty()) { DevFrame f = spare.back(); spare.pop_back(); return f; }
        DevFrame f;
        if (!alloc_frame(f)) f = DevFrame();
        return f;
    }
    bool d2h(tc_frame_buf_t *dst, const DevFrame &src) {
        return cudaMemcpy2DAsync(dst->y, dst->stride_y, src.y, sy, fw, fh, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
               cudaMemcpy2DAsync(dst->cb, dst->stride_c, src.cb, sc, fw / 2, fh / 2, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
               cudaMemcpy2DAsync(dst->cr, dst->stride_c, src.cr, sc, fw / 2, fh / 2, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
               cudaStreamSynchronize(st) == cudaSuccess;
    }
    tc_error_t decode(const uint8_t *data, size_t size, const tc_pixel_t **y, int *ys, const tc_pixel_t **cb,
                      int *cbs, const tc_pixel_t **cr, int *crs);
    tc_error_t legacy_body(const uint8_t *data, size_t size, Reader &bs, const Header &hdr);
    tc_error_t emit(tc_frame_buf_t *f, const tc_pixel_t **y, int *ys, const tc_pixel_t **cb, int *cbs,
                    const tc_pixel_t **cr, int *crs) {
        if (y) *y = f->y;
        if (ys) *ys = f->stride_y;
        if (cb) *cb = f->cb;
        if (cbs) *cbs = f->stride_c;
        if (cr) *cr = f->cr;
        if (crs) *crs = f->stride_c;
        return TC_OK;
    }
    tc_error_t pop_display(const tc_pixel_t **y, int *ys, const tc_pixel_t **cb, int *cbs,
                           const tc_pixel_t **cr, int *crs) {
        for (size_t i = 0; i < disp_pocs.size(); ++i)
            if (disp_pocs[i] == disp_next) {
                if (!disp_out) disp_out = tcb_host_frame_alloc(W, H, 1);
                if (!disp_out) return TC_ERR_MEMORY;
                tc_frame_buf_t *f = disp_frames[i];
                const int cw = (disp_out->width < f->width ? disp_out->width : f->width);
                const int chh = (disp_out->height < f->height ? disp_out->height : f->height);
                for (int r = 0; r < chh; ++r) memcpy(disp_out->y + (size_t)r * disp_out->stride_y, f->y + (size_t)r * f->stride_y, cw);
                for (int r = 0; r < chh / 2; ++r) {
                    memcpy(disp_out->cb + (size_t)r * disp_out->stride_c, f->cb + (size_t)r * f->stride_c, cw / 2);
                    memcpy(disp_out->cr + (size_t)r * disp_out->stride_c, f->cr + (size_t)r * f->stride_c, cw / 2);
                }
                tcb_host_frame_free(f);
                disp_frames.erase(disp_frames.begin() + i);
                disp_pocs.erase(disp_pocs.begin() + i);
                disp_next++;
                return emit(disp_out, y, ys, cb, cbs, cr, crs);
            }
        return TC_ERR_NEED_MORE;
    }
};

tc_error_t DecImpl::decode(const uint8_t *data, size_t size, const tc_pixel_t **y, int *ys,
                           const tc_pixel_t **cb, int *cbs, const tc_pixel_t **cr, int *crs) {
    const uint64_t t_parse0 = now_ns();
    Reader bs;
    bs.init(data, size);
    Header hdr;
    tc_error_t err = read_header(bs, hdr);
    if (err != TC_OK) return err;
    const bool legacy_stream = hdr.version != TC_VERSION_V2;
    if ((hdr.W & 1) || (hdr.H & 1)) return TC_ERR_BITSTREAM;
    if (legacy_stream && (hdr.tools & TC_TOOL_ENTRY_POINTS)) return TC_ERR_BITSTREAM;
    if (W == 0 || H == 0) { W = hdr.W; H = hdr.H; }
    if (!cur.y || fw != hdr.W || fh != hdr.H)
        if (!setup(hdr.W, hdr.H)) return TC_ERR_MEMORY;
    crc_valid = 1;
    if (hdr.has_crc) {
        if (size >= 2) {
            const size_t p = size - 2;
            if (crc16_ccitt(data, p) != (uint16_t)((data[p] << 8) | data[p + 1])) crc_valid = 0;
        } else {
            crc_valid = 0;
        }
    }
    if (!legacy_stream && (hdr.flags & TC_FLAG_WPP)) return TC_ERR_BITSTREAM;
    entropy = (hdr.version != TC_VERSION_V0 && (hdr.tools & TC_TOOL_ENTROPY_CODED)) ? 1 : 0;
    bs.align();
    if (hdr.frame_type == 0 && hdr.frame_num > 0)
        for (int i = 0; i < TC_REF_FRAMES; ++i) {
            if (dpb_ok[i]) spare.push_back(dpb[i]);
            dpb_ok[i] = 0; dpb_poc[i] = -1; dpb[i] = DevFrame();
        }
    uint64_t t_parse1 = 0;
    if (legacy_stream) {
        const tc_error_t le = legacy_body(data, size, bs, hdr);
        if (le != TC_OK) return le;
        t_parse1 = now_ns();
    } else {
    // ---- parse every CTU into its record ------------------------------
    const int multiref_tool = (hdr.tools & TC_TOOL_MULTI_REF) != 0;
    const int sao_tool = (hdr.tools & TC_TOOL_SAO) != 0;
    auto parse_rows = [&](Reader &r, RDec *rc, uint8_t *ctx, int row0, int row1) -> bool {
        Parser p{&r, rc, ctx, fw, fh, hdr.frame_type, multiref_tool, sao_tool, dpb_ok, nullptr, 0, 0, 0};
        for (int row = row0; row < row1; ++row)
            for (int col = 0; col < cols; ++col) {
                p.o = h_rec + row * cols + col;
                p.ctu(row, col);
                if (r.error) return false;
            }
        return true;
    };
    if (hdr.tools & TC_TOOL_ENTRY_POINTS) {
        // Entry-point table (reference src/decoder.c:2096-2190).
        if (rows < 1 || rows > 64 || cols < 1) return TC_ERR_BITSTREAM;
        if (bs.pos >= bs.size) return TC_ERR_BITSTREAM;
        const uint32_t nrows = bs.bits(16);
        if (bs.error || nrows != (uint32_t)rows) return TC_ERR_BITSTREAM;
        uint32_t off[64];
        for (int i = 0; i < rows; ++i) {
            off[i] = bs.bits(32);
            if (bs.error) return TC_ERR_BITSTREAM;
        }
        const size_t payload = bs.pos;
        size_t data_end = size;
        if (hdr.has_crc) {
            if (data_end < 2) return TC_ERR_BITSTREAM;
            data_end -= 2;
        }
        if (data_end < payload) return TC_ERR_BITSTREAM;
        const size_t datalen = data_end - payload;
        if (off[0] != 0) return TC_ERR_BITSTREAM;
        for (int i = 1; i < rows; ++i)
            if (off[i] < off[i - 1] || off[i] > datalen) return TC_ERR_BITSTREAM;
        for (int r = 0; r < rows; ++r) {
            const size_t start = payload + off[r];
            const size_t end = r + 1 < rows ? payload + off[r + 1] : data_end;
            if (end < start || end > size) return TC_ERR_BITSTREAM;
        }
        // Every row is its own substream with fresh contexts and writes
        // only its own CTU records, so the rows parse on up to `threads`
        // host threads (tc_decoder_set_threads); any bad row fails the frame.
        bool row_bad[64];
        auto parse_part = [&](int first, int step) {
            for (int r = first; r < rows; r += step) {
                const size_t start = payload + off[r];
                const size_t end = r + 1 < rows ? payload + off[r + 1] : data_end;
                Reader rr;
                rr.init(data + start, end - start);
                RDec rc;
                uint8_t ctx[TC_NUM_CONTEXTS_RC];
                memset(ctx, 0, sizeof(ctx));
                if (entropy) rc.init(&rr);
                row_bad[r] = !parse_rows(rr, entropy ? &rc : nullptr, ctx, r, r + 1);
            }
        };
        const int nth = std::max(1, std::min(threads, rows));
        if (nth > 1) {
            std::vector<std::thread> th;
            for (int t = 1; t < nth; ++t) th.emplace_back(parse_part, t, nth);
            parse_part(0, nth);
            for (auto &x : th) x.join();
        } else {
            parse_part(0, 1);
        }
        for (int r = 0; r < rows; ++r)
            if (row_bad[r]) return TC_ERR_BITSTREAM;
    } else {
        RDec rc;
        uint8_t ctx[TC_NUM_CONTEXTS_RC];
        memset(ctx, 0, sizeof(ctx));
        if (entropy) rc.init(&bs);
        if (!parse_rows(bs, entropy ? &rc : nullptr, ctx, 0, rows)) return TC_ERR_BITSTREAM;
    }
    t_parse1 = now_ns();
    // ---- device reconstruction ------------------------------------------
    FrameParams P;
    memset(&P, 0, sizeof(P));
    P.W = W; P.H = H; P.stride_y = sy; P.stride_c = sc; P.ctu_cols = cols; P.ctu_rows = rows;
    P.rec_y = cur.y; P.rec_cb = cur.cb; P.rec_cr = cur.cr;
    for (int i = 0; i < MAX_REFS; ++i) {
        P.ref_valid[i] = dpb_ok[i];
        P.ref_poc[i] = dpb_poc[i];
        const DevFrame &f = dpb_ok[i] ? dpb[i] : cur;
        P.ref_y[i] = f.y; P.ref_cb[i] = f.cb; P.ref_cr[i] = f.cr;
    }
    P.out = d_rec;
    P.frame_type = hdr.frame_type;
    P.poc = hdr.frame_num;
    P.qp = hdr.qp;
    P.qp_c = clampi(hdr.qp + 1, 0, 63);
    P.fresh_skip = (hdr.tools & TC_TOOL_FRESH_SKIP) != 0;
    static const int qs[64] = TCB_QSCALE_INIT;
    static const int jw[4] = TCB_JND_INIT;
    for (int b = 0; b < 4; ++b) {
        P.eff_l[b] = maxi((qs[P.qp] * jw[b] + 4) >> 3, 1);
        P.eff_c[b] = maxi((qs[P.qp_c] * jw[b] + 4) >> 3, 1);
    }
    if (!d_params && dev_alloc(&d_params, sizeof(FrameParams)) != cudaSuccess) return TC_ERR_MEMORY;
    const int nctu = rows * cols;
    if (cudaMemcpyAsync(d_params, &P, sizeof(P), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(d_rec, h_rec, sizeof(CtuOut) * nctu, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return TC_ERR_INTERNAL;
    for (size_t d = 0; d < diag_off.size(); ++d)
        if (launch_decode_items(d_params, d_items + diag_off[d], diag_cnt[d], st) != cudaSuccess)
            return TC_ERR_INTERNAL;
    }   // v2 stream
    // DPB: slot 3 falls out and its buffer takes a copy of the
    // reconstruction into slot 0 (another buffer when slot 3 is empty, taken
    // before anything moves, so a failed allocation leaves the DPB as it
    // was).  The copy follows this frame's kernels on the stream.
    DevFrame nf;
    if (dpb_ok[TC_REF_FRAMES - 1]) {
        nf = dpb[TC_REF_FRAMES - 1];
    } else {
        nf = take_frame();
        if (!nf.y) return TC_ERR_MEMORY;
    }
    for (int i = TC_REF_FRAMES - 1; i > 0; --i) { dpb[i] = dpb[i - 1]; dpb_ok[i] = dpb_ok[i - 1]; dpb_poc[i] = dpb_poc[i - 1]; }
    if (cudaMemcpyAsync(nf.y, cur.y, (size_t)sy * fh, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(nf.cb, cur.cb, (size_t)sc * (fh / 2), cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(nf.cr, cur.cr, (size_t)sc * (fh / 2), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return TC_ERR_INTERNAL;
    dpb[0] = nf; dpb_ok[0] = 1; dpb_poc[0] = hdr.frame_num;
    if (!d2h(out, cur)) return TC_ERR_INTERNAL;
    const uint64_t t_rec = now_ns();
    if (profile) { prof[0] += t_parse1 - t_parse0; prof[2] += t_rec - t_parse1; }
    if (hdr.has_ext) {
        // Display reorder (reference src/decoder.c:2880-2925).
        const int is_rap = (hdr.flags & TC_FLAG_RAP) != 0;
        if (is_rap && disp_active) {
            for (auto *f : disp_frames) tcb_host_frame_free(f);
            disp_frames.clear(); disp_pocs.clear();
            disp_next = hdr.frame_num;
        }
        disp_active = 1;
        if ((int)disp_frames.size() < TC_REF_FRAMES + 1) {
            tc_frame_buf_t *f = tcb_host_frame_alloc(fw, fh, 0);
            if (!f) return TC_ERR_MEMORY;
            for (int r = 0; r < fh; ++r) memcpy(f->y + (size_t)r * f->stride_y, out->y + (size_t)r * out->stride_y, fw);
            for (int r = 0; r < fh / 2; ++r) {
                memcpy(f->cb + (size_t)r * f->stride_c, out->cb + (size_t)r * out->stride_c, fw / 2);
                memcpy(f->cr + (size_t)r * f->stride_c, out->cr + (size_t)r * out->stride_c, fw / 2);
            }
            disp_frames.push_back(f);
            disp_pocs.push_back(hdr.frame_num);
        }
        return pop_display(y, ys, cb, cbs, cr, crs);
    }
    return emit(out, y, ys, cb, cbs, cr, crs);
}

// Legacy stream body: rows as per-row runs behind a 16-bit entry table
// (TC_FLAG_WPP) or one run, raw or range coded; parse on the host, then
// the legacy CTU wavefront reconstructs into `cur`, whose previous contents
// (the last decoded frame) stand in for samples not yet decoded, as in the
// reference decoder (src/decoder.c:2620-2770, 652-683).
tc_error_t DecImpl::legacy_body(const uint8_t *data, size_t size, Reader &bs, const Header &hdr) {
    if (upload_legacy_tables() != cudaSuccess) return TC_ERR_INTERNAL;
    const int ft = hdr.frame_type;
    const size_t nblk = (size_t)cols * rows * legacy::BLOCKS;
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
            Parser p{&rr, nullptr, ctx, fw, fh, ft, 0, 0, dpb_ok, nullptr, 0, 0, 0};
            for (int c = 0; c < cols; ++c)
                parse_legacy_ctu(p, h_lblk + (size_t)(r * cols + c) * legacy::BLOCKS, c * 64, r * 64, fw, fh, ft);
        }
    } else {
        RDec rc;
        if (entropy) rc.init(&bs);
        Parser p{&bs, entropy ? &rc : nullptr, ctx, fw, fh, ft, 0, 0, dpb_ok, nullptr, 0, 0, 0};
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < cols; ++c)
                parse_legacy_ctu(p, h_lblk + (size_t)(r * cols + c) * legacy::BLOCKS, c * 64, r * 64, fw, fh, ft);
    }
    legacy::LFrame F;
    memset(&F, 0, sizeof(F));
    F.W = fw; F.H = fh; F.sy = sy; F.sc = sc; F.ctu_cols = cols; F.ctu_rows = rows;
    F.rec_y = cur.y; F.rec_cb = cur.cb; F.rec_cr = cur.cr;
    int fp = -1, bp = 0x7FFFFFFF;
    for (int i = 0; i < TC_REF_FRAMES; ++i) {
        F.dpb_y[i] = dpb_ok[i] ? dpb[i].y : nullptr;
        if (!dpb_ok[i] || dpb_poc[i] < 0) continue;
        if (dpb_poc[i] < hdr.frame_num && dpb_poc[i] > fp) { fp = dpb_poc[i]; F.fwd_y = dpb[i].y; }
        if (dpb_poc[i] > hdr.frame_num && dpb_poc[i] < bp) { bp = dpb_poc[i]; F.bwd_y = dpb[i].y; }
    }
    F.frame_type = ft;
    F.qp = hdr.qp;
    F.blocks = d_lblk;
    if (cudaMemcpyAsync(d_lblk, h_lblk, sizeof(legacy::LBlock) * nblk, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return TC_ERR_INTERNAL;
    for (size_t d = 0; d < ldiag_off.size(); ++d)
        if (launch_legacy_ctus(F, d_litems + ldiag_off[d], ldiag_cnt[d], false, st) != cudaSuccess)
            return TC_ERR_INTERNAL;
    return TC_OK;
}

}  // namespace tcb

struct tc_decoder {
    tcb::DecImpl *impl;
};

extern "C" {

tc_decoder_t *tc_decoder_create(int32_t width, int32_t height) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return nullptr;
    if (init_device_tables() != cudaSuccess) return nullptr;
    tc_decoder_t *d = (tc_decoder_t *)calloc(1, sizeof(tc_decoder_t));
    if (!d) return nullptr;
    d->impl = new (std::nothrow) DecImpl();
    if (!d->impl) { free(d); return nullptr; }
    DecImpl &e = *d->impl;
    cudaGetDevice(&e.device);
    if (cudaStreamCreateWithFlags(&e.st, cudaStreamNonBlocking) != cudaSuccess) {
        delete d->impl; free(d); return nullptr;
    }
    e.W = width > 0 && height > 0 ? width : 0;
    e.H = width > 0 && height > 0 ? height : 0;
    return d;
}

void tc_decoder_destroy(tc_decoder_t *dec) {
    if (!dec) return;
    if (dec->impl) {
        DecImpl &e = *dec->impl;
        e.release_geometry();
        for (auto *f : e.disp_frames) tcb_host_frame_free(f);
        tcb_host_frame_free(e.disp_out);
        cudaFree(e.d_params);
        if (e.st) cudaStreamDestroy(e.st);
        delete dec->impl;
    }
    free(dec);
}

tc_error_t tc_decoder_decode(tc_decoder_t *dec, const uint8_t *data, size_t size, const tc_pixel_t **y,
                             int *stride_y, const tc_pixel_t **cb, int *stride_cb, const tc_pixel_t **cr,
                             int *stride_cr) {
    // no frame unless one is output: callers that ignore the status read
    // NULL planes rather than stale pointers
    if (y) *y = nullptr;
    if (cb) *cb = nullptr;
    if (cr) *cr = nullptr;
    if (stride_y) *stride_y = 0;
    if (stride_cb) *stride_cb = 0;
    if (stride_cr) *stride_cr = 0;
    if (!dec || !dec->impl || !data || size == 0) return TC_ERR_PARAM;
    if (cudaSetDevice(dec->impl->device) != cudaSuccess) return TC_ERR_INTERNAL;
    return dec->impl->decode(data, size, y, stride_y, cb, stride_cb, cr, stride_cr);
}

void tc_decoder_get_info(tc_decoder_t *dec, int32_t *width, int32_t *height) {
    if (!dec || !dec->impl) return;
    if (width) *width = dec->impl->W;
    if (height) *height = dec->impl->H;
}

tc_error_t tc_decoder_flush_tail(tc_decoder_t *dec, const tc_pixel_t **y, int *stride_y, const tc_pixel_t **cb,
                                 int *stride_cb, const tc_pixel_t **cr, int *stride_cr) {
    if (!dec || !dec->impl || !dec->impl->disp_active) return TC_ERR_EOF;
    const tc_error_t r = dec->impl->pop_display(y, stride_y, cb, stride_cb, cr, stride_cr);
    return r == TC_ERR_NEED_MORE ? TC_ERR_EOF : r;
}

int tc_decoder_crc_valid(tc_decoder_t *dec) { return dec && dec->impl ? dec->impl->crc_valid : 0; }
int tc_decoder_entropy_coded(tc_decoder_t *dec) { return dec && dec->impl ? dec->impl->entropy : 0; }
void tc_decoder_set_profile(tc_decoder_t *dec, int enabled) { if (dec && dec->impl) dec->impl->profile = enabled; }
void tc_decoder_reset_profile(tc_decoder_t *dec) {
    if (dec && dec->impl) memset(dec->impl->prof, 0, sizeof(dec->impl->prof));
}
void tc_decoder_get_profile(tc_decoder_t *dec, uint64_t *parse_ns, uint64_t *coeff_ns, uint64_t *transform_ns,
                            uint64_t *motion_ns, uint64_t *chroma_ns, uint64_t *deblock_ns, uint64_t *copy_ns) {
    if (!dec || !dec->impl) return;
    const uint64_t *p = dec->impl->prof;
    if (parse_ns) *parse_ns = p[0];
    if (coeff_ns) *coeff_ns = p[1];
    if (transform_ns) *transform_ns = p[2];
    if (motion_ns) *motion_ns = p[3];
    if (chroma_ns) *chroma_ns = p[4];
    if (deblock_ns) *deblock_ns = p[5];
    if (copy_ns) *copy_ns = p[6];
}
void tc_decoder_set_threads(tc_decoder_t *dec, int nthreads) {
    if (!dec || !dec->impl) return;
    dec->impl->threads = nthreads < 1 ? 1 : (nthreads > 16 ? 16 : nthreads);
}

}  // extern "C"
