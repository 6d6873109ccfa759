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
#include "tcb_parse.h"

using namespace tcb;
using namespace tcb::parse;

namespace {

uint64_t now_ns() {
    timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (uint64_t)t.tv_sec * 1000000000ull + (uint64_t)t.tv_nsec;
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
    const tc_error_t pe = parse_legacy_frame(data, size, bs, hdr, entropy, fw, fh, cols, rows, h_lblk);
    if (pe != TC_OK) return pe;
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
