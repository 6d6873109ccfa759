// tcb_encoder.cpp — tc_encoder_* (reference include/tcodec.h:27-57) on the
// B200 pixel pipeline.
//
// Host responsibilities per frame (reference src/encoder.c:2625-3121
// encode_poc_frame): frame type (key interval, scene cut on a device
// histogram, B-frame schedule), QP / rate control, header and tool flags,
// DPB bookkeeping, entropy coding of the device's CTU records, entry-point
// tables and CRC.  Device responsibilities: everything that touches pixels
// (the v2 CTU engine, or the legacy 8x8 block kernel when use_v2 = 0).
// Frames stay resident in HBM: the DPB is a ring of device frame buffers
// and only the packet, the CTU records and the host copy of the
// reconstruction (API contract: encoder->recon) come back each frame.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <thread>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/tcodec.h"
#include "../../include/tcodec_b200.h"
#include "tcb_encoder.h"
#include "tcb_entropy.h"
#include "tcb_launch.h"

using namespace tcb;

namespace {

int qscale(int qp) {
    static const int t[64] = TCB_QSCALE_INIT;
    return t[qp < 0 ? 0 : (qp > 63 ? 63 : qp)];
}
int jnd(int band) {
    static const int t[4] = TCB_JND_INIT;
    return t[band < 0 ? 0 : (band > 3 ? 3 : band)];
}
// Effective quant step (reference tcodec_common.h:226-230).
int eff_scale(int qp, int band) {
    const int e = (qscale(qp) * jnd(band) + 4) >> 3;
    return e < 1 ? 1 : e;
}

// Rate control: CQP keeps the configured QP; CBR/VBR steer QP through the
// logistic rho(QP) model and a one-second budget buffer (reference
// src/ratectl.c:20-156).
double rho_from_qp(int qp) { return 1.0 / (1.0 + exp(-((double)qp - 28.0) / 8.0)); }
int qp_from_rho(double r) {
    if (r <= 0.01) return 0;
    if (r >= 0.99) return 63;
    const double q = 28.0 + 8.0 * log(r / (1.0 - r));
    return clampi((int)(q + 0.5), 0, 63);
}

}  // namespace

void EncImpl::rc_init(const tc_config_t &c) {
    rc_method = c.rc_method;
    rc_qp = clampi(c.qp, 0, 63);
    rc_base_qp = rc_qp;
    const int fn = c.fps_num > 0 ? c.fps_num : 60, fd = c.fps_den > 0 ? c.fps_den : 1;
    const double fps = (double)fn / (double)fd;
    rc_frame_target = (c.target_bitrate > 0 && fps > 0) ? (long long)((double)c.target_bitrate / fps) : 0;
    rc_buffer_size = (double)c.target_bitrate;
    rc_buffer_level = 0.5;
}

void EncImpl::rc_frame_start() {
    if (rc_method == TC_RC_CQP) { rc_qp = rc_base_qp; return; }
    if (rc_method == TC_RC_CBR || rc_method == TC_RC_VBR) {
        const double f = rc_buffer_level;
        double adj = 0.0;
        if (f > 0.8) adj = -2.0;
        else if (f > 0.6) adj = -1.0;
        else if (f < 0.2) adj = 2.0;
        else if (f < 0.4) adj = 1.0;
        double t = rho_from_qp(rc_qp) + adj * 0.05;
        t = t < 0.05 ? 0.05 : (t > 0.95 ? 0.95 : t);
        rc_qp = qp_from_rho(t);
    }
}

void EncImpl::rc_frame_end(long long bits) {
    if (rc_buffer_size > 0) {
        rc_buffer_level += ((double)rc_frame_target - (double)bits) / rc_buffer_size;
        rc_buffer_level = rc_buffer_level < 0.0 ? 0.0 : (rc_buffer_level > 1.0 ? 1.0 : rc_buffer_level);
    }
}

#define CK(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) { last_cuda_error = _e; return false; } } while (0)

size_t EncImpl::device_footprint(const tc_config_t &c) {
    const int W = c.width, H = c.height;
    const size_t sy = ((W + 63) / 64) * 64, sc = ((W / 2 + 63) / 64) * 64;
    const size_t nctu = (size_t)((W + 63) / 64) * ((H + 63) / 64);
    const size_t cells = (size_t)((W + 7) / 8) * ((H + 7) / 8);
    auto R = DeviceArena::round_up;
    const size_t frame = R(sy * H + 64) + 2 * R(sc * (H / 2) + 64);
    size_t n = (NPOOL + 1) * frame;                       // DPB pool + input
    n += 2 * R(sizeof(MvCell) * cells);                   // MV grids
    n += R(sizeof(CtuOut) * nctu);                        // decision records
    n += R(sizeof(FrameParams)) + R(16 * sizeof(int)) + R(sizeof(unsigned long long)) + R(sizeof(int));
    n += R(sizeof(int) * nctu) + R(2 * sizeof(int)) + R(sizeof(int) * nctu);   // flags, ctrl, queue
    if (c.enable_b_frames) n += BF_MAX * frame;           // reorder buffers at their cap
    return n;
}

bool EncImpl::init(const tc_config_t &c) {
    cfg = c;
    W = c.width; H = c.height;
    sy = ((W + 63) / 64) * 64;
    sc = ((W / 2 + 63) / 64) * 64;
    ctu_cols = (W + 63) / 64;
    ctu_rows = (H + 63) / 64;
    grid_w = (W + 7) / 8;
    grid_h = (H + 7) / 8;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return false;
    CK(cudaGetDevice(&device));
    CK(init_device_tables());
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    own_st = st;
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    const size_t ybytes = (size_t)sy * H + 64, cbytes = (size_t)sc * (H / 2) + 64;
    for (int i = 0; i < NPOOL; ++i) {
        CK(dmalloc(&pool[i].y, ybytes));
        CK(dmalloc(&pool[i].cb, cbytes));
        CK(dmalloc(&pool[i].cr, cbytes));
        CK(cudaMemset(pool[i].y, 0, ybytes));
        CK(cudaMemset(pool[i].cb, 0, cbytes));
        CK(cudaMemset(pool[i].cr, 0, cbytes));
    }
    CK(dmalloc(&cur.y, ybytes));
    CK(dmalloc(&cur.cb, cbytes));
    CK(dmalloc(&cur.cr, cbytes));
    CK(cudaMemset(cur.y, 0, ybytes));
    CK(cudaMemset(cur.cb, 0, cbytes));
    CK(cudaMemset(cur.cr, 0, cbytes));
    for (int i = 0; i < 2; ++i) {
        CK(dmalloc(&grid[i], sizeof(MvCell) * grid_w * grid_h));
        std::vector<MvCell> init(grid_w * grid_h);
        for (auto &g : init) { g.dx = 0; g.dy = 0; g.intra = 1; g.pad = 0; }
        CK(cudaMemcpy(grid[i], init.data(), sizeof(MvCell) * init.size(), cudaMemcpyHostToDevice));
    }
    const int nctu = ctu_cols * ctu_rows;
    CK(dmalloc(&d_out, sizeof(CtuOut) * nctu));
    CK(pinned_alloc(&h_out, sizeof(CtuOut) * nctu));
    CK(dmalloc(&d_params, sizeof(FrameParams)));
    CK(dmalloc(&d_hist, 16 * sizeof(int)));
    CK(pinned_alloc(&h_hist, 16 * sizeof(int)));
    CK(dmalloc(&d_sse, sizeof(unsigned long long)));
    CK(pinned_alloc(&h_sse, sizeof(unsigned long long)));
    CK(dmalloc(&d_err, sizeof(int)));
    CK(cudaMemset(d_err, 0, sizeof(int)));
    CK(dmalloc(&d_done, sizeof(int) * ctu_cols * ctu_rows));
    CK(cudaMemset(d_done, 0, sizeof(int) * ctu_cols * ctu_rows));
    CK(dmalloc(&d_ctrl, 2 * sizeof(int)));
    CK(pinned_alloc(&h_ctrl, 2 * sizeof(int)));
    CK(pinned_alloc(&h_params_pin, sizeof(FrameParams)));
    CK(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
    {
        const char *wf = getenv("TCB_WAVEFRONT");
        persistent = !(wf && strcmp(wf, "diagonal") == 0);
    }
    // Anti-diagonal wavefront item lists.
    std::vector<int> items;
    for (int d = 0; d < ctu_rows + ctu_cols - 1; ++d) {
        diag_off.push_back((int)items.size());
        for (int r = 0; r < ctu_rows; ++r) {
            const int col = d - r;
            if (col >= 0 && col < ctu_cols) items.push_back((r << 10) | col);
        }
        diag_cnt.push_back((int)items.size() - diag_off.back());
    }
    CK(dmalloc(&d_items, sizeof(int) * items.size()));
    CK(cudaMemcpy(d_items, items.data(), sizeof(int) * items.size(), cudaMemcpyHostToDevice));
    for (int i = 0; i < TC_REF_FRAMES; ++i) { dpb_slot[i] = -1; dpb_poc[i] = -1; }
    if (!c.use_v2) {
        // Legacy 8x8 block path: records, wavefront of diagonals c + 2r,
        // and the row layout (reference src/encoder.c:2495-2506: rows as
        // separate runs when there are several rows and threads and no
        // range coder).
        legacy = true;
        const int threads = c.threads > 0 ? c.threads : 4;
        legacy_wpp = ctu_rows > 1 && threads > 1 && !c.enable_entropy_coded;
        CK(upload_legacy_tables());
        CK(dmalloc(&d_lblk, sizeof(legacy::LBlock) * (size_t)nctu * legacy::BLOCKS));
        CK(pinned_alloc(&h_lblk, sizeof(legacy::LBlock) * (size_t)nctu * legacy::BLOCKS));
        std::vector<int> litems;
        for (int d = 0; d < ctu_cols + 2 * (ctu_rows - 1); ++d) {
            ldiag_off.push_back((int)litems.size());
            for (int r = 0; r < ctu_rows; ++r) {
                const int col = d - 2 * r;
                if (col >= 0 && col < ctu_cols) litems.push_back((r << 10) | col);
            }
            ldiag_cnt.push_back((int)litems.size() - ldiag_off.back());
        }
        CK(dmalloc(&d_litems, sizeof(int) * litems.size()));
        CK(cudaMemcpy(d_litems, litems.data(), sizeof(int) * litems.size(), cudaMemcpyHostToDevice));
    }
    out_buf_size = (size_t)W * H * 3;
    out_buf = (uint8_t *)calloc(out_buf_size, 1);
    if (!out_buf) return false;
    rc_init(c);
    bf_b_mode = c.enable_b_frames ? 1 : 0;
    // B-frame reorder buffers, allocated once: the reorder path then makes
    // no device allocation (and no implicit device synchronisation) per frame.
    // Each frame joins bf_free before its planes are allocated, so a failed
    // allocation leaves nothing that release() does not free.
    if (bf_b_mode)
        for (size_t i = 0; i < BF_MAX; ++i) {
            bf_free.emplace_back();
            DevFrame &f = bf_free.back();
            CK(dmalloc(&f.y, ybytes));
            CK(dmalloc(&f.cb, cbytes));
            CK(dmalloc(&f.cr, cbytes));
        }
    return true;
}

void EncImpl::release() {
    if (st) cudaStreamSynchronize(st);
    if (own_st) cudaStreamSynchronize(own_st);
    for (int i = 0; i < NPOOL; ++i) { dfree(pool[i].y); dfree(pool[i].cb); dfree(pool[i].cr); }
    dfree(cur.y); dfree(cur.cb); dfree(cur.cr);
    dfree(grid[0]); dfree(grid[1]);
    dfree(d_out); cudaFreeHost(h_out);
    dfree(d_params); dfree(d_hist); cudaFreeHost(h_hist);
    dfree(d_sse); cudaFreeHost(h_sse); dfree(d_err); dfree(d_items);
    dfree(d_done); dfree(d_ctrl); cudaFreeHost(h_ctrl); cudaFreeHost(h_params_pin);
    for (auto &f : bf_frames) { dfree(f.y); dfree(f.cb); dfree(f.cr); }
    for (auto &f : bf_free) { dfree(f.y); dfree(f.cb); dfree(f.cr); }
    bf_frames.clear();
    bf_free.clear();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (own_st) cudaStreamDestroy(own_st);
    free(out_buf);
    free(out_buf_alt);
    cudaFreeHost(h_out_alt);
    dfree(d_lblk); cudaFreeHost(h_lblk); cudaFreeHost(h_lblk_alt); dfree(d_litems);
}

int EncImpl::free_pool_slot() const {
    for (int i = 0; i < NPOOL; ++i) {
        bool used = false;
        for (int k = 0; k < TC_REF_FRAMES; ++k) used |= dpb_slot[k] == i;
        if (!used) return i;
    }
    return -1;
}

bool EncImpl::upload(const tc_pixel_t *y, int ys, const tc_pixel_t *cb, int cbs, const tc_pixel_t *cr,
                     int crs, const DevFrame &dst, cudaMemcpyKind kind) {
    CK(cudaMemcpy2DAsync(dst.y, sy, y, ys, W, H, kind, st));
    CK(cudaMemcpy2DAsync(dst.cb, sc, cb, cbs, W / 2, H / 2, kind, st));
    CK(cudaMemcpy2DAsync(dst.cr, sc, cr, crs, W / 2, H / 2, kind, st));
    return true;
}

// Device-side copy of a frame (B-frame reorder buffer <-> working input).
bool EncImpl::dcopy(const DevFrame &dst, const DevFrame &src) {
    CK(cudaMemcpy2DAsync(dst.y, sy, src.y, sy, W, H, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpy2DAsync(dst.cb, sc, src.cb, sc, W / 2, H / 2, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpy2DAsync(dst.cr, sc, src.cr, sc, W / 2, H / 2, cudaMemcpyDeviceToDevice, st));
    return true;
}

// ---------------------------------------------------------------------------
// Frame driver, in stages so that many streams can share each CTU-engine
// launch (batched form): plan (B-frame schedule) -> stage_a (scene-cut
// histogram) -> stage_b (frame type, header fields, device parameters,
// global motion hint) -> wavefront launches -> stage_c (copy-back) ->
// commit_frame (DPB update and the other bookkeeping the next frame needs)
// -> stage_d (header, entropy coding, packet).  Single-stream encodes run
// the same stages back to back (reference src/encoder.c:2625-3121
// encode_poc_frame); a pipelined batch runs stage_d of one frame during the
// next frame's device step.
// ---------------------------------------------------------------------------
tc_error_t EncImpl::stage_a(int poc, int b_layer_qp_off) {
    pend.poc = poc;
    pend.qp_off = b_layer_qp_off;
    pend.need_hist = 0;
    if (!bf_b_mode) {
        const int kint = cfg.keyframe_interval > 0 ? cfg.keyframe_interval : 30;
        int is_key = force_keyframe || frame_count == 0;
        if (!is_key && frame_count % kint == 0) is_key = 1;
        if (!is_key && frame_count > 0) {
            if (launch_hist16(cur.y, W, H, sy, d_hist, st) != cudaSuccess) return TC_ERR_INTERNAL;
            ++kernel_launches;
            if (cudaMemcpyAsync(h_hist, d_hist, 16 * sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
                return TC_ERR_INTERNAL;
            pend.need_hist = 1;
        }
    }
    return TC_OK;
}

tc_error_t EncImpl::stage_b() {
    const int poc = pend.poc, b_layer_qp_off = pend.qp_off;
    // ---- frame type ----------------------------------------------------
    const int kint = cfg.keyframe_interval > 0 ? cfg.keyframe_interval : 30;
    int is_key;
    if (bf_b_mode) {
        is_key = force_keyframe || poc == 0 || (poc % kint == 0);
    } else {
        is_key = force_keyframe || frame_count == 0;
        if (!is_key && frame_count % kint == 0) is_key = 1;
        if (pend.need_hist) {
            // Scene cut: chi-square distance of 16-bin input histograms
            // (reference src/encoder.c:2650-2678).
            if (prev_hist_valid) {
                double dist = 0.0;
                const double total = (double)W * H;
                for (int i = 0; i < 16; ++i) {
                    const double expected = (prev_hist[i] + h_hist[i]) / 2.0;
                    if (expected > 0) {
                        const double diff = (double)h_hist[i] - (double)prev_hist[i];
                        dist += (diff * diff) / expected;
                    }
                }
                if (dist / total > 0.5) is_key = 1;
            }
            memcpy(prev_hist, h_hist, sizeof(prev_hist));
            prev_hist_valid = 1;
        }
    }
    force_keyframe = 0;
    const int frame_type = is_key ? 0 : (b_layer_qp_off > 0 ? 2 : 1);
    rc_frame_start();
    int qp = rc_qp;
    if (frame_type == 2) qp = clampi(qp + b_layer_qp_off, 0, 63);

    // ---- header fields (reference src/encoder.c:2713-2819, 2365-2399); the
    // header is written with the frame's entropy coding (stage_d), since its
    // entry-point flag depends on the previous frame's coded size
    int profile = cfg.profile, level = cfg.level_idx;
    if (profile > TC_PROFILE_MAX) profile = TC_PROFILE_BASELINE_MOBILE;
    if (level > TC_LEVEL_MAX) level = TC_LEVEL_AUTO;
    uint8_t flags = is_key ? TC_FLAG_KEY_FRAME : 0;
    if (is_key) flags |= TC_FLAG_RAP;
    if (cfg.enable_crc) flags |= TC_FLAG_CRC;
    uint16_t tools = TC_TOOL_SKIP_MERGE | TC_TOOL_CFL_CHROMA | TC_TOOL_JND_WEIGHTING |
                     TC_TOOL_MEDIAN_MV_PRED | TC_TOOL_SIX_TAP_INTERP;
    if (cfg.preset >= TC_PRESET_MEDIUM && profile >= TC_PROFILE_STREAMING_MAIN) tools |= TC_TOOL_MULTI_REF;
    if (cfg.enable_entropy_coded) tools |= TC_TOOL_ENTROPY_CODED;
    if (frame_type == 2) tools |= TC_TOOL_BIPRED;
    tools |= TC_TOOL_SAO;
    if (cfg.preset >= TC_PRESET_MEDIUM) tools |= TC_TOOL_FRESH_SKIP;
    if (bf_b_mode) flags |= TC_FLAG_EXT_HEADER;
    pend.hdr_flags = flags;
    pend.hdr_tools = tools;
    pend.hdr_pl = (profile << 4) | (level & 0x0F);

    if (is_key && poc > 0)
        for (int i = 0; i < TC_REF_FRAMES; ++i) { dpb_slot[i] = -1; dpb_poc[i] = -1; }

    // ---- device frame parameters ------------------------------------------
    const int rs = free_pool_slot();
    if (rs < 0) return TC_ERR_INTERNAL;
    if (legacy) return stage_b_legacy(is_key, frame_type, qp, rs);
    const DevFrame rec = pool[rs];
    FrameParams &P = h_params;
    memset(&P, 0, sizeof(P));
    P.W = W; P.H = H; P.stride_y = sy; P.stride_c = sc;
    P.ctu_cols = ctu_cols; P.ctu_rows = ctu_rows; P.grid_w = grid_w; P.grid_h = grid_h;
    P.cur_y = cur.y; P.cur_cb = cur.cb; P.cur_cr = cur.cr;
    P.rec_y = rec.y; P.rec_cb = rec.cb; P.rec_cr = rec.cr;
    for (int i = 0; i < MAX_REFS; ++i) {
        const int s = dpb_slot[i];
        P.ref_valid[i] = s >= 0;
        P.ref_poc[i] = dpb_poc[i];
        const DevFrame &f = s >= 0 ? pool[s] : pool[rs];
        P.ref_y[i] = f.y; P.ref_cb[i] = f.cb; P.ref_cr[i] = f.cr;
    }
    P.prev_grid = grid[1 - grid_cur];
    P.cur_grid = grid[grid_cur];
    P.out = d_out;
    P.frame_type = frame_type;
    P.poc = poc;
    P.qp = qp;
    P.qp_c = clampi(qp + 1, 0, 63);
    P.preset = cfg.preset;
    P.multiref = cfg.preset >= TC_PRESET_MEDIUM && profile >= TC_PROFILE_STREAMING_MAIN && frame_type == 1;
    P.fresh_skip = cfg.preset >= TC_PRESET_MEDIUM;
    P.prev_valid = prev_mv_valid;
    P.glob_valid = 0;
    long long lam = tc_lambda_host(qp);
    if (frame_type == 0) lam = (lam * 3) / 4;
    P.lambda = lam;
    P.lambda_c = tc_lambda_host(P.qp_c);
    P.lambda_sao = tc_lambda_host(qp);
    for (int b = 0; b < 4; ++b) {
        P.eff_l[b] = eff_scale(qp, b); P.rcp_l[b] = quant_rcp(P.eff_l[b]);
        P.eff_c[b] = eff_scale(P.qp_c, b); P.rcp_c[b] = quant_rcp(P.eff_c[b]);
    }
    P.err = d_err;
    P.done = d_done;
    P.epoch = ++epoch;
    P.search_window = engine_tuning(W, H).search_window;
    *h_params_pin = P;   // the previous frame's upload has completed (every step ends synchronised)
    if (cudaMemcpyAsync(d_params, h_params_pin, sizeof(P), cudaMemcpyHostToDevice, st) != cudaSuccess)
        return TC_ERR_INTERNAL;
    pend.glob = frame_type == 1 && P.ref_valid[0];
    pend.glob_ref = P.ref_y[0];
    if (pend.glob && !defer_glob) {
        if (launch_glob_mv(cur.y, P.ref_y[0], W, H, sy, d_params, st) != cudaSuccess) return TC_ERR_INTERNAL;
        ++kernel_launches;
    }
    pend.is_key = is_key;
    pend.frame_type = frame_type;
    pend.qp = qp;
    pend.rs = rs;
    pend.multiref = P.multiref;
    return TC_OK;
}

// Legacy frame parameters (reference src/encoder.c:1648-1677 candidate
// references, 1646-1648 search range, 1846 lambda).
tc_error_t EncImpl::stage_b_legacy(int is_key, int frame_type, int qp, int rs) {
    const DevFrame rec = pool[rs];
    legacy::LFrame &F = lframe;
    memset(&F, 0, sizeof(F));
    F.W = W; F.H = H; F.sy = sy; F.sc = sc; F.ctu_cols = ctu_cols; F.ctu_rows = ctu_rows;
    F.cur_y = cur.y; F.cur_cb = cur.cb; F.cur_cr = cur.cr;
    F.rec_y = rec.y; F.rec_cb = rec.cb; F.rec_cr = rec.cr;
    for (int i = 0; i < TC_REF_FRAMES; ++i) F.dpb_y[i] = dpb_slot[i] >= 0 ? pool[dpb_slot[i]].y : nullptr;
    if (frame_type == 2) {
        // Forward: the largest POC below this frame's; backward: the
        // smallest above (reference src/encoder.c:204-228).
        int fp = -1, bp = 0x7FFFFFFF;
        for (int i = 0; i < TC_REF_FRAMES; ++i) {
            const int sl = dpb_slot[i], p = dpb_poc[i];
            if (sl < 0 || p < 0) continue;
            if (p < pend.poc && p > fp) { fp = p; F.fwd_y = pool[sl].y; }
            if (p > pend.poc && p < bp) { bp = p; F.bwd_y = pool[sl].y; }
        }
        if (F.fwd_y) { F.cand_y[F.n_cand] = F.fwd_y; F.cand_sel[F.n_cand] = 0; F.n_cand++; }
        if (F.bwd_y) { F.cand_y[F.n_cand] = F.bwd_y; F.cand_sel[F.n_cand] = 1; F.n_cand++; }
    } else if (frame_type == 1) {
        const int max_refs = (cfg.preset == TC_PRESET_SLOW && cfg.profile >= TC_PROFILE_STREAMING_MAIN) ? TC_REF_FRAMES : 1;
        for (int ri = 0; ri < max_refs && F.n_cand < 2; ++ri)
            if (dpb_slot[ri] >= 0) { F.cand_y[F.n_cand] = pool[dpb_slot[ri]].y; F.cand_sel[F.n_cand] = ri; F.n_cand++; }
    }
    F.frame_type = frame_type;
    F.qp = qp;
    F.search_range = cfg.preset == TC_PRESET_ULTRAFAST ? 16 : (cfg.preset == TC_PRESET_SLOW ? 64 : 32);
    F.lambda = tc_lambda_host(qp);
    F.blocks = d_lblk;
    pend.glob = 0;
    pend.is_key = is_key;
    pend.frame_type = frame_type;
    pend.qp = qp;
    pend.rs = rs;
    pend.multiref = 0;
    return TC_OK;
}

// The new reconstruction starts as a copy of the previous one, then the
// legacy CTU wavefront runs one diagonal per launch.
tc_error_t EncImpl::launch_legacy() {
    const DevFrame rec = pool[pend.rs];
    if (timing) cudaEventRecord(ev0, st);
    if (prev_rs >= 0 && prev_rs != pend.rs) {
        const DevFrame &pv = pool[prev_rs];
        if (cudaMemcpyAsync(rec.y, pv.y, (size_t)sy * H, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(rec.cb, pv.cb, (size_t)sc * (H / 2), cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(rec.cr, pv.cr, (size_t)sc * (H / 2), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            return TC_ERR_INTERNAL;
    }
    for (size_t d = 0; d < ldiag_off.size(); ++d)
        if (launch_legacy_ctus(lframe, d_litems + ldiag_off[d], ldiag_cnt[d], true, st) != cudaSuccess)
            return TC_ERR_INTERNAL;
    kernel_launches += (long long)ldiag_off.size();
    if (timing) cudaEventRecord(ev1, st);
    return TC_OK;
}

tc_error_t EncImpl::launch_own() {
    if (legacy) return launch_legacy();
    if (timing) cudaEventRecord(ev0, st);
    if (persistent) {
        if (cudaMemsetAsync(d_ctrl, 0, 2 * sizeof(int), st) != cudaSuccess ||
            launch_ctu_persistent(d_params, d_items, ctu_cols * ctu_rows, d_ctrl, num_sms, st) != cudaSuccess)
            return TC_ERR_INTERNAL;
        kernel_launches += 1;
    } else {
        for (size_t d = 0; d < diag_off.size(); ++d)
            if (launch_ctu_items(d_params, d_items + diag_off[d], diag_cnt[d], st) != cudaSuccess)
                return TC_ERR_INTERNAL;
        kernel_launches += (long long)diag_off.size();
    }
    if (timing) cudaEventRecord(ev1, st);
    return TC_OK;
}

tc_error_t EncImpl::stage_c(bool with_recon) {
    const int nctu = ctu_cols * ctu_rows;
    const DevFrame rec = pool[pend.rs];
    if (legacy) {
        if (cudaMemcpyAsync(h_lblk, d_lblk, sizeof(legacy::LBlock) * (size_t)nctu * legacy::BLOCKS,
                            cudaMemcpyDeviceToHost, st) != cudaSuccess)
            return TC_ERR_INTERNAL;
    } else if (cudaMemcpyAsync(h_out, d_out, sizeof(CtuOut) * nctu, cudaMemcpyDeviceToHost, st) != cudaSuccess) {
        return TC_ERR_INTERNAL;
    }
    if (launch_frame_sse(cur.y, rec.y, W, H, sy, d_sse, st) != cudaSuccess) return TC_ERR_INTERNAL;
    ++kernel_launches;
    if (cudaMemcpyAsync(h_sse, d_sse, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(h_ctrl, d_ctrl, 2 * sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return TC_ERR_INTERNAL;
    return with_recon ? readback_recon() : TC_OK;
}

// Host copy of the reconstruction (tc_encoder_t.recon), when enabled.
tc_error_t EncImpl::readback_recon() {
    const DevFrame rec = pool[pend.rs];
    if (recon_host && recon_readback) {
        if (cudaMemcpy2DAsync(recon_host->y, recon_host->stride_y, rec.y, sy, W, H, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaMemcpy2DAsync(recon_host->cb, recon_host->stride_c, rec.cb, sc, W / 2, H / 2, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaMemcpy2DAsync(recon_host->cr, recon_host->stride_c, rec.cr, sc, W / 2, H / 2, cudaMemcpyDeviceToHost, st) != cudaSuccess)
            return TC_ERR_INTERNAL;
    }
    return TC_OK;
}

// Second record / packet buffers for pipelined batches (constant QP only:
// with rate control a frame's QP depends on the previous frame's bits).
bool EncImpl::set_pipelined(bool on) {
    if (on && rc_method != TC_RC_CQP) return false;
    if (on && !h_out_alt) {
        if (pinned_alloc(&h_out_alt, sizeof(CtuOut) * (size_t)ctu_cols * ctu_rows) != cudaSuccess) {
            h_out_alt = nullptr;
            return false;
        }
        out_buf_alt = (uint8_t *)calloc(out_buf_size, 1);
        if (!out_buf_alt) return false;
    }
    pipelined = on;
    return true;
}

// After the frame's device step has completed: the device's error word,
// then the sequence bookkeeping the next frame's planning depends on (DPB
// shift, temporal MV grid, frame count, reorder buffer), and the frame's
// entropy-coding job (its pending state, records and SSE) for stage_d.  A
// pipelined encoder switches to its second record and packet buffers here,
// so the next device step can land while this frame is entropy coded.
tc_error_t EncImpl::commit_frame() {
    if (!legacy && persistent && h_ctrl[1]) return TC_ERR_INTERNAL;   // a bounded wait expired on the device
    ent.p = pend;
    ent.sse = *h_sse;
    ent.rec = h_out;
    ent.lrec = h_lblk;
    prev_rs = pend.rs;
    ent.buf = out_buf;
    ent_ready = true;
    // DPB shift: slot 3 falls out, the new reconstruction enters slot 0
    // (reference src/encoder.c:3085-3097).
    for (int i = TC_REF_FRAMES - 1; i > 0; --i) { dpb_slot[i] = dpb_slot[i - 1]; dpb_poc[i] = dpb_poc[i - 1]; }
    dpb_slot[0] = pend.rs;
    dpb_poc[0] = pend.poc;
    frame_count++;
    grid_cur = 1 - grid_cur;   // this frame's grid becomes the temporal predictor
    prev_mv_valid = 1;
    if (pend.bf_idx >= 0) {
        bf_free.push_back(bf_frames[pend.bf_idx]);   // back to the reorder pool
        bf_frames.erase(bf_frames.begin() + pend.bf_idx);
        bf_pocs.erase(bf_pocs.begin() + pend.bf_idx);
        pend.bf_idx = -1;
    }
    if (pipelined) {
        std::swap(h_out, h_out_alt);
        std::swap(out_buf, out_buf_alt);
    }
    return TC_OK;
}

// Header, entropy coding of the committed frame's CTU records, CRC and the
// packet (reference src/encoder.c:2713-2819, 2906-2965).
tc_error_t EncImpl::stage_d(tc_packet_t *pkt) {
    if (!ent_ready) return TC_ERR_INTERNAL;
    ent_ready = false;
    if (legacy) return stage_d_legacy(pkt);
    const Pending &pd = ent.p;
    const int poc = pd.poc, is_key = pd.is_key, frame_type = pd.frame_type, qp = pd.qp, multiref = pd.multiref;
    const CtuOut *rec_out = ent.rec;
    uint8_t *const buf = ent.buf;
    const int use_ep = !prev_v2_valid || prev_v2_rowbytes >= 256;
    memset(buf, 0, out_buf_size);
    fbw.init(buf, out_buf_size);
    BitWriter &bw = fbw;
    bw.put_bits(TC_MAGIC_0, 8); bw.put_bits(TC_MAGIC_1, 8); bw.put_bits(TC_MAGIC_2, 8);
    bw.put_bits(TC_VERSION_V2, 8);
    bw.put_bits((uint32_t)(uint16_t)W, 16); bw.put_bits((uint32_t)(uint16_t)H, 16);
    bw.put_bits(pd.hdr_flags, 8);
    bw.put_bits((uint8_t)(int8_t)(qp - TC_QP_DEFAULT), 8);
    bw.put_bits((uint8_t)(poc & 0xFF), 8);
    bw.put_bits((uint8_t)pd.hdr_pl, 8);
    bw.put_bits((uint16_t)(pd.hdr_tools | (use_ep ? TC_TOOL_ENTRY_POINTS : 0)), 16);
    if (bf_b_mode) bw.put_bits(frame_type == 0 ? 0 : (frame_type == 2 ? 2 : 1), 8);
    bw.align();
    const int entropy = cfg.enable_entropy_coded ? 1 : 0;
    if (use_ep) {
        // Entry-point rows (reference src/encoder.c:2906-2965).
        const int nrows = ctu_rows;
        bw.put_bits((uint32_t)nrows, 16);
        const size_t ep_table = bw.byte_pos;
        for (int i = 0; i < nrows; ++i) bw.put_bits(0, 32);
        bw.align();
        const size_t ep_payload = bw.byte_pos;
        const size_t per_row = out_buf_size / (size_t)(nrows > 1 ? nrows : 1) + 1024;
        if (nrows > 64) return TC_ERR_MEMORY;
        // Every row is coded into its own slot of row_buf (rows spread over
        // the encoder's entropy threads), then the rows are laid out in
        // order: the same bytes as coding them one after another.
        if (row_buf.size() < per_row * (size_t)nrows) row_buf.resize(per_row * (size_t)nrows);
        size_t row_bytes[64];
        bool row_bad[64];
        auto code_rows = [&](int first, int step) {
            for (int r = first; r < nrows; r += step) {
                BitWriter rw;
                rw.init(row_buf.data() + (size_t)r * per_row, per_row);
                RangeEncoder rc;
                uint8_t ctx[TC_NUM_CONTEXTS_RC];
                memset(ctx, 0, sizeof(ctx));
                rc.init(&rw);
                SyntaxSink sink{&rw, entropy ? &rc : nullptr, ctx};
                for (int c = 0; c < ctu_cols; ++c) {
                    const CtuGeom g{c * 64, r * 64, W, H, frame_type, multiref};
                    write_ctu_syntax(sink, rec_out[r * ctu_cols + c], g);
                }
                if (entropy) rc.flush();
                rw.align();
                row_bad[r] = rw.overflow;
                row_bytes[r] = rw.bytes();
            }
        };
        const int nth = std::max(1, std::min(entropy_threads, nrows));
        if (nth > 1) {
            std::vector<std::thread> th;
            for (int t = 1; t < nth; ++t) th.emplace_back(code_rows, t, nth);
            code_rows(0, nth);
            for (auto &x : th) x.join();
        } else {
            code_rows(0, 1);
        }
        uint32_t row_off[64];
        for (int r = 0; r < nrows; ++r) {
            if (row_bad[r]) return TC_ERR_MEMORY;
            const size_t rb = row_bytes[r];
            if (rb > per_row || bw.byte_pos + rb > out_buf_size) return TC_ERR_MEMORY;
            row_off[r] = (uint32_t)(bw.byte_pos - ep_payload);
            memcpy(buf + bw.byte_pos, row_buf.data() + (size_t)r * per_row, rb);
            bw.byte_pos += rb;
        }
        for (int i = 0; i < nrows; ++i) {
            uint8_t *p = buf + ep_table + (size_t)i * 4;
            p[0] = (uint8_t)(row_off[i] >> 24); p[1] = (uint8_t)(row_off[i] >> 16);
            p[2] = (uint8_t)(row_off[i] >> 8);  p[3] = (uint8_t)row_off[i];
        }
    } else {
        RangeEncoder rc;
        uint8_t ctx[TC_NUM_CONTEXTS_RC];
        memset(ctx, 0, sizeof(ctx));
        rc.init(&bw);
        SyntaxSink sink{&bw, entropy ? &rc : nullptr, ctx};
        for (int r = 0; r < ctu_rows; ++r)
            for (int c = 0; c < ctu_cols; ++c) {
                const CtuGeom g{c * 64, r * 64, W, H, frame_type, multiref};
                write_ctu_syntax(sink, rec_out[r * ctu_cols + c], g);
            }
        if (entropy) rc.flush();
        bw.align();
    }
    if (cfg.enable_crc) {
        const uint16_t crc = crc16_ccitt(buf, bw.bytes());
        bw.put_bits(crc >> 8, 8);
        bw.put_bits(crc & 0xFF, 8);
    }
    if (bw.overflow) return TC_ERR_MEMORY;
    const size_t frame_bytes = bw.bytes();
    rc_frame_end((long long)frame_bytes * 8);
    if (ctu_rows > 0) { prev_v2_rowbytes = frame_bytes / (size_t)ctu_rows; prev_v2_valid = 1; }

    // PSNR statistic (reference src/tcodec.c:34-54) from the device SSE.
    const unsigned long long sse = ent.sse;
    double psnr = 100.0;
    if (sse) {
        const double mse = (double)sse / ((double)W * (double)H);
        psnr = 10.0 * log10(255.0 * 255.0 / mse);
    }
    sum_psnr += psnr;
    pkt->data = buf;
    pkt->size = frame_bytes;
    pkt->pts = poc;
    pkt->key_frame = is_key;
    total_bytes += (long long)frame_bytes;
    total_frames++;
    return TC_OK;
}

// Legacy packet (reference src/encoder.c:2713-3121 for use_v2 == 0).
tc_error_t EncImpl::stage_d_legacy(tc_packet_t *pkt) {
    const Pending &pd = ent.p;
    const LegacyFrameSyntax h = legacy_frame_syntax(cfg, pd.is_key, pd.frame_type, pd.qp, pd.poc, bf_b_mode != 0,
                                                    legacy_wpp);
    const size_t frame_bytes = write_legacy_frame(ent.buf, out_buf_size, h, ent.lrec, ctu_cols, ctu_rows, row_buf);
    if (!frame_bytes) return TC_ERR_MEMORY;
    rc_frame_end((long long)frame_bytes * 8);
    const unsigned long long sse = ent.sse;
    double psnr = 100.0;
    if (sse) {
        const double mse = (double)sse / ((double)W * (double)H);
        psnr = 10.0 * log10(255.0 * 255.0 / mse);
    }
    sum_psnr += psnr;
    pkt->data = ent.buf;
    pkt->size = frame_bytes;
    pkt->pts = pd.poc;
    pkt->key_frame = pd.is_key;
    total_bytes += (long long)frame_bytes;
    total_frames++;
    return TC_OK;
}

tc_error_t EncImpl::encode_planned(tc_packet_t *pkt) {
    tc_error_t r = stage_a(pend.poc, pend.qp_off);
    if (r != TC_OK) return r;
    if (pend.need_hist && cudaStreamSynchronize(st) != cudaSuccess) return TC_ERR_INTERNAL;
    if ((r = stage_b()) != TC_OK) return r;
    if ((r = launch_own()) != TC_OK) return r;
    if ((r = stage_c()) != TC_OK) return r;
    if (cudaStreamSynchronize(st) != cudaSuccess) return TC_ERR_INTERNAL;
    if (timing) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev0, ev1);
        ctu_ms += ms;
        ctu_launches += (long long)(legacy ? ldiag_off.size() : diag_off.size());
        ctu_count += (long long)ctu_cols * ctu_rows;
        frames_timed++;
    }
    if ((r = commit_frame()) != TC_OK) return r;
    return stage_d(pkt);
}

// Frame parameters of the CTU engine from the public frame descriptor
// (same derivations as stage_b: multiref / fresh-skip tool conditions,
// keyframe lambda scaling, per-band quant steps).
bool tcb::frame_params_from_desc(const tcb_frame_desc_t &d, FrameParams &P) {
    if (d.width <= 0 || d.height <= 0 || (d.width & 1) || (d.height & 1) || d.width > TC_MAX_WIDTH ||
        d.height > TC_MAX_HEIGHT || d.stride_y < d.width || d.stride_c < d.width / 2 || !d.src_y || !d.src_cb ||
        !d.src_cr || !d.rec_y || !d.rec_cb || !d.rec_cr || !d.cur_mv_grid || !d.ctu_records ||
        d.frame_type < 0 || d.frame_type > 2 || d.qp < 0 || d.qp > 63 || d.preset < 0 || d.preset > 3)
        return false;
    memset(&P, 0, sizeof(P));
    P.W = d.width; P.H = d.height; P.stride_y = d.stride_y; P.stride_c = d.stride_c;
    P.ctu_cols = (d.width + 63) / 64; P.ctu_rows = (d.height + 63) / 64;
    P.grid_w = (d.width + 7) / 8; P.grid_h = (d.height + 7) / 8;
    P.cur_y = d.src_y; P.cur_cb = d.src_cb; P.cur_cr = d.src_cr;
    P.rec_y = d.rec_y; P.rec_cb = d.rec_cb; P.rec_cr = d.rec_cr;
    for (int i = 0; i < MAX_REFS; ++i) {
        const bool ok = d.ref_y[i] && d.ref_cb[i] && d.ref_cr[i];
        P.ref_valid[i] = ok;
        P.ref_poc[i] = ok ? d.ref_poc[i] : -1;
        P.ref_y[i] = ok ? d.ref_y[i] : d.src_y;
        P.ref_cb[i] = ok ? d.ref_cb[i] : d.src_cb;
        P.ref_cr[i] = ok ? d.ref_cr[i] : d.src_cr;
    }
    P.prev_valid = d.prev_mv_grid != nullptr;
    P.prev_grid = (const MvCell *)(d.prev_mv_grid ? d.prev_mv_grid : d.cur_mv_grid);
    P.cur_grid = (MvCell *)d.cur_mv_grid;
    P.out = (CtuOut *)d.ctu_records;
    P.frame_type = d.frame_type;
    P.poc = d.poc;
    P.qp = d.qp;
    P.qp_c = clampi(d.qp + 1, 0, 63);
    P.preset = d.preset;
    const int profile = d.profile > TC_PROFILE_MAX ? TC_PROFILE_BASELINE_MOBILE : d.profile;
    P.multiref = d.preset >= TC_PRESET_MEDIUM && profile >= TC_PROFILE_STREAMING_MAIN && d.frame_type == 1;
    P.fresh_skip = d.preset >= TC_PRESET_MEDIUM;
    P.glob_valid = d.global_mv_valid ? 1 : 0;
    P.glob_x = d.global_mv_x;
    P.glob_y = d.global_mv_y;
    long long lam = tc_lambda_host(d.qp);
    if (d.frame_type == 0) lam = (lam * 3) / 4;
    P.lambda = lam;
    P.lambda_c = tc_lambda_host(P.qp_c);
    P.lambda_sao = tc_lambda_host(d.qp);
    for (int b = 0; b < 4; ++b) {
        P.eff_l[b] = eff_scale(d.qp, b); P.rcp_l[b] = quant_rcp(P.eff_l[b]);
        P.eff_c[b] = eff_scale(P.qp_c, b); P.rcp_c[b] = quant_rcp(P.eff_c[b]);
    }
    P.search_window = engine_tuning(d.width, d.height).search_window;
    return true;
}

long long tcb::tc_lambda_host(int qp) {
    const long long s = qscale(qp);
    long long l = (s * s * 200) >> 10;
    if (l < 1) l = 1;
    if (l > (1ll << 30)) l = 1ll << 30;
    return l;
}

// ---------------------------------------------------------------------------
// B-frame reorder (reference src/encoder.c:3132-3277): display-order inputs
// wait in device buffers and are emitted in coding order A(0), then per
// group A(4k), B(4k-2), B(4k-3), B(4k-1).
// ---------------------------------------------------------------------------
static int bf_schedule_poc(int p) {
    if (p == 0) return 0;
    const int k = (p + 3) / 4, c = (p - 1) % 4;
    static const int off[4] = {0, -2, -3, -1};
    return 4 * k + off[c];
}
static int bf_sched_qp_off(int p) {
    if (p == 0) return 0;
    const int c = (p - 1) % 4;
    if (c == 1) return 1;
    if (c == 2 || c == 3) return 2;
    return 0;
}
static int bf_anchor_slot(int p) { return p == 0 ? 0 : p - ((p - 1) % 4); }

int EncImpl::bf_find(int poc) const {
    for (size_t i = 0; i < bf_pocs.size(); ++i)
        if (bf_pocs[i] == poc) return (int)i;
    return -1;
}
bool EncImpl::bf_can_emit() const {
    if (bf_pocs.empty()) return false;
    const int p = bf_emit_pos;
    if (bf_find(bf_schedule_poc(p)) < 0) return false;
    if (p == 0) return true;
    if ((p - 1) % 4 == 0) return true;
    return bf_emit_pos > bf_anchor_slot(p);
}
tc_error_t EncImpl::bf_push_current() {
    if (bf_pocs.size() >= BF_MAX || bf_free.empty()) return TC_OK;
    DevFrame f = bf_free.back();
    bf_free.pop_back();
    if (!dcopy(f, cur)) return TC_ERR_INTERNAL;
    bf_frames.push_back(f);
    bf_pocs.push_back(bf_next_input);
    return TC_OK;
}

// Schedule the next coding-order frame from the reorder buffer into `cur`.
tc_error_t EncImpl::bf_plan_scheduled() {
    const int p = bf_emit_pos;
    const int poc = bf_schedule_poc(p);
    const int idx = bf_find(poc);
    bf_emit_pos++;
    if (!dcopy(cur, bf_frames[idx])) return TC_ERR_INTERNAL;
    pend.poc = poc;
    pend.qp_off = bf_sched_qp_off(p);
    pend.bf_idx = idx;
    return TC_OK;
}

// One input frame is staged in `cur`: decide whether it produces a coded
// frame now (TC_OK, pend filled) or waits for the B-frame schedule
// (TC_ERR_NEED_MORE) (reference src/encoder.c:3181-3212).
tc_error_t EncImpl::plan_input() {
    pend.bf_idx = -1;
    if (bf_b_mode) {
        const tc_error_t r = bf_push_current();
        if (r != TC_OK) return r;
        bf_next_input++;
        if (!bf_can_emit()) return TC_ERR_NEED_MORE;
        return bf_plan_scheduled();
    }
    pend.poc = frame_count;
    pend.qp_off = 0;
    return TC_OK;
}

// Tail drain (reference src/encoder.c:3256-3277): TC_OK with pend filled,
// or TC_ERR_EOF.
tc_error_t EncImpl::plan_flush() {
    pend.bf_idx = -1;
    if (!bf_b_mode) return TC_ERR_EOF;
    if (bf_can_emit()) return bf_plan_scheduled();
    if (!bf_pocs.empty()) {
        int best = 0;
        for (size_t i = 1; i < bf_pocs.size(); ++i)
            if (bf_pocs[i] < bf_pocs[best]) best = (int)i;
        if (!dcopy(cur, bf_frames[best])) return TC_ERR_INTERNAL;
        pend.poc = bf_pocs[best];
        pend.qp_off = 0;
        pend.bf_idx = best;
        return TC_OK;
    }
    return TC_ERR_EOF;
}

tc_error_t EncImpl::encode_input(tc_packet_t *out) {
    const tc_error_t r = plan_input();
    if (r != TC_OK) return r;
    return encode_planned(out);
}

// ---------------------------------------------------------------------------
// Public API
// ---------------------------------------------------------------------------
tc_encoder_t *tcb::encoder_create(const tc_config_t *config, DeviceArena *arena) {
    if (!config) return nullptr;
    if (config->width <= 0 || config->height <= 0 || (config->width & 1) || (config->height & 1) ||
        config->width > TC_MAX_WIDTH || config->height > TC_MAX_HEIGHT)
        return nullptr;
    tc_encoder_t *enc = (tc_encoder_t *)calloc(1, sizeof(tc_encoder_t));
    if (!enc) return nullptr;
    enc->cfg = *config;
    enc->impl = new (std::nothrow) EncImpl();
    if (enc->impl) enc->impl->arena = arena;
    if (!enc->impl || !enc->impl->init(*config)) {
        tc_encoder_destroy(enc);
        return nullptr;
    }
    enc->cur = tcb_host_frame_alloc(config->width, config->height, 0);
    enc->recon = tcb_host_frame_alloc(config->width, config->height, 1);
    if (!enc->cur || !enc->recon) { tc_encoder_destroy(enc); return nullptr; }
    enc->impl->recon_host = enc->recon;
    const unsigned hw = std::thread::hardware_concurrency();
    enc->impl->entropy_threads = (int)std::min(8u, hw ? hw : 1u);
    return enc;
}

extern "C" {

tc_encoder_t *tc_encoder_create(const tc_config_t *config) { return tcb::encoder_create(config, nullptr); }

void tc_encoder_destroy(tc_encoder_t *enc) {
    if (!enc) return;
    if (enc->impl) { enc->impl->release(); delete enc->impl; }
    tcb_host_frame_free(enc->cur);
    tcb_host_frame_free(enc->recon);
    free(enc);
}

tc_error_t tc_encoder_encode(tc_encoder_t *enc, const tc_pixel_t *y, int stride_y,
                             const tc_pixel_t *cb, int stride_cb, const tc_pixel_t *cr,
                             int stride_cr, tc_packet_t *packet_out) {
    if (packet_out) memset(packet_out, 0, sizeof(*packet_out));   // empty unless a packet is produced
    if (!enc || !enc->impl || !y || !cb || !cr || !packet_out) return TC_ERR_PARAM;
    EncImpl &e = *enc->impl;
    if (cudaSetDevice(e.device) != cudaSuccess) return TC_ERR_INTERNAL;
    if (!e.upload(y, stride_y, cb, stride_cb, cr, stride_cr, e.cur)) return TC_ERR_INTERNAL;
    return e.encode_input(packet_out);
}

tc_error_t tcb_encoder_encode_device(tc_encoder_t *enc, const tc_pixel_t *d_y, int stride_y,
                                     const tc_pixel_t *d_cb, int stride_cb, const tc_pixel_t *d_cr,
                                     int stride_cr, tc_packet_t *packet_out) {
    if (packet_out) memset(packet_out, 0, sizeof(*packet_out));
    if (!enc || !enc->impl || !d_y || !d_cb || !d_cr || !packet_out) return TC_ERR_PARAM;
    EncImpl &e = *enc->impl;
    if (cudaSetDevice(e.device) != cudaSuccess) return TC_ERR_INTERNAL;
    if (!e.upload(d_y, stride_y, d_cb, stride_cb, d_cr, stride_cr, e.cur, cudaMemcpyDeviceToDevice))
        return TC_ERR_INTERNAL;
    return e.encode_input(packet_out);
}

void *tcb_encoder_stream(tc_encoder_t *enc) { return enc && enc->impl ? (void *)enc->impl->st : nullptr; }

void tcb_encoder_set_timing(tc_encoder_t *enc, int enabled) {
    if (enc && enc->impl) enc->impl->timing = enabled != 0;
}

void tcb_encoder_get_timing(tc_encoder_t *enc, double *ctu_ms, int64_t *ctu_launches, int64_t *ctu_count,
                            int64_t *frames, int64_t *kernel_launches) {
    if (!enc || !enc->impl) return;
    EncImpl &e = *enc->impl;
    if (kernel_launches) *kernel_launches = e.kernel_launches;
    e.kernel_launches = 0;
    if (ctu_ms) *ctu_ms = e.ctu_ms;
    if (ctu_launches) *ctu_launches = e.ctu_launches;
    if (ctu_count) *ctu_count = e.ctu_count;
    if (frames) *frames = e.frames_timed;
    e.ctu_ms = 0.0; e.ctu_launches = 0; e.ctu_count = 0; e.frames_timed = 0;
}

void tcb_encoder_set_recon_readback(tc_encoder_t *enc, int enabled) {
    if (enc && enc->impl) enc->impl->recon_readback = enabled != 0;
}

void tcb_encoder_set_entropy_threads(tc_encoder_t *enc, int threads) {
    if (enc && enc->impl) enc->impl->entropy_threads = std::max(1, std::min(64, threads));
}

tc_error_t tc_encoder_flush_tail(tc_encoder_t *enc, tc_packet_t *packet_out) {
    if (packet_out) memset(packet_out, 0, sizeof(*packet_out));
    if (!enc || !enc->impl || !packet_out) return TC_ERR_PARAM;
    EncImpl &e = *enc->impl;
    if (!e.bf_b_mode) return TC_ERR_EOF;
    if (cudaSetDevice(e.device) != cudaSuccess) return TC_ERR_INTERNAL;
    const tc_error_t r = e.plan_flush();
    if (r != TC_OK) return r;
    return e.encode_planned(packet_out);
}

void tc_encoder_force_keyframe(tc_encoder_t *enc) {
    if (enc && enc->impl) enc->impl->force_keyframe = 1;
}

void tc_encoder_get_stats(tc_encoder_t *enc, int64_t *total_bytes, int32_t *total_frames,
                          double *avg_psnr) {
    if (!enc || !enc->impl) return;
    const EncImpl &e = *enc->impl;
    if (total_bytes) *total_bytes = (int32_t)e.total_bytes;
    if (total_frames) *total_frames = e.total_frames;
    if (avg_psnr) *avg_psnr = e.total_frames > 0 ? e.sum_psnr / e.total_frames : 0.0;
}

}  // extern "C"
