// tcb_encoder.h — private encoder state of libtcodec_b200.
#pragma once
#include <stddef.h>
#include <stdint.h>

#include <new>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/tcodec.h"
#include "../../include/tcodec_b200.h"
#include "tcb_arena.h"
#include "tcb_common.cuh"
#include "tcb_entropy.h"
#include "tcb_legacy_types.h"

struct tc_encoder;

namespace tcb {

struct DevFrame {
    uint8_t *y = nullptr, *cb = nullptr, *cr = nullptr;
};

long long tc_lambda_host(int qp);
bool frame_params_from_desc(const tcb_frame_desc_t &d, FrameParams &P);

// Engine knobs of one frame size (tcb_engine_set_tuning; defaults when
// none were set): the search's SAD-table radius and the order in which a
// batch step merges its streams' CTU wavefronts.
struct EngineTuning {
    int search_window = 4;
    int queue_order = TCB_QUEUE_DIAGONAL;
};
EngineTuning engine_tuning(int width, int height);
void set_engine_tuning(int width, int height, const EngineTuning *t);

struct EncImpl {
    static constexpr int NPOOL = 6;   // 4 DPB slots + the frame being built + spare
    static constexpr size_t BF_MAX = 8;   // B-frame reorder buffers held at most
    tc_config_t cfg{};
    int W = 0, H = 0, sy = 0, sc = 0, ctu_cols = 0, ctu_rows = 0, grid_w = 0, grid_h = 0;
    int device = 0;
    cudaStream_t st = nullptr;         // stream all work is issued on
    cudaStream_t own_st = nullptr;     // the encoder's own stream
    cudaError_t last_cuda_error = cudaSuccess;
    DevFrame pool[NPOOL];
    DevFrame cur;
    int dpb_slot[TC_REF_FRAMES]{}, dpb_poc[TC_REF_FRAMES]{};
    int last_rec = -1;
    MvCell *grid[2] = {nullptr, nullptr};
    int grid_cur = 0;
    CtuOut *d_out = nullptr, *h_out = nullptr;
    FrameParams h_params{};
    FrameParams *h_params_pin = nullptr;   // pinned staging of h_params for the upload (capturable)
    FrameParams *d_params = nullptr;
    int *d_items = nullptr;
    std::vector<int> diag_off, diag_cnt;
    int *d_hist = nullptr, *h_hist = nullptr;
    unsigned long long *d_sse = nullptr, *h_sse = nullptr;
    int *d_err = nullptr;
    // persistent wavefront: per-CTU publish flags, queue counter + error word
    int *d_done = nullptr, *d_ctrl = nullptr, *h_ctrl = nullptr;
    int epoch = 0, num_sms = 148;
    bool persistent = true;
    tc_frame_buf_t *recon_host = nullptr;
    bool recon_readback = true;
    // optional CTU-engine timing
    bool timing = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double ctu_ms = 0.0;
    long long ctu_launches = 0, ctu_count = 0, frames_timed = 0, kernel_launches = 0;
    uint8_t *out_buf = nullptr;
    size_t out_buf_size = 0;
    // sequence state
    int frame_count = 0, force_keyframe = 0;
    int prev_hist[16]{}, prev_hist_valid = 0, prev_mv_valid = 0;
    size_t prev_v2_rowbytes = 0;
    int prev_v2_valid = 0;
    long long total_bytes = 0;
    int total_frames = 0;
    double sum_psnr = 0.0;
    // rate control
    int rc_method = 0, rc_qp = 32, rc_base_qp = 32;
    long long rc_frame_target = 0;
    double rc_buffer_size = 0.0, rc_buffer_level = 0.5;
    // B-frame reorder
    int bf_b_mode = 0, bf_emit_pos = 0, bf_next_input = 0;
    std::vector<DevFrame> bf_frames;   // occupied reorder buffers (with bf_pocs)
    std::vector<DevFrame> bf_free;     // unoccupied reorder buffers
    std::vector<int> bf_pocs;

    // Device memory comes from `arena` when set (served sessions), else
    // from cudaMalloc.
    DeviceArena *arena = nullptr;
    template <typename T> cudaError_t dmalloc(T **p, size_t n) {
        if (!arena) return dev_alloc(p, n);
        if (alloc_fault_now()) { *p = nullptr; return cudaErrorMemoryAllocation; }
        *p = (T *)arena->alloc(n);
        return *p ? cudaSuccess : cudaErrorMemoryAllocation;
    }
    void dfree(void *p) {
        if (!p) return;
        if (arena && arena->owns(p)) arena->release(p);
        else cudaFree(p);
    }
    // Device bytes a stream of configuration c holds at most (arena
    // granules; B-frame reorder buffers at their cap included).
    static size_t device_footprint(const tc_config_t &c);
    bool init(const tc_config_t &c);
    void release();
    int free_pool_slot() const;
    tc_error_t encode_input(tc_packet_t *out);
    bool upload(const tc_pixel_t *y, int ys, const tc_pixel_t *cb, int cbs, const tc_pixel_t *cr, int crs,
                const DevFrame &dst, cudaMemcpyKind kind = cudaMemcpyHostToDevice);
    bool dcopy(const DevFrame &dst, const DevFrame &src);
    // staged frame driver
    struct Pending {
        int poc = 0, qp_off = 0, need_hist = 0, is_key = 0, frame_type = 0, qp = 0,
            rs = -1, multiref = 0, bf_idx = -1, glob = 0;
        int hdr_flags = 0, hdr_tools = 0, hdr_pl = 0;   // frame header fields (entry-point bit added at coding)
        const uint8_t *glob_ref = nullptr;
    } pend;
    // The frame committed after its device step, awaiting entropy coding.
    struct EntropyJob {
        Pending p;
        unsigned long long sse = 0;
        const CtuOut *rec = nullptr;   // its decision records (host copy)
        const legacy::LBlock *lrec = nullptr;   // legacy path: its block records
        uint8_t *buf = nullptr;        // its packet buffer
    } ent;
    bool ent_ready = false;
    // Pipelined batches (constant QP only): second record and packet
    // buffers, swapped at every commit, so one frame is entropy coded while
    // the next one's device step runs.
    bool pipelined = false;
    CtuOut *h_out_alt = nullptr;
    uint8_t *out_buf_alt = nullptr;
    bool set_pipelined(bool on);
    // Batched streams leave the global-motion walk to the batch, which runs
    // every stream's walk in one launch on the batch's parameter copies.
    bool defer_glob = false;
    BitWriter fbw;
    std::vector<uint8_t> row_buf;
    // Legacy (v0 / v1) 8x8 block path (use_v2 == 0): block records on the
    // device and their host copies, the wavefront of diagonals c + 2r, the
    // pool slot of the previous reconstruction (the frame being coded
    // starts as its copy: the reference codes in place and reads samples of
    // not yet coded blocks from it) and whether rows are coded as separate
    // byte-aligned runs (the reference's WPP layout).
    bool legacy = false, legacy_wpp = false;
    legacy::LBlock *d_lblk = nullptr, *h_lblk = nullptr, *h_lblk_alt = nullptr;
    legacy::LFrame lframe{};
    int *d_litems = nullptr;
    std::vector<int> ldiag_off, ldiag_cnt;
    int prev_rs = -1;
    // Host threads that entropy-code one frame's entry-point rows (each row
    // is an independent range-coded substream). A lone encoder uses up to 8;
    // a batch or server codes each of its streams on its own thread and sets
    // its encoders to 1.
    int entropy_threads = 1;
    tc_error_t plan_input();
    tc_error_t plan_flush();
    tc_error_t stage_a(int poc, int b_layer_qp_off);
    tc_error_t stage_b();
    tc_error_t launch_own();
    tc_error_t stage_b_legacy(int is_key, int frame_type, int qp, int rs);
    tc_error_t launch_legacy();
    tc_error_t stage_d_legacy(tc_packet_t *pkt);
    tc_error_t stage_c(bool with_recon = true);   // copy-back; the host recon copy unless with_recon is false
    tc_error_t readback_recon();
    tc_error_t commit_frame();
    tc_error_t stage_d(tc_packet_t *pkt);
    tc_error_t encode_planned(tc_packet_t *pkt);
    tc_error_t bf_plan_scheduled();
    void rc_init(const tc_config_t &c);
    void rc_frame_start();
    void rc_frame_end(long long bits);
    int bf_find(int poc) const;
    bool bf_can_emit() const;
    tc_error_t bf_push_current();
};

// tc_encoder_create with the device memory taken from `arena` (NULL:
// cudaMalloc).
tc_encoder_t *encoder_create(const tc_config_t *config, DeviceArena *arena);

}  // namespace tcb

// Public handle.  The first three members keep the reference's
// tc_encoder_t prefix (tcodec_common.h:609-612) so callers that read
// encoder->recon after an encode (the reference test suite does) see the
// host copy of the reconstruction.
struct tc_encoder {
    tc_config_t cfg;
    tc_frame_buf_t *cur;
    tc_frame_buf_t *recon;
    tcb::EncImpl *impl;
};

extern "C" {
tc_frame_buf_t *tcb_host_frame_alloc(int width, int height, int pinned);
void tcb_host_frame_free(tc_frame_buf_t *f);
}
