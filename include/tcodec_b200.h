/*
 * tcodec_b200.h — B200-specific C ABI next to include/tcodec.h.
 *
 * Part 1: encoder extensions that have no counterpart in the reference
 *         (device-resident input, stream handle, kernel timing).
 * Part 2: batched standalone kernels of the v2 pixel pipeline.  Each one
 *         replaces a reference routine (cited per entry point) with an
 *         sm_100a kernel that processes many independent items per launch.
 *         All pointers are DEVICE pointers, all launches go on `stream`
 *         (a cudaStream_t, NULL = legacy default stream) and are
 *         asynchronous; the return value reports launch errors only
 *         (0 = OK, TC_ERR_PARAM for invalid sizes, TC_ERR_INTERNAL for a
 *         CUDA error).
 */
#ifndef TCODEC_B200_H
#define TCODEC_B200_H

#include "tcodec.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------
 * Part 1: encoder extensions (no reference counterpart).
 * ------------------------------------------------------------------- */

/* Same as tc_encoder_encode (reference tcodec.h:39-43) but the planes are
 * device pointers already resident in HBM; no host->device copy happens. */
tc_error_t tcb_encoder_encode_device(tc_encoder_t *enc,
                                     const tc_pixel_t *d_y, int stride_y,
                                     const tc_pixel_t *d_cb, int stride_cb,
                                     const tc_pixel_t *d_cr, int stride_cr,
                                     tc_packet_t *packet_out);

/* The CUDA stream (cudaStream_t) the encoder launches all its work on. */
void *tcb_encoder_stream(tc_encoder_t *enc);

/* Kernel timing: when enabled, CUDA events bracket every frame's
 * CTU-engine launches; totals accumulate until read (reading resets
 * them).  kernel_launches counts every kernel this encoder launched. */
void tcb_encoder_set_timing(tc_encoder_t *enc, int enabled);
void tcb_encoder_get_timing(tc_encoder_t *enc, double *ctu_ms, int64_t *ctu_launches,
                            int64_t *ctu_count, int64_t *frames, int64_t *kernel_launches);

/* Skip the per-frame device->host copy of the reconstruction into
 * encoder->recon (default on, as the reference keeps it current). */
void tcb_encoder_set_recon_readback(tc_encoder_t *enc, int enabled);

/* Host threads that entropy-code a frame's entry-point rows (frames of
 * more than one CTU row in entry-point mode code every row as its own
 * range-coded substream).  Clamped to [1, 64]; the packets do not depend
 * on it.  Default min(8, hardware threads) for tc_encoder_create, 1 for
 * the encoders of a batch or server, which code their streams in
 * parallel instead. */
void tcb_encoder_set_entropy_threads(tc_encoder_t *enc, int threads);

/* ---------------------------------------------------------------------
 * Batched form (no reference counterpart): N independent v2 streams that
 * advance one frame per call and share every CTU-engine launch.  Each
 * stream is an ordinary tc_encoder_t (tcb_batch_encoder) with its own
 * configuration, DPB and bitstream; packets are bit-identical to encoding
 * that stream alone.
 * ------------------------------------------------------------------- */
typedef struct tcb_batch tcb_batch_t;

/* One encoder per configs[i]; NULL on invalid config or device failure.
 * Batches run the v2 CTU engine: every config must set use_v2. */
tcb_batch_t *tcb_batch_create(const tc_config_t *configs, int n);
void tcb_batch_destroy(tcb_batch_t *batch);
int tcb_batch_size(tcb_batch_t *batch);
tc_encoder_t *tcb_batch_encoder(tcb_batch_t *batch, int i);
void *tcb_batch_stream(tcb_batch_t *batch);

/* Feed one frame to every stream i with y[i] != NULL (host pointers, or
 * device pointers when on_device != 0).  status[i] is TC_OK with
 * packets[i] filled, TC_ERR_NEED_MORE (no input or B-frame buffering), or
 * an error.  Packet data stays valid until the stream's next packet. */
tc_error_t tcb_batch_encode(tcb_batch_t *batch, const tc_pixel_t *const *y, const int *stride_y,
                            const tc_pixel_t *const *cb, const int *stride_cb,
                            const tc_pixel_t *const *cr, const int *stride_cr, int on_device,
                            tc_packet_t *packets, int *status);
/* Drain B-frame tails: TC_OK while any stream emitted (status per stream,
 * TC_ERR_EOF for drained ones), TC_ERR_EOF once all are drained. */
tc_error_t tcb_batch_flush(tcb_batch_t *batch, tc_packet_t *packets, int *status);

void tcb_batch_set_timing(tcb_batch_t *batch, int enabled);
void tcb_batch_get_timing(tcb_batch_t *batch, double *ctu_ms, int64_t *ctu_launches, int64_t *ctu_count,
                          int64_t *steps, int64_t *kernel_launches);
/* Host wall-clock split of the timed steps (timing enabled): planning and
 * launch, waiting for the device, entropy coding.  Reading resets. */
void tcb_batch_get_host_timing(tcb_batch_t *batch, double *plan_ms, double *wait_ms, double *entropy_ms);
/* CUDA-graph replay of each step's device work (default off): the step's
 * launch sequence (parameter uploads, global-motion kernel, work queue,
 * CTU engine, copy-back) is captured and replayed as one graph launch;
 * executable graphs are cached per step shape and updated in place with
 * the step's pointers.  Packets are identical either way.  graph_builds
 * counts instantiations, graph_launches replays; reading resets.  Returns
 * 0, or, for the last in-place update the runtime refused since the
 * previous read, 1000 * (cudaGraphNodeType + 1) + the node's position. */
void tcb_batch_set_graphs(tcb_batch_t *batch, int enabled);
/* Pipelined steps (default off; constant-QP streams only): each call
 * entropy-codes the previous call's frames on host threads while its own
 * frames run on the device, so packets arrive one call later (status
 * TC_OK with the previous frame's packet, TC_ERR_NEED_MORE otherwise);
 * tcb_batch_flush returns the last ones.  Packets are byte-identical to
 * the unpipelined batch, and tc_encoder_t.recon holds the latest device
 * step.  Set it before the first frame or after a full flush; TC_ERR_PARAM
 * if a stream uses rate control or frames are still pending. */
tc_error_t tcb_batch_set_pipelined(tcb_batch_t *batch, int enabled);
/* Pipelined batch: entropy-code the frames still pending from the last call
 * and return their packets (TC_OK), without planning or running new frames
 * (tcb_batch_flush would also run the B-frame tails); TC_ERR_EOF when
 * nothing is pending. */
tc_error_t tcb_batch_drain(tcb_batch_t *batch, tc_packet_t *packets, int *status);
int tcb_batch_get_graph_stats(tcb_batch_t *batch, int64_t *graph_launches, int64_t *graph_builds);

/* ---------------------------------------------------------------------
 * Served form (no reference counterpart): encode sessions that arrive and
 * leave at any time, admitted under a device-memory budget and advanced
 * together (continuous batching).  Each admitted session keeps its
 * reference frames, MV grids and QP state on the device; every step
 * encodes one frame of every admitted session that has input, in shared
 * CTU-engine launches.  A session's packets are bit-identical to encoding
 * it alone with tc_encoder_*.
 * ------------------------------------------------------------------- */
typedef struct tcb_server tcb_server_t;

typedef struct tcb_server_packet {
    int session;            /* id returned by tcb_server_open */
    int status;             /* TC_OK: packet filled; TC_ERR_NEED_MORE: frame
                               buffered for B reordering; else an error
                               (the session is retired) */
    tc_packet_t packet;     /* data valid until the next tcb_server_step */
} tcb_server_packet_t;

/* Frames a session may have queued on the host before the server takes
 * them (tcb_server_push returns TC_ERR_NEED_MORE beyond this). */
#define TCB_SERVER_QUEUE 2

/* One device allocation of hbm_budget_bytes holds every admitted session;
 * at most max_active sessions (<= 256) are admitted at once. */
tcb_server_t *tcb_server_create(size_t hbm_budget_bytes, int max_active);
void tcb_server_destroy(tcb_server_t *server);
/* Device bytes a session of this configuration occupies while admitted
 * (0 for an invalid configuration). */
size_t tcb_server_session_bytes(const tc_config_t *config);
/* Queue a session (FIFO).  Returns its id (>= 0), TC_ERR_PARAM for an
 * invalid configuration (sessions run the v2 CTU engine: use_v2 must be
 * set), TC_ERR_MEMORY if it can never fit the budget. */
int tcb_server_open(tcb_server_t *server, const tc_config_t *config);
/* Queue the session's next frame (host planes, copied before returning). */
tc_error_t tcb_server_push(tcb_server_t *server, int session,
                           const tc_pixel_t *y, int stride_y,
                           const tc_pixel_t *cb, int stride_cb,
                           const tc_pixel_t *cr, int stride_cr);
/* No more input: the session drains its B-frame tail, then is retired
 * and its device memory returns to the budget. */
tc_error_t tcb_server_finish(tcb_server_t *server, int session);
/* 0 waiting for admission, 1 admitted, 2 retired. */
int tcb_server_session_state(tcb_server_t *server, int session);
/* Admit waiting sessions that fit, then encode one frame of every admitted
 * session with input.  Writes one entry per session that ran (cap must be
 * >= max_active) and returns their number, or a negative tc_error_t. */
int tcb_server_step(tcb_server_t *server, tcb_server_packet_t *out, int cap);
void tcb_server_stats(tcb_server_t *server, int *waiting, int *active, int *retired,
                      size_t *bytes_in_use, size_t *bytes_budget);
/* CUDA-graph replay of every step's device work (as tcb_batch_set_graphs). */
void tcb_server_set_graphs(tcb_server_t *server, int enabled);
/* Host milliseconds spent since creation admitting sessions (setting up
 * their encoders in the budget's arena) and in whole tcb_server_step calls
 * (admission, uploads, the device step and entropy coding), and the number
 * of sessions admitted. */
void tcb_server_get_timing(tcb_server_t *server, double *admit_ms, double *step_ms,
                           long long *admitted);

/* ---------------------------------------------------------------------
 * Part 2: standalone kernels.
 * ------------------------------------------------------------------- */

/* One frame for the CTU engine.  Every pointer is a device pointer; all
 * planes share stride_y / stride_c.  ref_*[i] == NULL marks an empty DPB
 * slot.  prev_mv_grid / cur_mv_grid hold ceil(W/8)*ceil(H/8) cells of
 * tcb_mv_cell_bytes() each (prev may be NULL); ctu_records holds
 * ceil(W/64)*ceil(H/64) records of tcb_ctu_record_bytes() each: the
 * decision tree, quantised coefficients in syntax order and SAO
 * parameters of every CTU, ready for the v2 syntax writer. */
typedef struct tcb_frame_desc {
    int width, height, stride_y, stride_c;
    const tc_pixel_t *src_y, *src_cb, *src_cr;
    tc_pixel_t *rec_y, *rec_cb, *rec_cr;
    const tc_pixel_t *ref_y[TC_REF_FRAMES], *ref_cb[TC_REF_FRAMES], *ref_cr[TC_REF_FRAMES];
    int ref_poc[TC_REF_FRAMES];
    const void *prev_mv_grid;
    void *cur_mv_grid;
    void *ctu_records;
    int frame_type;        /* 0 key, 1 P, 2 B */
    int poc, qp, preset, profile;
    int global_mv_valid, global_mv_x, global_mv_y;   /* encoder-only hint, quarter-pel */
} tcb_frame_desc_t;

size_t tcb_ctu_record_bytes(void);
size_t tcb_mv_cell_bytes(void);
/* Device scratch tcb_ctu_encode_frame needs for a width x height frame. */
size_t tcb_ctu_scratch_bytes(int width, int height);

/* Encode every CTU of one frame (decide, write pass, deblocking, SAO) as a
 * persistent wavefront kernel: replaces the per-CTU loop of the reference
 * frame encoder, src/encoder.c:2939-2946 calling encode_ctu_v2
 * (src/encoder.c:1399-1522).  `scratch` is device memory of at least
 * tcb_ctu_scratch_bytes(width, height) bytes (queue, publish flags,
 * frame parameters); it may be reused once the call's work has finished. */
tc_error_t tcb_ctu_encode_frame(const tcb_frame_desc_t *desc, void *scratch, size_t scratch_bytes,
                                void *stream);

/* tcb_ctu_encode_frame without any device allocation (no counterpart in
 * the reference).  For callers that cannot allocate device memory: an
 * application whose own pool allocator owns all of the GPU's memory, a
 * plugin host that only lends out the frame buffers it manages, or a
 * real-time loop in which cudaMalloc / cudaFree and the synchronisation
 * cudaFree implies are not allowed.  The caller still passes every input
 * and output buffer in `desc`; the scratch is a fixed device array inside
 * the library, sized for TCB_CTU_STATIC_MAX_CTUS CTUs (17,664 bytes),
 * which every GPU that loads the library holds until the process exits.
 *
 *  - Frames of more than TCB_CTU_STATIC_MAX_CTUS CTUs (ceil(W/64) *
 *    ceil(H/64); 3840x2160 is 2,040) return TC_ERR_MEMORY; use
 *    tcb_ctu_encode_frame for them.  Invalid descriptors return
 *    TC_ERR_PARAM.
 *  - The first call on a device, made with that device current, looks up
 *    the array's device address and uploads the constant tables; make
 *    that first call before any stream capture.  The first launch of the
 *    CTU engine in a process (through this or any other entry point) can
 *    also make the CUDA driver enlarge its local-memory reservation for
 *    the engine's stack and register spills, which is device memory the
 *    driver takes; later calls take none.
 *  - Every call on a device shares the one array, which keeps the last
 *    call's contents; each call resets what must start at zero on
 *    `stream` before its encode kernel runs.  Calls whose work overlaps
 *    on the GPU (different streams, or different host threads, without
 *    ordering between them) race on the array and give wrong results:
 *    order them on one stream or serialise them.
 *  - Calls nothing that allocates (no cudaMalloc, cudaFree, pinned host
 *    memory or library allocator); launches are asynchronous on `stream`. */
#define TCB_CTU_STATIC_MAX_CTUS 2048
tc_error_t tcb_ctu_encode_frame_static(const tcb_frame_desc_t *desc, void *stream);

/* Result of the last frame launched with this scratch (or with the static
 * scratch): waits for `stream`, then returns TC_OK, or TC_ERR_INTERNAL
 * when a CTU's wait for its left / above neighbour ran out (the frame's
 * output is then not valid) or the device reported an error.  The two
 * frame entry points above return once the work is queued; this is how a
 * caller learns that it completed.  No reference counterpart (the
 * reference's per-CTU loop cannot stall). */
tc_error_t tcb_ctu_frame_result(const void *scratch, void *stream);
tc_error_t tcb_ctu_frame_result_static(void *stream);

/* Bound of a CTU's wait for a neighbour's publish flag, in back-off
 * iterations of at most 2,048 ns each; default 2^22 (about 8.6 s).  Set
 * for the current device; applies to every CTU-engine launch on it
 * (frame entry points, encoders, batches, served sessions) that starts
 * afterwards.  spins < 1 returns TC_ERR_PARAM. */
tc_error_t tcb_set_neighbor_wait_limit(long long spins);
tc_error_t tcb_get_neighbor_wait_limit(long long *spins);

/* Test hook: tcb_ctu_encode_frame with the first CTU of the wavefront
 * queue left out.  Its publish flag is never set, so the waits of its
 * right and lower neighbours run out (bounded, see above) and
 * tcb_ctu_frame_result reports TC_ERR_INTERNAL; the device context stays
 * usable.  Frames of at least 2 CTUs. */
tc_error_t tcb_debug_ctu_encode_frame_without_first(const tcb_frame_desc_t *desc, void *scratch,
                                                    size_t scratch_bytes, void *stream);

/* Test hook: the next n device or pinned-host allocations of the library
 * succeed and the one after fails, once (n < 0: none).  Returns the count
 * that was still pending (negative when the armed failure has happened or
 * none was armed).  A failure surfaces as NULL from the create calls or
 * TC_ERR_MEMORY from encode / decode / batch calls, with the object still
 * usable or destroyable. */
long long tcb_debug_fail_allocations_after(long long n);

/* One frame for standalone motion compensation.  Device pointers; the
 * reference and prediction planes share stride_y / stride_c. */
typedef struct tcb_mc_frame {
    int width, height, stride_y, stride_c;
    const tc_pixel_t *ref_y, *ref_cb, *ref_cr;
    tc_pixel_t *pred_y, *pred_cb, *pred_cr;
    const int16_t *mv;     /* ceil(W/8) * ceil(H/8) (dx, dy) pairs in quarter
                              luma samples, raster order of the 8x8 blocks */
} tcb_mc_frame_t;

/* Motion-compensated prediction of n frames: every 8x8 luma block and its
 * 4x4 chroma blocks predicted from the reference at the block's vector,
 * exactly as tc_inter_predict / tc_inter_predict_chroma (reference
 * src/motion.c:493-632) with an 8x8 block; samples beyond the frame are not
 * written.  One launch per 32 frames. */
tc_error_t tcb_mc_frames(const tcb_mc_frame_t *frames, int n, void *stream);

/* One frame for the standalone in-loop filters.  Device pointers; the
 * reconstruction planes are filtered in place. */
typedef struct tcb_filter_frame {
    int width, height, stride_y, stride_c;
    tc_pixel_t *y, *cb, *cr;          /* reconstruction (in place) */
    const tc_pixel_t *src_y;          /* source luma: SAO decision only */
    int stride_src;
    int qp;                           /* frame QP */
    int16_t *sao_params;              /* SAO out, may be NULL: 3 int16 per CTU
                                         (present, band, offset), raster order */
} tcb_filter_frame_t;

/* Deblocking of the internal 4-pixel edges of every full 64x64 CTU of n
 * frames (partial CTUs at the right / bottom border are left alone, as in
 * the reference): replaces tc_deblock_ctu (reference src/filter.c:23-237)
 * as called per CTU at src/encoder.c:1457-1458.  One launch per 32 frames. */
tc_error_t tcb_deblock_frames(const tcb_filter_frame_t *frames, int n, void *stream);

/* Luma SAO band offset of every CTU of n frames: choose
 * (tc_sao_choose_bo, reference src/filter.c:269-319), rate gate
 * (src/encoder.c:1463-1493, lambda = tc_lambda(qp) * 6) and apply
 * (tc_sao_ctu_luma, src/filter.c:251-266) against src_y. */
tc_error_t tcb_sao_frames(const tcb_filter_frame_t *frames, int n, void *stream);

/* Autotuner of the frame kernels' tile shape (threads per CTA: deblocking
 * 64 / 128 / 256, SAO 64 / 128, motion compensation 64 / 128 / 256).
 * tcb_autotune_frame_kernels times every variant of the three kernels on
 * `frames` (1..32) scratch frames of width x height with random content and
 * vectors (device memory allocated and freed inside; the call
 * synchronises), keeps the fastest per kernel for that frame size, and
 * later calls whose first frame has that size use it (process-wide).
 * tcb_autotune_threads returns the tuned threads per CTA of a kernel at a
 * size, plus TCB_STAGING_TMA for deblocking when TMA staging won (0: not
 * tuned; the kernel then uses its default, 128 / 128 / 256 threads and
 * vector loads). */
#define TCB_KERNEL_DEBLOCK 0
#define TCB_KERNEL_SAO 1
#define TCB_KERNEL_MC 2
/* Added to a deblocking variant: the CTU tiles are staged through the
 * tensor-memory accelerator (2D tile copies into shared memory and back)
 * instead of 16-byte vector loads, for launches whose planes are 16-byte
 * aligned with 16-byte multiple strides. */
#define TCB_STAGING_TMA 0x10000
tc_error_t tcb_autotune_frame_kernels(int width, int height, int frames);
int tcb_autotune_threads(int kernel, int width, int height);
/* Record a choice directly (a table saved from an earlier tuning run):
 * threads must be a variant of the kernel, 0 removes the entry. */
tc_error_t tcb_autotune_set_threads(int kernel, int width, int height, int threads);

/* Engine knobs per frame size (no reference counterpart).  Neither changes
 * any output; both change how long a step takes, which depends on the frame
 * size and the content, so they are measured (tcodec_b200.tuning times every
 * combination on the caller's frames) rather than fixed:
 *   search_window  radius R (2..5) of the motion search's SAD tables: the
 *                  small-hexagon and diamond stages of blocks up to 16x16
 *                  read their candidates from (2R+1)^2 positions computed in
 *                  one pass; larger R costs more per table and refills less;
 *   queue_order    how a batch step merges its streams' CTU wavefronts:
 *                  TCB_QUEUE_DIAGONAL takes every stream's anti-diagonal d
 *                  before any stream's d+1; TCB_QUEUE_STAGGERED starts
 *                  stream s s diagonals later, so the streams' short first
 *                  and last diagonals do not all fall together.  A batch
 *                  uses the order tuned for its largest frame size.
 * Defaults (nothing set, or set back with 0, 0): R = 4, diagonal order.
 * The setting applies to frames planned afterwards by any encoder, batch or
 * server in the process, and to tcb_ctu_encode_frame(_static). */
#define TCB_SEARCH_WINDOW_MIN 2
#define TCB_SEARCH_WINDOW_MAX 5
#define TCB_QUEUE_DIAGONAL 0
#define TCB_QUEUE_STAGGERED 1
tc_error_t tcb_engine_set_tuning(int width, int height, int search_window, int queue_order);
tc_error_t tcb_engine_get_tuning(int width, int height, int *search_window, int *queue_order);
/* Bounded waits of the frame kernels that gave up since the last call
 * (a staged tile that never arrived; the CTU is then left unfiltered).
 * 0 in a healthy run; reading resets.  Synchronises the device. */
unsigned int tcb_frame_kernels_errors(void);

#ifdef __cplusplus
}
#endif

#endif /* TCODEC_B200_H */
