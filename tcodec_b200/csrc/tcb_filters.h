// tcb_filters.h — launch interface of the standalone frame filters
// (tcb_filters.cu).  Frame descriptors travel as the kernel parameter, up
// to MAX frames per launch; CTA g finds its frame by the CTU prefix sums.
#pragma once
#include <stdint.h>

#include <cuda_runtime.h>

#include "../../include/tcodec_b200.h"

namespace tcb {

struct DeblockFrame {
    uint8_t *y, *cb, *cr;
    int W, H, sy, sc, qp;
};
struct DeblockJobs {
    static constexpr int MAX = 32;
    int n;
    int ctu_off[MAX + 1];      // first CTA of each frame (full CTUs only)
    DeblockFrame f[MAX];
};

struct SaoFrame {
    uint8_t *rec;              // luma reconstruction, filtered in place
    const uint8_t *org;        // source luma
    int W, H, sr, so;
    int lambda_sao;            // tc_lambda(qp) of the frame
    int16_t *params;           // 3 per CTU: present, band, offset (may be NULL)
};
struct SaoJobs {
    static constexpr int MAX = 32;
    int n;
    int ctu_off[MAX + 1];
    SaoFrame f[MAX];
};

// threads: CTA size variant (deblocking 64 / 128 / 256, SAO 64 / 128;
// anything else selects 128); for deblocking, TCB_STAGING_TMA added to it
// moves the tiles with the tensor-memory accelerator where the planes allow.
cudaError_t launch_deblock_frames(const DeblockFrame *frames, int n, cudaStream_t st, int threads);
// Bounded TMA waits in the deblocking kernel that gave up since the last
// call (0 in a healthy run); reading resets.
unsigned int tma_waits_expired();
cudaError_t launch_sao_frames(const SaoFrame *frames, int n, cudaStream_t st, int threads);

// Motion compensation over tcb_mc_frame_t descriptors (tcb_mc.cu);
// threads 64 / 128 / 256 per CTA, anything else selects 256.
cudaError_t launch_mc_frames(const tcb_mc_frame_t *frames, int n, cudaStream_t st, int threads);

// Tile-shape choices of the frame-kernel autotuner (tcb_autotune.cpp):
// threads per CTA tuned for kernel k at a frame size, 0 if not tuned.
int tuned_threads(int kernel, int width, int height);
void set_tuned_threads(int kernel, int width, int height, int threads);

}  // namespace tcb
