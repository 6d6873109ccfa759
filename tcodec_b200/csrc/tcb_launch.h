// tcb_launch.h — host-callable launch wrappers of the sm_100a kernels.
#pragma once
#include <math.h>
#include <cuda_runtime.h>

#include "tcb_common.cuh"
#include "tcb_legacy_types.h"

namespace tcb {

cudaError_t init_device_tables();
cudaError_t init_engine_tables();
size_t ctu_smem_bytes();
cudaError_t init_decode_tables();
cudaError_t launch_decode_items(const FrameParams *d_params, const int *d_items, int n, cudaStream_t st);
cudaError_t launch_ctu_persistent(const FrameParams *d_params, const int *d_items, int n, int *d_ctrl,
                                  int grid, cudaStream_t st);
cudaError_t launch_ctu_items(const FrameParams *d_params, const int *d_items, int n, cudaStream_t st);
struct GlobJob {
    const uint8_t *cur, *ref;
    int W, H, s;
    FrameParams *fp;
};
struct GlobJobs {                  // passed by value as the kernel parameter
    static constexpr int MAX = 64;
    int n;
    GlobJob job[MAX];
};
cudaError_t launch_glob_mv_multi(const GlobJob *jobs, int n, cudaStream_t st);
cudaError_t launch_glob_mv(const uint8_t *cur, const uint8_t *ref, int W, int H, int s,
                           FrameParams *d_params, cudaStream_t st);
cudaError_t launch_hist16(const uint8_t *y, int W, int H, int s, int *d_hist, cudaStream_t st);
// Legacy (v0 / v1) 8x8 block path: one launch per wavefront diagonal;
// `encode` picks the encoder (decisions + reconstruction) or the decoder
// (reconstruction from parsed records).
cudaError_t upload_legacy_tables();
cudaError_t launch_legacy_ctus(const legacy::LFrame &F, const int *d_items, int n, bool encode, cudaStream_t st);
cudaError_t launch_frame_sse(const uint8_t *a, const uint8_t *b, int W, int H, int s,
                             unsigned long long *d_out, cudaStream_t st);

}  // namespace tcb
