// tcb_filters.h — launch interface of the standalone frame filters
// (tcb_filters.cu).  Frame descriptors travel as the kernel parameter, up
// to MAX frames per launch; CTA g finds its frame by the CTU prefix sums.
#pragma once
#include <stdint.h>

#include <cuda_runtime.h>

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

cudaError_t launch_deblock_frames(const DeblockFrame *frames, int n, cudaStream_t st);
cudaError_t launch_sao_frames(const SaoFrame *frames, int n, cudaStream_t st);

}  // namespace tcb
