// tcb_mc.cu — motion-compensated prediction of whole frames from a
// reference and an 8x8-block vector field, many frames per launch: the
// reference's tc_inter_predict (src/motion.c:493-584: integer copy, full
// six-tap block, or per-sample edge-safe path, chosen per block) and
// tc_inter_predict_chroma (src/motion.c:597-632: 1/8-sample bilinear with
// clamped coordinates) applied to every 8x8 luma / 4x4 chroma block.
//
// One 256-thread CTA per 64x64 luma tile (64 blocks): four threads per
// block, each producing two luma rows (8 bytes each, one 8-byte store) and
// one row of each chroma plane (4 bytes each).  The sample arithmetic is
// the CTU engine's (tcb_pixel.cuh), so predictions equal the encoder's.
#include <cuda_runtime.h>

#include <vector>

#include "../../include/tcodec_b200.h"
#include "tcb_common.cuh"
#include "tcb_pixel.cuh"

namespace tcb {

namespace {

struct McFrame {
    const uint8_t *ry, *rcb, *rcr;
    uint8_t *py, *pcb, *pcr;
    const int16_t *mv;
    int W, H, sy, sc;
};
struct McJobs {                      // passed by value as the kernel parameter
    static constexpr int MAX = 32;
    int n;
    int tile_off[MAX + 1];           // first CTA (64x64 tile) of each frame
    McFrame f[MAX];
};

constexpr int MT = 256;

__global__ void __launch_bounds__(MT, 4) mc_frames_kernel(McJobs J) {
    int k = 0;
    while (k + 1 < J.n && J.tile_off[k + 1] <= (int)blockIdx.x) ++k;
    const McFrame &F = J.f[k];
    const int local = blockIdx.x - J.tile_off[k], tcols = (F.W + 63) >> 6;
    const int t = threadIdx.x, b = t >> 2, q = t & 3;
    const int X = ((local % tcols) << 6) + (b & 7) * 8, Y = ((local / tcols) << 6) + (b >> 3) * 8;
    if (X >= F.W || Y >= F.H) return;
    const int gw = (F.W + 7) >> 3;
    const int2 v = make_int2(F.mv[2 * ((Y >> 3) * gw + (X >> 3))], F.mv[2 * ((Y >> 3) * gw + (X >> 3)) + 1]);
    const int mvx = X * 4 + v.x, mvy = Y * 4 + v.y;
    // ---- luma: rows 2q, 2q+1 of the 8x8 block
    LumaMC m;
    m.init(F.ry, F.sy, F.W, F.H, mvx, mvy, 8);
    const int wl = min(8, F.W - X);
#pragma unroll
    for (int rr = 0; rr < 2; ++rr) {
        const int r = 2 * q + rr;
        if (Y + r >= F.H) break;
        uint8_t px[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) px[c] = (uint8_t)m.at(c, r);
        uint8_t *dst = F.py + (size_t)(Y + r) * F.sy + X;
        if (wl == 8 && (((uintptr_t)dst) & 7) == 0) {
            uint2 w;
            w.x = px[0] | px[1] << 8 | px[2] << 16 | (uint32_t)px[3] << 24;
            w.y = px[4] | px[5] << 8 | px[6] << 16 | (uint32_t)px[7] << 24;
            *(uint2 *)dst = w;
        } else {
            for (int c = 0; c < wl; ++c) dst[c] = px[c];
        }
    }
    // ---- chroma: row q of the 4x4 block, both planes
    const int Wc = F.W >> 1, Hc = F.H >> 1, cx = X >> 1, cy = (Y >> 1) + q;
    if (cy < Hc) {
        const int wc = min(4, Wc - cx);
#pragma unroll
        for (int pl = 0; pl < 2; ++pl) {
            const uint8_t *ref = pl ? F.rcr : F.rcb;
            uint8_t *dst = (pl ? F.pcr : F.pcb) + (size_t)cy * F.sc + cx;
            uint8_t px[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) px[c] = (uint8_t)chroma_mc_at(ref, F.sc, Wc, Hc, mvx, mvy, c, q);
            if (wc == 4 && (((uintptr_t)dst) & 3) == 0)
                *(uint32_t *)dst = px[0] | px[1] << 8 | px[2] << 16 | (uint32_t)px[3] << 24;
            else
                for (int c = 0; c < wc; ++c) dst[c] = px[c];
        }
    }
}

}  // namespace

}  // namespace tcb

extern "C" tc_error_t tcb_mc_frames(const tcb_mc_frame_t *frames, int n, void *stream) {
    using namespace tcb;
    if (n < 0 || (n > 0 && !frames)) return TC_ERR_PARAM;
    for (int i = 0; i < n; ++i) {
        const tcb_mc_frame_t &f = frames[i];
        if (f.width <= 0 || f.height <= 0 || (f.width & 1) || (f.height & 1) || f.width > TC_MAX_WIDTH ||
            f.height > TC_MAX_HEIGHT || f.stride_y < f.width || f.stride_c < f.width / 2 || !f.ref_y ||
            !f.ref_cb || !f.ref_cr || !f.pred_y || !f.pred_cb || !f.pred_cr || !f.mv)
            return TC_ERR_PARAM;
    }
    for (int i = 0; i < n;) {
        McJobs J;
        J.n = 0;
        int total = 0;
        while (i < n && J.n < McJobs::MAX) {
            const tcb_mc_frame_t &f = frames[i];
            J.f[J.n] = {f.ref_y, f.ref_cb, f.ref_cr, f.pred_y, f.pred_cb, f.pred_cr, f.mv,
                        f.width, f.height, f.stride_y, f.stride_c};
            J.tile_off[J.n] = total;
            total += ((f.width + 63) >> 6) * ((f.height + 63) >> 6);
            ++J.n;
            ++i;
        }
        J.tile_off[J.n] = total;
        mc_frames_kernel<<<total, MT, 0, (cudaStream_t)stream>>>(J);
        if (cudaGetLastError() != cudaSuccess) return TC_ERR_INTERNAL;
    }
    return TC_OK;
}
