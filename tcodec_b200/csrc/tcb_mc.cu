// tcb_mc.cu — motion-compensated prediction of whole frames from a
// reference and an 8x8-block vector field, many frames per launch: the
// reference's tc_inter_predict (src/motion.c:493-584: integer copy, full
// six-tap block, or per-sample edge-safe path, chosen per block) and
// tc_inter_predict_chroma (src/motion.c:597-632: 1/8-sample bilinear with
// clamped coordinates) applied to every 8x8 luma / 4x4 chroma block.
//
// Two threads per 8x8 block, blocks in raster order (a warp covers 16
// neighbouring blocks, so its loads and stores are contiguous runs): thread
// h produces luma columns 4h..4h+3 of the block and chroma plane h (Cb, Cr).
// The six-tap and bilinear paths run on packed sample pairs
// (tcb_mc_pairs.cuh) for planes whose stride is a multiple of 4 bytes;
// blocks near the frame edge, and planes with other strides, take the
// per-sample arithmetic of the CTU engine (tcb_pixel.cuh), so predictions
// equal the encoder's; a CTA queues those blocks and all of its threads
// share their samples after its packed blocks (McEdge below).
#include <cuda_runtime.h>

#include "../../include/tcodec_b200.h"
#include "tcb_common.cuh"
#include "tcb_filters.h"
#include "tcb_mc_pairs.cuh"
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
    int cta_off[MAX + 1];            // first CTA of each frame
    McFrame f[MAX];
};

// Threads per CTA are a template parameter (64, 128 or 256; the autotuner
// times each per frame size, 256 without tuning); the register budget is
// cut for 768 resident threads per SM (80 registers).
constexpr int MC_DEFAULT_THREADS = 256;

// Four bytes v to dst, only the first w of them at a clipped block edge.
__device__ __forceinline__ void store4(uint8_t *dst, uint32_t v, int w) {
    if (w == 4 && (((uintptr_t)dst) & 3) == 0) {
        *(uint32_t *)dst = v;
    } else {
        for (int c = 0; c < w; ++c) dst[c] = (uint8_t)(v >> (8 * c));
    }
}

template <int DX, int DY>
__device__ __forceinline__ void luma_fixed(const uint8_t *ref, int s, int fx, int fy, int h, uint32_t out[8]) {
    mc_luma_six_tap(ref, s, fx, fy, h, PairPhaseFixed<DX, DY>(), out);
}
// The full six-tap block with its quarter phase (dx * 4 + dy, 1..15) fixed.
__device__ __forceinline__ void luma_six_tap_fixed(const uint8_t *ref, int s, int fx, int fy, int h, int phase,
                                                   uint32_t out[8]) {
    switch (phase) {
        case 1: luma_fixed<0, 1>(ref, s, fx, fy, h, out); break;
        case 2: luma_fixed<0, 2>(ref, s, fx, fy, h, out); break;
        case 3: luma_fixed<0, 3>(ref, s, fx, fy, h, out); break;
        case 4: luma_fixed<1, 0>(ref, s, fx, fy, h, out); break;
        case 5: luma_fixed<1, 1>(ref, s, fx, fy, h, out); break;
        case 6: luma_fixed<1, 2>(ref, s, fx, fy, h, out); break;
        case 7: luma_fixed<1, 3>(ref, s, fx, fy, h, out); break;
        case 8: luma_fixed<2, 0>(ref, s, fx, fy, h, out); break;
        case 9: luma_fixed<2, 1>(ref, s, fx, fy, h, out); break;
        case 10: luma_fixed<2, 2>(ref, s, fx, fy, h, out); break;
        case 11: luma_fixed<2, 3>(ref, s, fx, fy, h, out); break;
        case 12: luma_fixed<3, 0>(ref, s, fx, fy, h, out); break;
        case 13: luma_fixed<3, 1>(ref, s, fx, fy, h, out); break;
        case 14: luma_fixed<3, 2>(ref, s, fx, fy, h, out); break;
        default: luma_fixed<3, 3>(ref, s, fx, fy, h, out); break;
    }
}

// The per-sample edge-safe path costs 30-40 times the packed one.  A block
// that needs it would hold its whole warp (16 blocks) for that long, so its
// threads only queue it in shared memory; once the CTA's packed blocks are
// done, all MT threads share the queued blocks' samples, one sample each.
// (Sharing within the warp instead, without the CTA barrier, measured 5 %
// slower on random vectors.)
struct McEdge {
    int h, X, Y, mvx, mvy;
    __device__ __forceinline__ McEdge(const McFrame &F, int g) {
        const int gw = (F.W + 7) >> 3, blk = g >> 1;
        h = g & 1;
        const int by = blk / gw, bx = blk - by * gw;
        X = bx * 8;
        Y = by * 8;
        mvx = X * 4 + F.mv[2 * blk];
        mvy = Y * 4 + F.mv[2 * blk + 1];
    }
};

// The queued half blocks (entries: thread indices within the CTA, whose
// first element is g0), one sample per thread: luma 32 per entry (4 columns
// x 8 rows), chroma 16 (the 4x4 block of plane h).  Not inlined, so that
// its registers do not add to the packed path's; the frame comes by value,
// as an address into the kernel parameter would copy every frame to the
// stack.
template <int MT>
__device__ __noinline__ void mc_edge_samples(const McFrame F, int g0, const uint16_t *q_luma, int n_luma,
                                             const uint16_t *q_chroma, int n_chroma) {
    const int nl = n_luma * 32, nc = n_chroma * 16;
    for (int i = threadIdx.x; i < nl; i += MT) {
        const McEdge B(F, g0 + q_luma[i >> 5]);
        const int c = i & 3, y = (i >> 2) & 7, x = B.X + 4 * B.h + c;
        if (x < F.W && B.Y + y < F.H)
            F.py[(size_t)(B.Y + y) * F.sy + x] = (uint8_t)interp_luma_safe(
                F.ry, F.sy, F.W, F.H, (B.mvx >> 2) + 4 * B.h + c, (B.mvy >> 2) + y, B.mvx & 3, B.mvy & 3);
    }
    for (int i = threadIdx.x; i < nc; i += MT) {
        const McEdge B(F, g0 + q_chroma[i >> 4]);
        const int Wc = F.W >> 1, Hc = F.H >> 1, c = i & 3, y = (i >> 2) & 3;
        const int x = (B.X >> 1) + c, yy = (B.Y >> 1) + y;
        if (x < Wc && yy < Hc)
            (B.h ? F.pcr : F.pcb)[(size_t)yy * F.sc + x] =
                (uint8_t)chroma_mc_at(B.h ? F.rcr : F.rcb, F.sc, Wc, Hc, B.mvx, B.mvy, c, y);
    }
}

template <int MT>
__global__ void __launch_bounds__(MT, 768 / MT) mc_frames_kernel(McJobs J) {
    __shared__ uint16_t q_luma[MT], q_chroma[MT];   // threads whose block takes the per-sample path
    __shared__ int n_luma, n_chroma;
    if (threadIdx.x == 0) n_luma = n_chroma = 0;
    int k = 0, hi = J.n - 1;                      // binary search for the frame of this CTA
    while (k < hi) {
        const int mid = (k + hi + 1) >> 1;
        if (J.cta_off[mid] <= (int)blockIdx.x) k = mid;
        else hi = mid - 1;
    }
    const McFrame &F = J.f[k];
    const int gw = (F.W + 7) >> 3, gh = (F.H + 7) >> 3;
    const int g0 = ((int)blockIdx.x - J.cta_off[k]) * MT;
    __syncthreads();
    if (((g0 + (int)threadIdx.x) >> 1) < gw * gh) {
        const McEdge B(F, g0 + (int)threadIdx.x);
        const int h = B.h, X = B.X, Y = B.Y, mvx = B.mvx, mvy = B.mvy;
        // ---- luma: columns 4h..4h+3
        const int fx = mvx >> 2, fy = mvy >> 2, dx = mvx & 3, dy = mvy & 3;
        uint32_t out[8];
        bool packed = true;
        if (dx == 0 && dy == 0 && fx >= 0 && fy >= 0 && fx + 8 <= F.W && fy + 8 <= F.H) {
#pragma unroll
            for (int y = 0; y < 8; ++y) out[y] = mc_load4(F.ry + (size_t)(fy + y) * F.sy + fx + 4 * h);
        } else if ((dx | dy) != 0 && fx >= 2 && fx + 10 < F.W && fy >= 2 && fy + 10 < F.H && (F.sy & 3) == 0) {
            // Blocks of one warp that share the phase (coherent motion) take
            // the path specialised for it; mixed phases take the selecting one.
            const int phase = dx * 4 + dy;
            const unsigned m = __activemask();
            if (__all_sync(m, phase == __shfl_sync(m, phase, __ffs(m) - 1))) {
                luma_six_tap_fixed(F.ry, F.sy, fx, fy, h, phase, out);
            } else {
                PairPhase ph;
                ph.init(dx, dy);
                mc_luma_six_tap(F.ry, F.sy, fx, fy, h, ph, out);
            }
        } else {
            q_luma[atomicAdd(&n_luma, 1)] = (uint16_t)threadIdx.x;
            packed = false;
        }
        const int x0 = X + 4 * h, wl = min(4, F.W - x0), hl = min(8, F.H - Y);
        if (packed && wl > 0) {
            uint8_t *dst = F.py + (size_t)Y * F.sy + x0;
#pragma unroll
            for (int y = 0; y < 8; ++y)
                if (y < hl) store4(dst + (size_t)y * F.sy, out[y], wl);
        }
        // ---- chroma: plane h, the 4x4 block at (X/2, Y/2)
        const int Wc = F.W >> 1, Hc = F.H >> 1, cx = X >> 1, cy = Y >> 1;
        const int xi = mvx >> 3, yi = mvy >> 3;
        if (xi >= 0 && xi + 4 < Wc && yi >= 0 && yi + 4 < Hc && (F.sc & 3) == 0) {
            uint32_t cout[4];
            mc_chroma_bilinear(h ? F.rcr : F.rcb, F.sc, xi, yi, mvx & 7, mvy & 7, cout);
            const int wc = min(4, Wc - cx), hc = min(4, Hc - cy);
            uint8_t *dst = (h ? F.pcr : F.pcb) + (size_t)cy * F.sc + cx;
#pragma unroll
            for (int y = 0; y < 4; ++y)
                if (y < hc) store4(dst + (size_t)y * F.sc, cout[y], wc);
        } else {
            q_chroma[atomicAdd(&n_chroma, 1)] = (uint16_t)threadIdx.x;
        }
    }
    __syncthreads();
    if (n_luma | n_chroma) mc_edge_samples<MT>(F, g0, q_luma, n_luma, q_chroma, n_chroma);
}

}  // namespace

cudaError_t launch_mc_frames(const tcb_mc_frame_t *frames, int n, cudaStream_t st, int threads) {
    const int MT = (threads == 64 || threads == 128) ? threads : MC_DEFAULT_THREADS;
    for (int i = 0; i < n;) {
        McJobs J;
        J.n = 0;
        int total = 0;
        while (i < n && J.n < McJobs::MAX) {
            const tcb_mc_frame_t &f = frames[i];
            J.f[J.n] = {f.ref_y, f.ref_cb, f.ref_cr, f.pred_y, f.pred_cb, f.pred_cr, f.mv,
                        f.width, f.height, f.stride_y, f.stride_c};
            J.cta_off[J.n] = total;
            const int blocks = ((f.width + 7) >> 3) * ((f.height + 7) >> 3);
            total += (2 * blocks + MT - 1) / MT;
            ++J.n;
            ++i;
        }
        J.cta_off[J.n] = total;
        if (MT == 64) mc_frames_kernel<64><<<total, 64, 0, st>>>(J);
        else if (MT == 128) mc_frames_kernel<128><<<total, 128, 0, st>>>(J);
        else mc_frames_kernel<256><<<total, 256, 0, st>>>(J);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

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
    const int threads = n ? tuned_threads(TCB_KERNEL_MC, frames[0].width, frames[0].height) : 0;
    return launch_mc_frames(frames, n, (cudaStream_t)stream, threads) == cudaSuccess ? TC_OK : TC_ERR_INTERNAL;
}
