// tcb_frame_kernels.cu — per-frame helper kernels around the CTU engine and
// the launch glue used by the host driver.
//
//   glob_mv_kernel   encoder-only global-motion hint: greedy two-pass walk
//                    over a downsampled SAD grid (reference
//                    src/encoder.c:171-202 estimate_global_mv); each warp
//                    scores one candidate, candidates commit in order.
//                    glob_mv_multi_kernel runs the walks of all streams of
//                    a batch step in one launch, one CTA per stream.
//   hist16_kernel    16-bin luma histogram for scene-cut detection (the
//                    chi-square test itself stays on the host in double,
//                    reference src/encoder.c:2655-2678).
//   frame_sse_kernel luma SSE of source vs reconstruction for the PSNR
//                    statistic (reference src/tcodec.c:34-54).
#include <cuda_runtime.h>

#include "tcb_engine.cuh"
#include "tcb_launch.h"

namespace tcb {

__device__ void glob_mv_walk(const uint8_t *__restrict__ cur, const uint8_t *__restrict__ ref, int W, int H,
                             int s, FrameParams *fp) {
    const int cw = W / 4, ch = H / 4;
    const int nx = (cw + 1) / 2, ny = (ch + 1) / 2, ns = nx * ny;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __shared__ long long sad[32];
    __shared__ int sh_dx, sh_dy;
    __shared__ long long sh_best;
    if (threadIdx.x == 0) { sh_dx = 0; sh_dy = 0; sh_best = (long long)1 << 60; }
    __syncthreads();
    for (int pass = 0; pass < 2; ++pass) {
        const int step = pass ? 1 : 2, range = pass ? 1 : 8;
        const int side = 2 * range / step + 1, n = side * side;
        int p0 = 0;
        while (p0 < n) {
            const int bdx = sh_dx, bdy = sh_dy;
            const long long best = sh_best;
            const int k = p0 + warp;
            long long acc = 0;
            if (k < n) {
                const int dy = -range + (k / side) * step, dx = -range + (k % side) * step;
                for (int i = lane; i < ns; i += 32) {
                    const int yy = (i / nx) * 2, xx = (i - (i / nx) * nx) * 2;
                    const int rx = xx * 4 + bdx + dx * 4, ry = yy * 4 + bdy + dy * 4;
                    if (rx < 0 || ry < 0 || rx >= W || ry >= H) { acc += 255 * 4; continue; }
                    const int d = (int)cur[(size_t)(yy * 4) * s + xx * 4] - (int)ref[(size_t)ry * s + rx];
                    acc += d < 0 ? -d : d;
                }
                for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            }
            if (lane == 0) sad[warp] = acc;
            __syncthreads();
            if (threadIdx.x == 0) {
                int found = -1;
                for (int w = 0; w < 32 && p0 + w < n; ++w)
                    if (sad[w] < best) { found = w; break; }
                if (found >= 0) {
                    const int kk = p0 + found;
                    const int dy = -range + (kk / side) * step, dx = -range + (kk % side) * step;
                    sh_best = sad[found];
                    sh_dx = bdx + dx * 4;
                    sh_dy = bdy + dy * 4;
                    sad[0] = kk + 1;          // next start
                } else {
                    sad[0] = p0 + 32;
                }
            }
            __syncthreads();
            p0 = (int)sad[0];
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {
        fp->glob_valid = 1;
        fp->glob_x = sh_dx * 4;
        fp->glob_y = sh_dy * 4;
    }
}

__global__ void __launch_bounds__(1024, 1)
glob_mv_kernel(const uint8_t *__restrict__ cur, const uint8_t *__restrict__ ref, int W, int H,
               int s, FrameParams *fp) {
    glob_mv_walk(cur, ref, W, H, s, fp);
}

// Every stream of a batch step in one launch: CTA j walks job j.
__global__ void __launch_bounds__(1024, 1) glob_mv_multi_kernel(GlobJobs jobs) {
    const GlobJob &j = jobs.job[blockIdx.x];
    glob_mv_walk(j.cur, j.ref, j.W, j.H, j.s, j.fp);
}

__global__ void hist16_kernel(const uint8_t *__restrict__ y, int W, int H, int s, int *hist) {
    __shared__ int h[16];
    if (threadIdx.x < 16) h[threadIdx.x] = 0;
    __syncthreads();
    for (int r = blockIdx.x; r < H; r += gridDim.x)
        for (int x = threadIdx.x; x < W; x += blockDim.x) atomicAdd(&h[y[(size_t)r * s + x] >> 4], 1);
    __syncthreads();
    if (threadIdx.x < 16 && h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], h[threadIdx.x]);
}

__global__ void frame_sse_kernel(const uint8_t *__restrict__ a, const uint8_t *__restrict__ b, int W,
                                 int H, int s, unsigned long long *out) {
    unsigned long long acc = 0;
    for (int r = blockIdx.x; r < H; r += gridDim.x)
        for (int x = threadIdx.x; x < W; x += blockDim.x) {
            const int d = (int)a[(size_t)r * s + x] - (int)b[(size_t)r * s + x];
            acc += (unsigned long long)(d * d);
        }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc) atomicAdd(out, acc);
}

cudaError_t init_device_tables() {
    cudaError_t e = init_engine_tables();
    if (e != cudaSuccess) return e;
    return init_decode_tables();
}

cudaError_t launch_glob_mv(const uint8_t *cur, const uint8_t *ref, int W, int H, int s,
                           FrameParams *d_params, cudaStream_t st) {
    glob_mv_kernel<<<1, 1024, 0, st>>>(cur, ref, W, H, s, d_params);
    return cudaGetLastError();
}

cudaError_t launch_glob_mv_multi(const GlobJob *jobs, int n, cudaStream_t st) {
    for (int i = 0; i < n; i += GlobJobs::MAX) {
        GlobJobs g;
        g.n = n - i < GlobJobs::MAX ? n - i : GlobJobs::MAX;
        for (int k = 0; k < g.n; ++k) g.job[k] = jobs[i + k];
        glob_mv_multi_kernel<<<g.n, 1024, 0, st>>>(g);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_hist16(const uint8_t *y, int W, int H, int s, int *d_hist, cudaStream_t st) {
    cudaMemsetAsync(d_hist, 0, 16 * sizeof(int), st);
    hist16_kernel<<<148, 256, 0, st>>>(y, W, H, s, d_hist);
    return cudaGetLastError();
}

cudaError_t launch_frame_sse(const uint8_t *a, const uint8_t *b, int W, int H, int s,
                             unsigned long long *d_out, cudaStream_t st) {
    cudaMemsetAsync(d_out, 0, sizeof(unsigned long long), st);
    frame_sse_kernel<<<148, 256, 0, st>>>(a, b, W, H, s, d_out);
    return cudaGetLastError();
}

}  // namespace tcb
