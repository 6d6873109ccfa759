// tcb_legacy.cu — device side of the legacy (v0 / v1) 8x8 block path
// (reference src/encoder.c:1526-2361, src/decoder.c:260-683).
//
// One warp per CTU.  A CTU reads the reconstruction of its left, above and
// above-right neighbours (intra references, including the above-right 8
// samples of a block) and, where the reference reads samples not yet coded
// in raster order, the previous frame's reconstruction that the caller
// leaves in the output planes.  The wavefront therefore runs CTU (r, c) on
// diagonal c + 2r: its left, above and above-right neighbours lie on
// earlier diagonals, and every CTU whose samples it may read before they
// are coded (right and below-left) on later ones.  One launch per diagonal
// keeps that order without any inter-CTA waiting.
#include <cuda_runtime.h>
#include <math.h>

namespace tcb {
namespace legacy {
static __constant__ int c_ldct4[4][4];
static __constant__ int c_ldct8[8][8];
__device__ __forceinline__ int ldct4(int k, int n) { return c_ldct4[k][n]; }
__device__ __forceinline__ int ldct8(int k, int n) { return c_ldct8[k][n]; }
}  // namespace legacy
}  // namespace tcb

#include "tcb_legacy.cuh"
#include "tcb_launch.h"

namespace tcb {
namespace legacy {

__global__ void __launch_bounds__(32) legacy_ctu_kernel(LFrame F, const int *items, int n, int enc) {
    __shared__ LState S;
    const int it = blockIdx.x;
    if (it >= n) return;
    const int v = items[it];
    code_ctu(S, F, v >> 10, v & 1023, enc != 0);
}

}  // namespace legacy

// DCT-II matrices in 14-bit fixed point from their closed form
// (m[k][n] = round(2^14 s_k cos((2n+1) k pi / 2N))), equal to the reference
// tables of src/transform.c:313-329.
cudaError_t upload_legacy_tables() {
    static bool done[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64 && done[dev]) return cudaSuccess;
    int d4[4][4], d8[8][8];
    const double pi = 3.14159265358979323846;
    for (int N = 4; N <= 8; N += 4)
        for (int k = 0; k < N; ++k)
            for (int m = 0; m < N; ++m) {
                const double s = k == 0 ? sqrt(1.0 / N) : sqrt(2.0 / N);
                const int v = (int)lround(16384.0 * s * cos((2 * m + 1) * k * pi / (2.0 * N)));
                if (N == 4) d4[k][m] = v; else d8[k][m] = v;
            }
    if ((e = cudaMemcpyToSymbol(legacy::c_ldct4, d4, sizeof(d4))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(legacy::c_ldct8, d8, sizeof(d8))) != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) done[dev] = true;
    return cudaSuccess;
}

cudaError_t launch_legacy_ctus(const legacy::LFrame &F, const int *d_items, int n, bool encode, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    legacy::legacy_ctu_kernel<<<n, 32, 0, st>>>(F, d_items, n, encode ? 1 : 0);
    return cudaGetLastError();
}

}  // namespace tcb
