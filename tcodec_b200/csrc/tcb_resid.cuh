// tcb_resid.cuh — fused residual path of one transform unit on a group of
// lanes of one warp: forward DCT-II (14-bit, two rounded passes) -> JND-band
// dead-zone quantisation -> RDOQ-lite (keep-vs-zero of |level| == 1) ->
// bit-model estimate -> centroid dequantisation -> inverse DCT.
//
//   8x8 TU: an "octet" of 8 consecutive lanes, lane r owns row r on the
//           row pass and column r afterwards.
//   4x4 TU: a "quad" of 4 consecutive lanes, same ownership.
//
// The row<->column exchange goes through a shared-memory scratch private to
// the lane group: 8 rows of 9 ints per octet (72), 4 rows of 5 ints per quad
// (20).  The padded rows put the 32 lanes of a warp (four octets at 72-int
// or eight quads at 20-int offsets) on 32 different banks for both the row
// writes and the column reads.  All 32 lanes of the
// warp must call these routines together (they use full-mask shuffles of
// width 8 / 4); inactive groups pass dummy data and discard the results.
//
// Arithmetic follows reference src/transform.c:331-439 (dct4_point,
// dct8_point2, tc_fdct*/tc_idct*_res), src/encoder.c:333-385 (rdoq_level1,
// count_siglevel_bits, lastpos_cost) and tcodec_common.h:226-246
// (quant/dequant).  Accumulators are 32-bit: encoder residuals are clipped
// to [-512, 511], so |coef| <= 4096, |dequant| <= 4096 + eff/2 <= 8037, and
// the largest inverse-pass sum is 8037 * 43284 / 2^14 * 43284 < 2^30.
#pragma once
#include <math.h>
#include <cuda_runtime.h>
#include "tcb_common.cuh"

namespace tcb {

// DCT matrices: one copy per translation unit (no relocatable device
// code); each unit that launches kernels using them uploads its copy with
// upload_dct_tables() before its first launch.
static __constant__ int c_dct4[4][4];
static __constant__ int c_dct8[8][8];

// Orthonormal DCT-II matrix in 14-bit fixed point:
// m[k][n] = round(2^14 * s_k * cos((2n+1) k pi / 2N)), s_0 = sqrt(1/N),
// s_k = sqrt(2/N).  Equals the reference tables of src/transform.c:313-329.
inline void dct_matrix(int N, int *m) {
    const double pi = 3.14159265358979323846;
    for (int k = 0; k < N; ++k)
        for (int n = 0; n < N; ++n) {
            const double s = k == 0 ? sqrt(1.0 / N) : sqrt(2.0 / N);
            m[k * N + n] = (int)lround(16384.0 * s * cos((2 * n + 1) * k * pi / (2.0 * N)));
        }
}

static inline cudaError_t upload_dct_tables() {
    int d4[4][4], d8[8][8];
    dct_matrix(4, &d4[0][0]);
    dct_matrix(8, &d8[0][0]);
    cudaError_t e = cudaMemcpyToSymbol(c_dct4, d4, sizeof(d4));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(c_dct8, d8, sizeof(d8));
}

struct QuantParams {
    int eff[4];
    uint32_t rcp[4];
    int off[4];           // eff / 3: quantiser rounding offset
    int bias[4];          // eff / 6: centroid dequantiser bias
    long long lambda;     // RDOQ lambda
    __host__ __device__ void set_band(int b, int e, uint32_t r) {
        eff[b] = e; rcp[b] = r; off[b] = e / 3; bias[b] = e / 6;
    }
};

// Frequency band of coefficient (row k, column col) of an N x N TU in
// raster order: DC, first quarter, second quarter, rest (the raster-index
// bands of freq_band).  With k a compile-time constant only the DC case
// depends on col.
template <int N>
__device__ __forceinline__ int band_rc(int k, int col) {
    if (k == 0) return col == 0 ? 0 : 1;
    if (N == 8) return k < 2 ? 1 : (k < 4 ? 2 : 3);
    return k < 2 ? 2 : 3;
}

__device__ __forceinline__ int oct_sum(int v) {
    v += __shfl_xor_sync(0xffffffffu, v, 4, 8);
    v += __shfl_xor_sync(0xffffffffu, v, 2, 8);
    v += __shfl_xor_sync(0xffffffffu, v, 1, 8);
    return v;
}
__device__ __forceinline__ int oct_max(int v) {
    v = max(v, __shfl_xor_sync(0xffffffffu, v, 4, 8));
    v = max(v, __shfl_xor_sync(0xffffffffu, v, 2, 8));
    v = max(v, __shfl_xor_sync(0xffffffffu, v, 1, 8));
    return v;
}
__device__ __forceinline__ int quad_sum(int v) {
    v += __shfl_xor_sync(0xffffffffu, v, 2, 4);
    v += __shfl_xor_sync(0xffffffffu, v, 1, 4);
    return v;
}
__device__ __forceinline__ int quad_max(int v) {
    v = max(v, __shfl_xor_sync(0xffffffffu, v, 2, 4));
    v = max(v, __shfl_xor_sync(0xffffffffu, v, 1, 4));
    return v;
}

// Quantise + RDOQ-lite one coefficient of band `band` (reference
// src/encoder.c:333-355): dead-zone quantiser with offset eff / 3, then a
// level of magnitude 1 is dropped when zero costs less.
__device__ __forceinline__ int quant_rdoq(int c, int band, const QuantParams &qp) {
    const int eff = qp.eff[band];
    const uint32_t rcp = qp.rcp[band];
    const int off = qp.off[band];
    int q = 0;
    if (c > 0) q = udiv_rcp((uint32_t)(c + off), eff, rcp);
    else if (c < 0) q = -udiv_rcp((uint32_t)(-c + off), eff, rcp);
    if (q == 1 || q == -1) {
        // zero wins when c^2 + lambda < (c - dq)^2 + 2 lambda, i.e. when
        // dq * (2c - dq) < lambda; |c| <= 2^15 and |dq| <= 9194 keep the
        // product below 2^30
        const int dq = q > 0 ? eff + qp.bias[band] : -eff - qp.bias[band];
        if ((long long)(dq * (2 * c - dq)) < qp.lambda) q = 0;
    }
    return q;
}

__device__ __forceinline__ int dequant_band(int q, int band, const QuantParams &qp) {
    const int eff = qp.eff[band], bias = qp.bias[band];
    return q > 0 ? q * eff + bias : (q < 0 ? q * eff - bias : 0);
}

// Bit-model term of one quantised level (reference src/encoder.c:360-370).
__device__ __forceinline__ int level_bits(int v) {
    return v == 0 ? 1 : 2 + 2 * bitlen((unsigned)absi(v));
}

// Exact 8- and 4-point DCT sums by partial butterflies.  The 14-bit
// matrices keep the cosine symmetries exactly (lround is odd-symmetric):
// c8[k][7-n] = (-1)^k c8[k][n], c8[2m][3-n] = (-1)^m c8[2m][n] for n < 4,
// c4[k][3-n] = (-1)^k c4[k][n].  So every sum the reference forms,
// out[k] = sum_n c[k][n] x[n] (forward) or out[n] = sum_k c[k][n] y[k]
// (inverse), is the same integer from even / odd halves: 24 products per
// 8-point transform instead of 64, 8 per 4-point instead of 16.
__device__ __forceinline__ void fdct8_sums(const int x[8], int out[8]) {
    int E[4], O[4];
#pragma unroll
    for (int n = 0; n < 4; ++n) { E[n] = x[n] + x[7 - n]; O[n] = x[n] - x[7 - n]; }
    const int EE0 = E[0] + E[3], EE1 = E[1] + E[2], EO0 = E[0] - E[3], EO1 = E[1] - E[2];
    out[0] = c_dct8[0][0] * EE0 + c_dct8[0][1] * EE1;
    out[4] = c_dct8[4][0] * EE0 + c_dct8[4][1] * EE1;
    out[2] = c_dct8[2][0] * EO0 + c_dct8[2][1] * EO1;
    out[6] = c_dct8[6][0] * EO0 + c_dct8[6][1] * EO1;
#pragma unroll
    for (int k = 1; k < 8; k += 2)
        out[k] = c_dct8[k][0] * O[0] + c_dct8[k][1] * O[1] + c_dct8[k][2] * O[2] + c_dct8[k][3] * O[3];
}
__device__ __forceinline__ void idct8_sums(const int y[8], int out[8]) {
    const int e0 = c_dct8[0][0] * y[0] + c_dct8[4][0] * y[4], e1 = c_dct8[0][1] * y[0] + c_dct8[4][1] * y[4];
    const int o0 = c_dct8[2][0] * y[2] + c_dct8[6][0] * y[6], o1 = c_dct8[2][1] * y[2] + c_dct8[6][1] * y[6];
    const int ev[4] = {e0 + o0, e1 + o1, e1 - o1, e0 - o0};
#pragma unroll
    for (int n = 0; n < 4; ++n) {
        const int od = c_dct8[1][n] * y[1] + c_dct8[3][n] * y[3] + c_dct8[5][n] * y[5] + c_dct8[7][n] * y[7];
        out[n] = ev[n] + od;
        out[7 - n] = ev[n] - od;
    }
}
__device__ __forceinline__ void fdct4_sums(const int x[4], int out[4]) {
    const int E0 = x[0] + x[3], E1 = x[1] + x[2], O0 = x[0] - x[3], O1 = x[1] - x[2];
    out[0] = c_dct4[0][0] * E0 + c_dct4[0][1] * E1;
    out[2] = c_dct4[2][0] * E0 + c_dct4[2][1] * E1;
    out[1] = c_dct4[1][0] * O0 + c_dct4[1][1] * O1;
    out[3] = c_dct4[3][0] * O0 + c_dct4[3][1] * O1;
}
__device__ __forceinline__ void idct4_sums(const int y[4], int out[4]) {
#pragma unroll
    for (int n = 0; n < 2; ++n) {
        const int ev = c_dct4[0][n] * y[0] + c_dct4[2][n] * y[2], od = c_dct4[1][n] * y[1] + c_dct4[3][n] * y[3];
        out[n] = ev + od;
        out[3 - n] = ev - od;
    }
}

// 8x8 TU on an octet.  In: res_row = clipped residual row `l8`.
// Out: q_col[k] = quantised level at (k, l8); r_col[k] = reconstructed
// residual at (k, l8) (int16-wrapped like tc_coeff_t); returns the bit
// estimate 1 + 2*nz + sig/level bits + last-position cost (uniform).
__device__ __forceinline__ int tu8_code(int l8, const int res_row[8], int *scr,
                                        const QuantParams &qp, int q_col[8], int r_col[8]) {
    int t[8];
    fdct8_sums(res_row, t);
#pragma unroll
    for (int k = 0; k < 8; ++k) scr[l8 * 9 + k] = (t[k] + 8192) >> 14;
    __syncwarp();
    int col[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) col[i] = scr[i * 9 + l8];
    __syncwarp();
    int nz = 0, last = -1, lball = 0;
    int cs8[8];
    fdct8_sums(col, cs8);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int c = (int16_t)((cs8[k] + 8192) >> 14);
        const int pos = k * 8 + l8;
        const int q = (int16_t)quant_rdoq(c, band_rc<8>(k, l8), qp);
        q_col[k] = q;
        if (q) { ++nz; last = pos; }
        lball += level_bits(q);
    }
    // The level bits of positions up to `last` are those of all 64 less one
    // per zero past it (level_bits(0) == 1), so they need not wait for
    // `last`: one packed sum (level bits << 8 | nonzero count, at most 2048
    // and 64) and one max, side by side.
    const int packed = oct_sum((lball << 8) | nz);
    last = oct_max(last);
    nz = packed & 0xFF;
    const int lb = (packed >> 8) - (63 - last);
    const int bits = 1 + 2 * nz + lb + lastpos_cost(last);
    // Dequantise and hand columns back as rows for the inverse row pass.
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        scr[k * 9 + l8] = (int16_t)dequant_band(q_col[k], band_rc<8>(k, l8), qp);
    }
    __syncwarp();
    int row[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) row[n] = scr[l8 * 9 + n];
    __syncwarp();
    int is8[8];
    idct8_sums(row, is8);
#pragma unroll
    for (int k = 0; k < 8; ++k) scr[l8 * 9 + k] = (is8[k] + 8192) >> 14;
    __syncwarp();
#pragma unroll
    for (int n = 0; n < 8; ++n) col[n] = scr[n * 9 + l8];
    __syncwarp();
    idct8_sums(col, is8);
#pragma unroll
    for (int k = 0; k < 8; ++k) r_col[k] = (int16_t)((is8[k] + 8192) >> 14);
    return bits;
}

// 4x4 TU on a quad (lane l4 owns row / column l4).  Same contract as
// tu8_code with n = 16 coefficients.
__device__ __forceinline__ int tu4_code(int l4, const int res_row[4], int *scr,
                                        const QuantParams &qp, int q_col[4], int r_col[4]) {
    int t[4];
    fdct4_sums(res_row, t);
#pragma unroll
    for (int k = 0; k < 4; ++k) scr[l4 * 5 + k] = (t[k] + 8192) >> 14;
    __syncwarp();
    int col[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) col[i] = scr[i * 5 + l4];
    __syncwarp();
    int nz = 0, last = -1, lball = 0;
    int cs4[4];
    fdct4_sums(col, cs4);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int c = (int16_t)((cs4[k] + 8192) >> 14);
        const int pos = k * 4 + l4;
        const int q = (int16_t)quant_rdoq(c, band_rc<4>(k, l4), qp);
        q_col[k] = q;
        if (q) { ++nz; last = pos; }
        lball += level_bits(q);
    }
    // as in tu8_code: all 16 level bits less one per zero past `last`
    const int packed = quad_sum((lball << 8) | nz);
    last = quad_max(last);
    nz = packed & 0xFF;
    const int lb = (packed >> 8) - (15 - last);
    const int bits = 1 + 2 * nz + lb + lastpos_cost(last);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        scr[k * 5 + l4] = (int16_t)dequant_band(q_col[k], band_rc<4>(k, l4), qp);
    }
    __syncwarp();
    int row[4];
#pragma unroll
    for (int n = 0; n < 4; ++n) row[n] = scr[l4 * 5 + n];
    __syncwarp();
    int is4[4];
    idct4_sums(row, is4);
#pragma unroll
    for (int k = 0; k < 4; ++k) scr[l4 * 5 + k] = (is4[k] + 8192) >> 14;
    __syncwarp();
#pragma unroll
    for (int n = 0; n < 4; ++n) col[n] = scr[n * 5 + l4];
    __syncwarp();
    idct4_sums(col, is4);
#pragma unroll
    for (int k = 0; k < 4; ++k) r_col[k] = (int16_t)((is4[k] + 8192) >> 14);
    return bits;
}

}  // namespace tcb
