// tcb_sao_decide.cuh — the v2 luma band-offset decision of one CTU from
// per-row statistics (reference src/filter.c:269-319 tc_sao_choose_bo and
// the rate gate of src/encoder.c:1463-1493), without a second pass over
// the pixels.
//
// Statistics rows, each a (count, sum of org - rec) over the CTU's pixels:
//   rows 1..30   pixels whose reconstruction is in band 1..30 (value >> 3)
//   rows 32..39  pixels whose reconstruction is the value 0..7   (band 0)
//   rows 40..47  pixels whose reconstruction is the value 248..255 (band 31)
// Rows 0 and 31 stay empty.
//
// With candidate offset c for band b, every pixel of the band changes its
// error from d = o - r to d - c unless r + c leaves 0..255, which only
// values 0..7 (c < 0) and 248..255 (c > 0) can do.  So the SSE is
// base - 2 c S + n c^2, plus, for each clipped value v with (n_v, S_v),
//   to 0:   (v + c)(2 d + v - c) summed:        2 (v + c) S_v + n_v (v + c)(v - c)
//   to 255: (v - 255 + c)(2 d + v - 255 - c):   2 (v - 255 + c) S_v + n_v (v - 255 + c)(v - 255 - c)
// (o = d + v; the o^2 terms cancel), which is exact.
#pragma once
#include <cstdint>

namespace tcb {

constexpr int SAO_ROWS = 48;

// Statistics row of a reconstructed sample value.
__host__ __device__ __forceinline__ int sao_row_of(int v) {
    return v < 8 ? 32 + v : (v >= 248 ? v - 208 : v >> 3);
}

// SSE of the CTU after offsetting band b by its candidate (written to
// *cand; 0 when the band is empty or its offset rounds to 0, and then the
// SSE returned is base).
__host__ __device__ inline long long sao_band_sse(int b, long long base, const int *row_cnt, const int *row_sum,
                                                  int *cand) {
    long long n = 0, s = 0;
    if (b == 0 || b == 31) {
        const int r0 = b ? 40 : 32;
        for (int k = 0; k < 8; ++k) { n += row_cnt[r0 + k]; s += row_sum[r0 + k]; }
    } else {
        n = row_cnt[b];
        s = row_sum[b];
    }
    *cand = 0;
    if (n == 0) return base;
    long long c = (s + (s >= 0 ? n / 2 : -(n / 2))) / n;
    c = c < -7 ? -7 : (c > 7 ? 7 : c);
    *cand = (int)c;
    if (c == 0) return base;
    long long sse = base - 2 * c * s + n * c * c;
    if (b == 0 && c < 0) {
        for (int v = 0; v < 8; ++v)
            if (v + c < 0) sse += 2 * (v + c) * row_sum[32 + v] + (long long)row_cnt[32 + v] * (v + c) * (v - c);
    } else if (b == 31 && c > 0) {
        for (int v = 248; v < 256; ++v)
            if (v + c > 255)
                sse += 2 * (v - 255 + c) * row_sum[v - 208] +
                       (long long)row_cnt[v - 208] * (v - 255 + c) * (v - 255 - c);
    }
    return sse;
}

}  // namespace tcb
