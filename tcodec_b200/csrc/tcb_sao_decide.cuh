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

#include "tcb_pair16.cuh"

namespace tcb {

constexpr int SAO_ROWS = 48;

// Statistics row of a reconstructed sample value.
__host__ __device__ __forceinline__ int sao_row_of(int v) {
    return v < 8 ? 32 + v : (v >= 248 ? v - 208 : v >> 3);
}

// sao_row_of of the four samples of a word at once (byte i of the result
// for byte i of r).  Bands 1..30 keep their band; bands 0 and 31 (band + 1
// is 1 or 32, with no bit of 0x1E set) take 32 + (v & 15), which is
// 32..39 for 0..7 and 40..47 for 248..255.
__host__ __device__ __forceinline__ uint32_t sao_rows4(uint32_t r) {
    const uint32_t band = (r >> 3) & 0x1F1F1F1Fu;
    const uint32_t value_row = (r & 0x0F0F0F0Fu) | 0x20202020u;
    const uint32_t inner = pair_prmt(((band + 0x01010101u) & 0x1E1E1E1Eu) + 0x7F7F7F7Fu, 0, 0xBA98);
    return (band & inner) | (value_row & ~inner);
}

// A statistics word gains 65536 + 256 + o - r per sample: the count in
// its high half and the biased difference 256 + o - r (1..511) in its low
// half.  Up to 128 samples keep the low half below 65536, so words of up
// to 128 samples in total can be added before they are split
// (sao_unpack); the sum is the low halves less 256 per sample.
constexpr uint32_t SAO_BIAS = 256;

// The biased differences 256 + o - r of the four samples of (r, o): bytes
// 0 and 2 in the low and high lanes of `even`, bytes 1 and 3 in those of
// `odd`.
__host__ __device__ __forceinline__ void sao_incr4(uint32_t r, uint32_t o, uint32_t &even, uint32_t &odd) {
    even = (o & 0x00FF00FFu) + SAO_BIAS * 0x00010001u - (r & 0x00FF00FFu);
    odd = pair_prmt(o, 0, 0x4341) + SAO_BIAS * 0x00010001u - pair_prmt(r, 0, 0x4341);
}
// The statistics increment of a lane: the lane with 1 in the count half.
__host__ __device__ __forceinline__ uint32_t sao_lane_lo(uint32_t x) { return pair_prmt(x, 1, 0x5410); }
__host__ __device__ __forceinline__ uint32_t sao_lane_hi(uint32_t x) { return pair_prmt(x, 1, 0x5432); }

// Count and biased sum of a word (or sum of words) of at most 128 samples;
// the row's sum of o - r is then bsum - SAO_BIAS * cnt.
__host__ __device__ __forceinline__ void sao_unpack(uint32_t w, int &cnt, int &bsum) {
    cnt += (int)(w >> 16);
    bsum += (int)(w & 0xFFFF);
}

// SSE of the CTU after offsetting band b by its candidate (written to
// *cand; 0 when the band is empty or its offset rounds to 0, and then the
// SSE returned is base).  Every term fits in 32 bits for a 64x64 CTU:
// base <= 4096 * 255^2 < 2^28, |S| <= 4096 * 255, |c| <= 7.
__host__ __device__ inline int sao_band_sse(int b, int base, const int *row_cnt, const int *row_sum, int *cand) {
    int n = 0, s = 0;
    if (b == 0 || b == 31) {
        const int r0 = b ? 40 : 32;
        for (int k = 0; k < 8; ++k) { n += row_cnt[r0 + k]; s += row_sum[r0 + k]; }
    } else {
        n = row_cnt[b];
        s = row_sum[b];
    }
    *cand = 0;
    if (n == 0) return base;
    int c = (s + (s >= 0 ? n / 2 : -(n / 2))) / n;
    c = c < -7 ? -7 : (c > 7 ? 7 : c);
    *cand = c;
    if (c == 0) return base;
    int sse = base - 2 * c * s + n * c * c;
    if (b == 0 && c < 0) {
        for (int v = 0; v < 8; ++v)
            if (v + c < 0) sse += 2 * (v + c) * row_sum[32 + v] + row_cnt[32 + v] * (v + c) * (v - c);
    } else if (b == 31 && c > 0) {
        for (int v = 248; v < 256; ++v)
            if (v + c > 255)
                sse += 2 * (v - 255 + c) * row_sum[v - 208] + row_cnt[v - 208] * (v - 255 + c) * (v - 255 - c);
    }
    return sse;
}

}  // namespace tcb
