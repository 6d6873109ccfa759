// tcb_mc_pairs.cuh — block motion compensation on packed sample pairs
// (tcb_pair16.cuh), for the standalone frame kernel.
//
// Luma, full six-tap block (reference src/motion.c:552-572, the path taken
// when the block and its six-tap support lie inside the frame): the
// reference evaluates every sample on its own, up to eleven six-tap
// filters each.  Every anchor a sample uses is a fixed function of its
// position, so here one thread computes, for four columns of an 8x8 block,
// the horizontal half-samples of 13 rows once, the vertical half-samples
// and the centre half-samples (vertical six-tap of the horizontal ones)
// once per output row, and forms the quarter-sample phase by selection
// (PairPhase): 3.3 six-tap filters per sample, two samples per
// instruction.
//
// Chroma, 1/8-sample bilinear (reference src/motion.c:597-632) for 4x4
// blocks whose clamped coordinates never clamp: four multiply-adds per
// pair.
//
// Both are __host__ __device__ so they can be run against the oracle on
// the CPU.
#pragma once
#include <cstddef>
#include <cstdint>

#include "tcb_pair16.cuh"

namespace tcb {

__host__ __device__ __forceinline__ uint32_t mc_ld32(const uint32_t *p) {
#ifdef __CUDA_ARCH__
    return __ldg(p);
#else
    return *p;
#endif
}

// The same nine / five bytes from words already aligned: w is the aligned
// word holding the first byte and sh its byte offset times 8.  With a row
// stride that is a multiple of 4 every row has the same offset, so a block's
// rows step w by the stride in words and compute the alignment once.
__host__ __device__ __forceinline__ void mc_load9w(const uint32_t *w, uint32_t sh, uint32_t &u0, uint32_t &u1,
                                                 uint32_t &u2) {
    const uint32_t w0 = mc_ld32(w), w1 = mc_ld32(w + 1), w2 = mc_ld32(w + 2);
    u0 = pair_fshr(w0, w1, sh);
    u1 = pair_fshr(w1, w2, sh);
    u2 = w2 >> sh;
}
__host__ __device__ __forceinline__ void mc_load5w(const uint32_t *w, uint32_t sh, uint32_t &u0, uint32_t &u1) {
    const uint32_t w0 = mc_ld32(w), w1 = mc_ld32(w + 1);
    u0 = pair_fshr(w0, w1, sh);
    u1 = w1 >> sh;
}
// The aligned word holding byte p, and p's offset in it times 8.
__host__ __device__ __forceinline__ const uint32_t *mc_align(const uint8_t *p, uint32_t &sh) {
    const uintptr_t a = (uintptr_t)p;
    sh = (uint32_t)(a & 3) * 8;
    return (const uint32_t *)(a & ~(uintptr_t)3);
}
// The bytes p[0..3] (as one little-endian word).
__host__ __device__ __forceinline__ uint32_t mc_load4(const uint8_t *p) {
    const uintptr_t a = (uintptr_t)p;
    const uint32_t *w = (const uint32_t *)(a & ~(uintptr_t)3);
    const uint32_t sh = (uint32_t)(a & 3) * 8;
    return sh ? pair_fshr(mc_ld32(w), mc_ld32(w + 1), sh) : mc_ld32(w);
}

// Columns 4h..4h+3 of the 8x8 luma prediction at integer position (fx, fy),
// quarter phase ph (PairPhase or PairPhaseFixed); the caller guarantees
// fx >= 2, fx + 10 < W, fy >= 2, fy + 10 < H and a stride s that is a
// multiple of 4.  out[y] holds row y's four samples.
template <class Phase>
__host__ __device__ __forceinline__ void mc_luma_six_tap(const uint8_t *ref, int s, int fx, int fy, int h,
                                                       const Phase &ph, uint32_t out[8]) {
    // Per row r (frame row fy - 2 + r): even pairs E1..E3 at columns
    // (4h, 4h+1), (4h+2, 4h+3), (4h+4, 4h+5); odd pairs O1, O2 at
    // (4h+1, 4h+2), (4h+3, 4h+4); horizontal halves H0, H1 at the two even
    // pairs (biased).  The value along x on integer row y (0..8, frame row
    // fy + y) serves output row y as its top and row y - 1 as its bottom
    // (T0, T1).  Output row y reads rows y..y+5 only, so it is formed as
    // soon as row y + 5 is in: a rolling window of six rows stays live, not
    // all thirteen.
    uint32_t E1[13], E2[13], E3[13], H0[13], H1[13], T0[9], T1[9];
    uint32_t sh;
    const uint32_t *w = mc_align(ref + (ptrdiff_t)(fy - 2) * s + fx + 4 * h - 2, sh);
    const int sw = s >> 2;
#pragma unroll
    for (int r = 0; r < 13; ++r, w += sw) {
        uint32_t u0, u1, u2;
        mc_load9w(w, sh, u0, u1, u2);                     // columns 4h-2 .. 4h+6
        const uint32_t x0 = pair_lo(u0), x1 = pair_hi(u0), x2 = pair_lo(u1), x3 = pair_hi(u1), x4 = pair_lo(u2);
        const uint32_t o0 = pair_mid(x0, x1), o1 = pair_mid(x1, x2), o2 = pair_mid(x2, x3), o3 = pair_mid(x3, x4);
        E1[r] = x1; E2[r] = x2; E3[r] = x3;
        H0[r] = pair_six_tap(x0, o0, x1, o1, x2, o2, PAIR_K_RAW);
        H1[r] = pair_six_tap(x1, o1, x2, o2, x3, o3, PAIR_K_RAW);
        if (r >= 2 && r <= 10) {
            T0[r - 2] = ph.along_x(x1 + PAIR_B, H0[r], o1 + PAIR_B);
            T1[r - 2] = ph.along_x(x2 + PAIR_B, H1[r], o2 + PAIR_B);
        }
        if (r >= 5) {
            const int y = r - 5;
            const uint32_t c0 = pair_six_tap(E1[y], E1[y + 1], E1[y + 2], E1[y + 3], E1[y + 4], E1[y + 5], PAIR_K_RAW);
            const uint32_t c1 = pair_six_tap(E2[y], E2[y + 1], E2[y + 2], E2[y + 3], E2[y + 4], E2[y + 5], PAIR_K_RAW);
            const uint32_t c2 = pair_six_tap(E3[y], E3[y + 1], E3[y + 2], E3[y + 3], E3[y + 4], E3[y + 5], PAIR_K_RAW);
            const uint32_t d0 = pair_six_tap(H0[y], H0[y + 1], H0[y + 2], H0[y + 3], H0[y + 4], H0[y + 5], PAIR_K_HALF);
            const uint32_t d1 = pair_six_tap(H1[y], H1[y + 1], H1[y + 2], H1[y + 3], H1[y + 4], H1[y + 5], PAIR_K_HALF);
            const uint32_t m0 = ph.along_x(c0, d0, pair_mid(c0, c1)), m1 = ph.along_x(c1, d1, pair_mid(c1, c2));
            out[y] = pair_pack(ph.finish(T0[y], m0, T0[y + 1]), ph.finish(T1[y], m1, T1[y + 1]));
        }
    }
}

// The 4x4 chroma prediction at 1/8-sample position (xi + fx/8, yi + fy/8);
// the caller guarantees xi >= 0, xi + 4 < W, yi >= 0, yi + 4 < H (no
// coordinate clamps) and a stride s that is a multiple of 4.  out[y] holds
// row y's four samples.
__host__ __device__ __forceinline__ void mc_chroma_bilinear(const uint8_t *ref, int s, int xi, int yi, int fx,
                                                          int fy, uint32_t out[4]) {
    const uint32_t w00 = (8 - fx) * (8 - fy), w01 = fx * (8 - fy), w10 = (8 - fx) * fy, w11 = fx * fy;
    uint32_t A0[5], A1[5], B0[5], B1[5];   // pairs at columns (0,1), (2,3) and (1,2), (3,4)
    uint32_t sh;
    const uint32_t *w = mc_align(ref + (ptrdiff_t)yi * s + xi, sh);
    const int sw = s >> 2;
#pragma unroll
    for (int r = 0; r < 5; ++r, w += sw) {
        uint32_t u0, u1;
        mc_load5w(w, sh, u0, u1);
        const uint32_t x0 = pair_lo(u0), x1 = pair_hi(u0), x2 = pair_lo(u1);
        A0[r] = x0; A1[r] = x1; B0[r] = pair_mid(x0, x1); B1[r] = pair_mid(x1, x2);
    }
    // Lanes stay below 64 * 255 + 32.
#pragma unroll
    for (int y = 0; y < 4; ++y) {
        const uint32_t k = 32u * 0x00010001u;
        const uint32_t v0 = A0[y] * w00 + B0[y] * w01 + A0[y + 1] * w10 + B0[y + 1] * w11 + k;
        const uint32_t v1 = A1[y] * w00 + B1[y] * w01 + A1[y + 1] * w10 + B1[y + 1] * w11 + k;
        out[y] = pair_pack((v0 >> 6) & 0x03FF03FFu, (v1 >> 6) & 0x03FF03FFu);
    }
}

}  // namespace tcb
