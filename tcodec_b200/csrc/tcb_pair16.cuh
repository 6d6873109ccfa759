// tcb_pair16.cuh — two 16-bit lanes per 32-bit word for the byte kernels.
//
// A "pair" holds two samples, the left one in bits 0..15.  Sums, products
// by small constants and shifts then work on both lanes with one 32-bit
// instruction, exactly, provided that every lane stays in [0, 65535] at
// every step (no carry or borrow crosses bit 16).  Signed intermediates
// (six-tap half-samples, which reach -80) are therefore carried with a
// bias: lane = value + 208.  The bias is a multiple of two and 208 * 32 is
// a multiple of 32, so the six-tap's (s + 16) >> 5 and the quarter-sample
// average (a + b + 1) >> 1 give the biased value of the reference's floor
// arithmetic with no correction term.  The lane ranges each helper relies
// on are stated beside it.
//
// The helpers are __host__ __device__ so the packed arithmetic can be
// checked against the scalar formulas on the CPU.
#pragma once
#include <cstdint>

namespace tcb {

constexpr uint32_t PAIR_BIAS = 208;                       // lane bias of half-samples
constexpr uint32_t PAIR_B = PAIR_BIAS * 0x00010001u;      // the bias in both lanes

// PTX prmt.b32 (default mode): byte i of the result is byte (s >> 4i) & 7
// of {b, a}, or, when bit 3 of that nibble is set, the sign of that byte
// replicated (__byte_perm uses only the low three bits, hence the inline
// PTX).
__host__ __device__ __forceinline__ uint32_t pair_prmt(uint32_t a, uint32_t b, uint32_t s) {
#ifdef __CUDA_ARCH__
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(s));
    return r;
#else
    const uint64_t v = (uint64_t)b << 32 | a;
    uint32_t r = 0;
    for (int i = 0; i < 4; ++i) {
        const uint32_t n = (s >> (4 * i)) & 15, byte = (uint32_t)(v >> ((n & 7) * 8)) & 0xFF;
        r |= ((n & 8) ? ((byte & 0x80) ? 0xFFu : 0u) : byte) << (8 * i);   // bit 3: replicate the sign bit
    }
    return r;
#endif
}
// (hi:lo) >> sh, low word; sh in [0, 31].
__host__ __device__ __forceinline__ uint32_t pair_fshr(uint32_t lo, uint32_t hi, uint32_t sh) {
#ifdef __CUDA_ARCH__
    return __funnelshift_r(lo, hi, sh);
#else
    return (uint32_t)((((uint64_t)hi << 32) | lo) >> (sh & 31));
#endif
}
// Lane-wise unsigned 16-bit max / min: one PTX max.u16x2 / min.u16x2
// (sm_90 and later).
__host__ __device__ __forceinline__ uint32_t pair_max(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
    uint32_t r;
    asm("max.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
#else
    uint32_t lo = (a & 0xFFFF) > (b & 0xFFFF) ? (a & 0xFFFF) : (b & 0xFFFF);
    uint32_t hi = (a >> 16) > (b >> 16) ? (a >> 16) : (b >> 16);
    return hi << 16 | lo;
#endif
}
__host__ __device__ __forceinline__ uint32_t pair_min(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
    uint32_t r;
    asm("min.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
#else
    uint32_t lo = (a & 0xFFFF) < (b & 0xFFFF) ? (a & 0xFFFF) : (b & 0xFFFF);
    uint32_t hi = (a >> 16) < (b >> 16) ? (a >> 16) : (b >> 16);
    return hi << 16 | lo;
#endif
}

// Bytes 2j, 2j+1 of w as a pair (j = 0 or 1).
__host__ __device__ __forceinline__ uint32_t pair_lo(uint32_t w) { return pair_prmt(w, 0, 0x4140); }
__host__ __device__ __forceinline__ uint32_t pair_hi(uint32_t w) { return pair_prmt(w, 0, 0x4342); }
// (right lane of a, left lane of b): the pair one sample to the right of a.
__host__ __device__ __forceinline__ uint32_t pair_mid(uint32_t a, uint32_t b) { return pair_fshr(a, b, 16); }

// Six-tap [1,-5,20,20,-5,1] on six pairs, (s + k) >> 5 per lane with
// k = 16 + 32 * (output bias - input bias) (the taps sum to 32).  Valid
// when, per lane, m2 + p3 + k + 20 (z0 + p1) <= 65535 and the final sum
// >= 0:
//   raw samples (0..255), k = 16 + 32 * 208  -> lanes 4122..17382
//   half-samples biased by 208 (128..527), k = 16 -> lanes 122..22150
__host__ __device__ __forceinline__ uint32_t pair_six_tap(uint32_t m2, uint32_t m1, uint32_t z0, uint32_t p1,
                                                        uint32_t p2, uint32_t p3, uint32_t k2) {
    uint32_t acc = m2 + p3 + k2;
    acc += (z0 + p1) * 20u;
    acc -= (m1 + p2) * 5u;
    return (acc >> 5) & 0x07FF07FFu;
}
constexpr uint32_t PAIR_K_RAW = (16u + 32u * PAIR_BIAS) * 0x00010001u;
constexpr uint32_t PAIR_K_HALF = 16u * 0x00010001u;

// (a + b + 1) >> 1 per lane (lanes <= 32767).
__host__ __device__ __forceinline__ uint32_t pair_avg(uint32_t a, uint32_t b) {
    return ((a + b + 0x00010001u) >> 1) & 0x7FFF7FFFu;
}

// Quarter-sample phase of a luma block (reference src/motion.c:190-260):
// along x, the value on an integer or half row is the integer sample a
// (dx 0), avg(a, half) (dx 1), the half sample (dx 2) or avg(half, next
// integer) (dx 3); along y the same between the top row, the half row and
// the bottom row; the result is clamped to 0..255.  With dy == 0 (or
// dx == 0) this is also the reference's horizontal-only (vertical-only)
// path: its truncating division and this floor differ only on negative
// sums, which the final clamp maps to 0 in both.  Anchors and results
// carry the 208 bias; finish() removes it.
//
// PairPhase selects at run time: L = dx < 2 ? integer : half and
// R = dx == 0 ? integer : dx == 3 ? next integer : half, then avg(L, R)
// (averaging a value with itself returns it, so no phase needs its own
// case) — one instruction stream for blocks of any phase.
struct PairPhase {
    bool xl, x0, x3, yl, y0, y3;
    __host__ __device__ __forceinline__ void init(int dx, int dy) {
        xl = dx < 2; x0 = dx == 0; x3 = dx == 3;
        yl = dy < 2; y0 = dy == 0; y3 = dy == 3;
    }
    __host__ __device__ __forceinline__ uint32_t along_x(uint32_t a, uint32_t h, uint32_t a1) const {
        return pair_avg(xl ? a : h, x0 ? a : (x3 ? a1 : h));
    }
    __host__ __device__ __forceinline__ uint32_t finish(uint32_t top, uint32_t mid, uint32_t bot) const {
        const uint32_t r = pair_avg(yl ? top : mid, y0 ? top : (y3 ? bot : mid));
        return pair_min(pair_max(r, PAIR_B), PAIR_B + 255u * 0x00010001u) - PAIR_B;
    }
};
// The same with the phase fixed at compile time: anchors the phase never
// reads are dead code.
template <int DX, int DY>
struct PairPhaseFixed {
    __host__ __device__ __forceinline__ static uint32_t pick(int f, uint32_t a, uint32_t h, uint32_t a1) {
        return f == 0 ? a : f == 1 ? pair_avg(a, h) : f == 2 ? h : pair_avg(h, a1);
    }
    __host__ __device__ __forceinline__ uint32_t along_x(uint32_t a, uint32_t h, uint32_t a1) const {
        return pick(DX, a, h, a1);
    }
    __host__ __device__ __forceinline__ uint32_t finish(uint32_t top, uint32_t mid, uint32_t bot) const {
        return pair_min(pair_max(pick(DY, top, mid, bot), PAIR_B), PAIR_B + 255u * 0x00010001u) - PAIR_B;
    }
};

// Two pairs of samples (each lane 0..255) as four bytes.
__host__ __device__ __forceinline__ uint32_t pair_pack(uint32_t lo, uint32_t hi) {
    return pair_prmt(lo, hi, 0x6420);
}

}  // namespace tcb
