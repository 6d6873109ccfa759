// tcb_filters.cu — the v2 in-loop filters as standalone frame kernels over
// planes resident in HBM, for many frames per launch:
//
//   deblock_frames_kernel  internal edges of every full 64x64 CTU of each
//                          frame (reference src/filter.c:23-237, called per
//                          CTU at src/encoder.c:1457-1458 and by the decoder,
//                          full CTUs only).
//   sao_frames_kernel      per-CTU luma band offset: choose (src/filter.c:
//                          269-319), rate gate (src/encoder.c:1463-1493),
//                          apply (src/filter.c:251-266); writes the chosen
//                          (present, band, offset) of every CTU.
//
// Both are byte kernels: one 128-thread CTA per CTU, the tile moved with
// 16-byte loads and stores (a byte path serves unaligned planes), each byte
// read once and written at most once.  Deblocking filters two edge
// positions per instruction on packed 16-bit lanes (tcb_deblock_pairs.cuh).
//
// SAO statistics without atomics: every thread owns two 16-pixel row
// segments (kept in registers for the whole CTU) and a private column of a
// [row][thread] table in shared memory, so its read-modify-writes never
// conflict.  A table word packs count and difference sum as
// count * 65536 + sum of (256 + o - r), which one integer add per pixel
// maintains exactly (tcb_sao_decide.cuh: SAO_BIAS, sao_unpack); the rows and increments of a
// word's four pixels come from a few word operations (sao_rows4,
// sao_incr4), leaving a lane extract, an address and the read-modify-write
// per pixel.  Rows are the 30 inner bands plus the 16 single
// sample values of bands 0 and 31, where an offset can clip; the SSE of
// every band after its offset then follows in closed form, clipping
// included (tcb_sao_decide.cuh), with no second pass over the pixels.
#include <string.h>

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include "tcb_common.cuh"
#include "tcb_deblock_pairs.cuh"
#include "tcb_filters.h"
#include "tcb_pixel.cuh"
#include "tcb_sao_decide.cuh"

namespace tcb {

namespace {

// Threads per CTA (one CTU each) are a template parameter: deblocking 64,
// 128 or 256, SAO 64 or 128 (its statistics table holds one column per
// thread; 256 would pass the 48 KB of static shared memory); the autotuner
// times each per frame size, 128 without tuning.  Small
// CTAs let many CTUs' loads be in flight per SM while other CTUs of the
// same SM filter.

// The frame whose CTA range [off[k], off[k+1]) holds CTA g (binary search
// over the n <= 32 frames of a launch; off[0] = 0 <= g).
__device__ __forceinline__ int find_frame(const int *off, int n, int g) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ bool aligned16(const void *p, int stride) {
    return (((uintptr_t)p) & 15) == 0 && (stride & 15) == 0;
}

// ---------------------------------------------------------------- deblock

template <int DFT>
__global__ void __launch_bounds__(DFT) deblock_frames_kernel(DeblockJobs J) {
    static_assert(DFT >= 32 && DFT % 32 == 0, "whole warps");
    constexpr int NPIECE = (384 + DFT - 1) / DFT;   // 16-byte pieces per thread (384 per CTU)
    __shared__ __align__(16) uint8_t ty[64 * 64];
    __shared__ __align__(16) uint8_t tc[2][32 * 32];
    const int k = find_frame(J.ctu_off, J.n, blockIdx.x);
    const DeblockFrame &F = J.f[k];
    const int local = blockIdx.x - J.ctu_off[k], cols = F.W >> 6;
    const int x0 = (local % cols) << 6, y0 = (local / cols) << 6;
    const int t = threadIdx.x;
    uint8_t *gy = F.y + (size_t)y0 * F.sy + x0;
    uint8_t *const gcb = F.cb + (size_t)(y0 >> 1) * F.sc + (x0 >> 1), *const gcr = F.cr + (size_t)(y0 >> 1) * F.sc + (x0 >> 1);
    auto gc = [&](int c) { return c ? gcr : gcb; };   // a select, not an indexed (local-memory) array
    const bool vec = aligned16(F.y, F.sy) && aligned16(F.cb, F.sc) && aligned16(F.cr, F.sc);
    // ---- load: 16-byte pieces 0..255 luma (row p>>2, segment p&3),
    // 256..383 chroma (plane, row, segment); all issued before any use
    if (vec) {
        uint4 v[NPIECE];
#pragma unroll
        for (int j = 0; j < NPIECE; ++j) {
            const int p = t + j * DFT;
            if (p >= 384) break;
            if (p < 256) {
                v[j] = __ldcs((const uint4 *)(gy + (size_t)(p >> 2) * F.sy + (p & 3) * 16));
            } else {
                const int q = p - 256, c = q >> 6, r = (q >> 1) & 31, sg = q & 1;
                v[j] = __ldcs((const uint4 *)(gc(c) + (size_t)r * F.sc + sg * 16));
            }
        }
#pragma unroll
        for (int j = 0; j < NPIECE; ++j) {
            const int p = t + j * DFT;
            if (p >= 384) break;
            if (p < 256) *(uint4 *)&ty[p * 16] = v[j];
            else {
                const int q = p - 256, c = q >> 6, r = (q >> 1) & 31, sg = q & 1;
                *(uint4 *)&tc[c][r * 32 + sg * 16] = v[j];
            }
        }
    } else {
        for (int i = t; i < 64 * 64; i += DFT) ty[i] = gy[(size_t)(i >> 6) * F.sy + (i & 63)];
        for (int i = t; i < 2 * 32 * 32; i += DFT) {
            const int c = i >> 10, p = i & 1023;
            tc[c][p] = gc(c)[(size_t)(p >> 5) * F.sc + (p & 31)];
        }
    }
    __syncthreads();
    // ---- vertical edges, then horizontal edges, as independent items
    // (tcb_deblock_pairs.cuh): 96 vertical rows (64 luma, 32 Cb), then 60
    // luma items of 16 columns and 56 chroma items of 4
    DeblockQp q;
    q.init(F.qp);
    for (int i = t; i < DEBLOCK_VERT_ROWS; i += DFT) deblock_vert_rows(ty, tc[0], i, q);
    __syncthreads();
    for (int i = t; i < deblock_horiz_wide_items<4>(); i += DFT) deblock_horiz_wide<4>(ty, tc[0], tc[1], i, q);
    __syncthreads();
    // ---- store
    if (vec) {
#pragma unroll
        for (int j = 0; j < NPIECE; ++j) {
            const int p = t + j * DFT;
            if (p >= 384) break;
            if (p < 256) {
                __stcs((uint4 *)(gy + (size_t)(p >> 2) * F.sy + (p & 3) * 16), *(const uint4 *)&ty[p * 16]);
            } else {
                const int q = p - 256, c = q >> 6, r = (q >> 1) & 31, sg = q & 1;
                __stcs((uint4 *)(gc(c) + (size_t)r * F.sc + sg * 16), *(const uint4 *)&tc[c][r * 32 + sg * 16]);
            }
        }
    } else {
        for (int i = t; i < 64 * 64; i += DFT) gy[(size_t)(i >> 6) * F.sy + (i & 63)] = ty[i];
        for (int i = t; i < 2 * 32 * 32; i += DFT) {
            const int c = i >> 10, p = i & 1023;
            gc(c)[(size_t)(p >> 5) * F.sc + (p & 31)] = tc[c][p];
        }
    }
}

// ---------------------------------------------------------------- deblock, TMA staging

// The same filter with the CTU tile moved by the tensor-memory accelerator:
// one thread issues three 2D tile copies (luma 64x64, Cb / Cr 32x32) that
// complete on an mbarrier, and after filtering three tile stores write it
// back.  Used for launches whose planes are 16-byte aligned with 16-byte
// multiple strides (what a tensor map requires); CTU x-coordinates are
// multiples of 64 (luma) and 32 (chroma) bytes and only full CTUs are
// filtered, so every box starts aligned and lies inside its plane.
struct DeblockTmaJobs {            // passed as a __grid_constant__ kernel parameter (about 12.7 KB)
    static constexpr int MAX = 32;
    CUtensorMap ty[MAX], tcb[MAX], tcr[MAX];
    int n;
    int ctu_off[MAX + 1];
    int cols[MAX], qp[MAX];
};

__device__ unsigned int g_tma_wait_expired;   // bounded TMA waits that gave up (0 in a healthy run)

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(dst), "l"(map), "r"(x), "r"(y), "r"(bar) : "memory");
}
__device__ __forceinline__ void tma_store_2d(const CUtensorMap *map, uint32_t src, int x, int y) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];"
                 ::"l"(map), "r"(x), "r"(y), "r"(src) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                 : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    return ok != 0;
}

template <int DFT>
__global__ void __launch_bounds__(DFT) deblock_tma_kernel(const __grid_constant__ DeblockTmaJobs J) {
    __shared__ __align__(128) uint8_t ty[64 * 64];
    __shared__ __align__(128) uint8_t tc[2][32 * 32];
    __shared__ __align__(8) uint64_t bar;
    const int k = find_frame(J.ctu_off, J.n, blockIdx.x);
    const int local = blockIdx.x - J.ctu_off[k];
    const int x0 = (local % J.cols[k]) << 6, y0 = (local / J.cols[k]) << 6;
    const int t = threadIdx.x;
    const uint32_t b = smem_addr(&bar);
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(64 * 64 + 2 * 32 * 32)
                     : "memory");
        tma_load_2d(smem_addr(ty), &J.ty[k], x0, y0, b);
        tma_load_2d(smem_addr(tc[0]), &J.tcb[k], x0 >> 1, y0 >> 1, b);
        tma_load_2d(smem_addr(tc[1]), &J.tcr[k], x0 >> 1, y0 >> 1, b);
    }
    __syncthreads();   // the barrier is initialised before anyone waits on it
    bool landed = false;
    for (int i = 0; i < (1 << 22) && !landed; ++i) landed = mbar_try_wait(b, 0);
    if (!__syncthreads_and(landed)) {
        // The tile never arrived: record it, give the copies in flight a
        // second bounded wait (the shared memory must not be released under
        // them) and leave this CTU unfiltered.
        if (t == 0) {
            atomicAdd(&g_tma_wait_expired, 1u);
            for (int i = 0; i < (1 << 22) && !mbar_try_wait(b, 0); ++i) {
            }
        }
        __syncthreads();
        return;
    }
    DeblockQp q;
    q.init(J.qp[k]);
    for (int i = t; i < DEBLOCK_VERT_ROWS; i += DFT) deblock_vert_rows(ty, tc[0], i, q);
    __syncthreads();
    for (int i = t; i < deblock_horiz_wide_items<4>(); i += DFT) deblock_horiz_wide<4>(ty, tc[0], tc[1], i, q);
    // the filters' shared-memory writes become visible to the bulk-copy
    // (async) proxy before the stores read the tile
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (t == 0) {
        tma_store_2d(&J.ty[k], smem_addr(ty), x0, y0);
        tma_store_2d(&J.tcb[k], smem_addr(tc[0]), x0 >> 1, y0 >> 1);
        tma_store_2d(&J.tcr[k], smem_addr(tc[1]), x0 >> 1, y0 >> 1);
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");   // tile read out before the CTA ends
    }
}

// ---------------------------------------------------------------- SAO

// Byte k (0..3) of w.
__device__ __forceinline__ int byte_k(uint32_t w, int k) { return (int)__byte_perm(w, 0, 0x4440 | k); }
// Byte i (0..15) of v, by selects (an indexed register array would live
// in local memory).
__device__ __forceinline__ int byte_i(const uint4 &v, int i) {
    const uint32_t w = i < 8 ? (i < 4 ? v.x : v.y) : (i < 12 ? v.z : v.w);
    return byte_k(w, i & 3);
}

// One sample pair into the thread's statistics column: the word of the
// sample's row (sao_row_of, computed: a lookup table would add a shared
// load with bank conflicts to every pixel) gains 65536 + SAO_BIAS + o - r.
template <int SFT>
__device__ __forceinline__ void sao_count(int *col, int r, int o) {
    col[sao_row_of(r) * SFT] += 65536 + (int)SAO_BIAS + o - r;
}

template <int SFT>
__global__ void __launch_bounds__(SFT) sao_frames_kernel(SaoJobs J) {
    constexpr int NSEG = 256 / SFT;           // 16-pixel segments per thread
    static_assert(SFT == 64 || SFT == 128, "SAO CTA: 256 16-pixel segments per CTU, table within 48 KB");
    // G columns of the table are summed before unpacking: a column holds
    // at most 16 * NSEG samples, and a sum of words splits exactly up to
    // 128 (sao_unpack).
    constexpr int G = NSEG <= 2 ? 4 : 2;
    constexpr int TPR = SFT >= 2 * SAO_ROWS ? 2 : 1;   // threads summing one row
    __shared__ __align__(16) int hist[SAO_ROWS][SFT];   // count * 65536 + sum of (256 + org - rec), per thread
    __shared__ int row_cnt[SAO_ROWS], row_sum[SAO_ROWS];
    __shared__ int red[SFT / 32];
    __shared__ int dec[3];
    const int k = find_frame(J.ctu_off, J.n, blockIdx.x);
    const SaoFrame &F = J.f[k];
    const int local = blockIdx.x - J.ctu_off[k], cols = (F.W + 63) >> 6;
    const int x0 = (local % cols) << 6, y0 = (local / cols) << 6;
    const int w = min(64, F.W - x0), h = min(64, F.H - y0);
    const int t = threadIdx.x;
    // segment j of this thread: row (t + j*SFT) >> 2, columns 16 * ((t + j*SFT) & 3)
    uint4 rv[NSEG], ov[NSEG];
    int nvalid[NSEG];
    bool vec[NSEG];
    const uint8_t *const rec0 = F.rec + (size_t)y0 * F.sr + x0, *const org0 = F.org + (size_t)y0 * F.so + x0;
    const bool full = w == 64 && h == 64 && aligned16(rec0, F.sr) && aligned16(org0, F.so);
#pragma unroll
    for (int j = 0; j < NSEG; ++j) {
        const int sg = t + j * SFT, row = sg >> 2, c0 = (sg & 3) * 16;
        if (full) {   // every segment whole and 16-byte aligned
            nvalid[j] = 16;
            vec[j] = true;
            rv[j] = __ldcs((const uint4 *)(rec0 + (size_t)row * F.sr + c0));
            ov[j] = __ldcs((const uint4 *)(org0 + (size_t)row * F.so + c0));
            continue;
        }
        nvalid[j] = row < h ? max(0, min(16, w - c0)) : 0;
        const uint8_t *gr = F.rec + (size_t)(y0 + row) * F.sr + x0 + c0;
        const uint8_t *go = F.org + (size_t)(y0 + row) * F.so + x0 + c0;
        vec[j] = nvalid[j] == 16 && aligned16(gr, F.sr) && aligned16(go, F.so);
        rv[j] = make_uint4(0, 0, 0, 0);
        ov[j] = make_uint4(0, 0, 0, 0);
        if (vec[j]) {
            rv[j] = __ldcs((const uint4 *)gr);
            ov[j] = __ldcs((const uint4 *)go);
        } else if (nvalid[j] > 0) {
            uint32_t r4[4] = {0, 0, 0, 0}, o4[4] = {0, 0, 0, 0};
#pragma unroll
            for (int i = 0; i < 16; ++i)
                if (i < nvalid[j]) { r4[i >> 2] |= (uint32_t)gr[i] << (8 * (i & 3)); o4[i >> 2] |= (uint32_t)go[i] << (8 * (i & 3)); }
            rv[j] = make_uint4(r4[0], r4[1], r4[2], r4[3]);
            ov[j] = make_uint4(o4[0], o4[1], o4[2], o4[3]);
        }
    }
    for (int i = t; i < SAO_ROWS * SFT / 4; i += SFT) ((int4 *)&hist[0][0])[i] = make_int4(0, 0, 0, 0);
    __syncthreads();
    // ---- pass 1: per-row (count, sum) and the unfiltered SSE (|d|^2 four
    // pixels at a time; padding bytes are zero in both vectors)
    int *col = &hist[0][t];
    int base = 0;
#pragma unroll
    for (int j = 0; j < NSEG; ++j) {
        const uint32_t rw[4] = {rv[j].x, rv[j].y, rv[j].z, rv[j].w}, ow[4] = {ov[j].x, ov[j].y, ov[j].z, ov[j].w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint32_t ad = __vabsdiffu4(rw[q], ow[q]);
            base = (int)__dp4a(ad, ad, (unsigned)base);
        }
        if (nvalid[j] == 16) {
            // rows and increments of four samples per word operation
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint32_t rows = sao_rows4(rw[q]);
                uint32_t even, odd;
                sao_incr4(rw[q], ow[q], even, odd);
                // shared-memory atomic adds with no result: one instruction
                // per sample instead of a load / add / store chain (the
                // column is private, so they never contend)
                atomicAdd(&col[(rows & 0xFF) * SFT], (int)sao_lane_lo(even));
                atomicAdd(&col[((rows >> 8) & 0xFF) * SFT], (int)sao_lane_lo(odd));
                atomicAdd(&col[((rows >> 16) & 0xFF) * SFT], (int)sao_lane_hi(even));
                atomicAdd(&col[(rows >> 24) * SFT], (int)sao_lane_hi(odd));
            }
        } else {
            for (int i = 0; i < nvalid[j]; ++i) sao_count<SFT>(col, byte_i(rv[j], i), byte_i(ov[j], i));
        }
    }
    const int bsum = __reduce_add_sync(0xffffffffu, (unsigned)base);
    if ((t & 31) == 0) red[t >> 5] = bsum;
    __syncthreads();
    // ---- row totals: TPR threads per row, summing G columns at a time
    // (16-byte loads) before unpacking
    if (t < TPR * SAO_ROWS) {
        const int row = t / TPR, part = t % TPR;
        const int4 *p = (const int4 *)&hist[row][part * (SFT / TPR)];
        int cnt = 0, sum = 0;
        auto unpack = [&](int x) { sao_unpack((uint32_t)x, cnt, sum); };
        // start each thread at its own 16-byte column group: the rows are
        // 128 words apart, so unrotated every lane would read the same banks
        constexpr int NV = SFT / TPR / 4;
        const int rot = (row * TPR + part) % NV;
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            const int4 v = p[(i + rot) % NV];
            if (G == 4) {
                unpack(v.x + v.y + v.z + v.w);
            } else {
                unpack(v.x + v.y);
                unpack(v.z + v.w);
            }
        }
        sum -= (int)SAO_BIAS * cnt;
        if (TPR == 2) {
            cnt += __shfl_xor_sync(0xffffffffu, cnt, 1);
            sum += __shfl_xor_sync(0xffffffffu, sum, 1);
        }
        if (!part) { row_cnt[row] = cnt; row_sum[row] = sum; }
    }
    __syncthreads();
    // ---- decision (warp 0): lane b scores band b; first band with the
    // smallest SSE; rate gate of 6 lambda
    if (t < 32) {
        int b0 = 0;
        for (int i = 0; i < SFT / 32; ++i) b0 += red[i];
        int cand;
        const int sse = sao_band_sse(t, b0, row_cnt, row_sum, &cand);
        int best = cand ? sse : b0;
        int bb = cand ? t : 32;
        for (int o = 16; o > 0; o >>= 1) {
            const int ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int obb = __shfl_xor_sync(0xffffffffu, bb, o);
            const int oc = __shfl_xor_sync(0xffffffffu, cand, o);
            if (ob < best || (ob == best && obb < bb)) { best = ob; bb = obb; cand = oc; }
        }
        if (t == 0) {
            int has = bb < 32 && best < b0;
            if (has && best + (long long)F.lambda_sao * 6 >= b0) has = 0;
            dec[0] = has;
            dec[1] = has ? bb : 0;
            dec[2] = has ? cand : 0;
            if (F.params) {
                int16_t *pp = F.params + 3 * local;
                pp[0] = (int16_t)dec[0]; pp[1] = (int16_t)dec[1]; pp[2] = (int16_t)dec[2];
            }
        }
    }
    __syncthreads();
    // ---- apply: bytes of the chosen band (exact per-byte test: band
    // indices are <= 31, so adding 0x7F sets bit 7 of every nonzero byte
    // without carries), offset on pairs; only segments with a hit are
    // written
    if (dec[0]) {
        const uint32_t bandx4 = (uint32_t)dec[1] * 0x01010101u, one = 0x00010001u;
        const uint32_t add = (uint32_t)(dec[2] + 128) * one, lo = 128u * one, hi = (128u + 255u) * one;
#pragma unroll
        for (int j = 0; j < NSEG; ++j) {
            if (nvalid[j] <= 0) continue;
            uint32_t wv[4] = {rv[j].x, rv[j].y, rv[j].z, rv[j].w}, hit[4];
            bool any = false;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint32_t tq = ((wv[q] >> 3) & 0x1F1F1F1Fu) ^ bandx4;
                hit[q] = ~(tq + 0x7F7F7F7Fu) & 0x80808080u;
                any |= hit[q] != 0;
            }
            if (!any) continue;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint32_t a = pair_min(pair_max(pair_lo(wv[q]) + add, lo), hi) - lo;
                const uint32_t b = pair_min(pair_max(pair_hi(wv[q]) + add, lo), hi) - lo;
                const uint32_t m = (hit[q] >> 7) * 0xFFu;
                wv[q] = (pair_pack(a, b) & m) | (wv[q] & ~m);
            }
            const int sg = t + j * SFT, row = sg >> 2, c0 = (sg & 3) * 16;
            uint8_t *gr = F.rec + (size_t)(y0 + row) * F.sr + x0 + c0;
            if (vec[j]) {
                __stcs((uint4 *)gr, make_uint4(wv[0], wv[1], wv[2], wv[3]));
            } else {
                const uint4 nv = make_uint4(wv[0], wv[1], wv[2], wv[3]);
                for (int i = 0; i < nvalid[j]; ++i) gr[i] = (uint8_t)byte_i(nv, i);
            }
        }
    }
}

}  // namespace

namespace {

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return (PFN_cuTensorMapEncodeTiled_v12000)p;
    }();
    return fn;
}

// 2D uint8 tensor map of a w x h plane with a box x box tile.
bool encode_plane(CUtensorMap *m, uint8_t *base, int w, int h, int stride, int box) {
    const auto enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)w, (cuuint64_t)h}, strides[1] = {(cuuint64_t)stride};
    const cuuint32_t boxd[2] = {(cuuint32_t)box, (cuuint32_t)box}, estr[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, base, dims, strides, boxd, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool tma_ok(const DeblockFrame &f) {
    auto al = [](const void *p, int s) { return (((uintptr_t)p) & 15) == 0 && (s & 15) == 0; };
    return al(f.y, f.sy) && al(f.cb, f.sc) && al(f.cr, f.sc) && f.W >= 64 && f.H >= 64;
}

}  // namespace

unsigned int tma_waits_expired() {
    unsigned int v = 0, z = 0;
    cudaMemcpyFromSymbol(&v, g_tma_wait_expired, sizeof(v));
    cudaMemcpyToSymbol(g_tma_wait_expired, &z, sizeof(z));
    return v;
}

namespace {

cudaError_t launch_group_tma(const DeblockFrame *frames, int m, cudaStream_t st, int threads) {
    DeblockTmaJobs J;
    memset(&J, 0, sizeof(J));
    int total = 0;
    for (int j = 0; j < m; ++j) {
        const DeblockFrame &f = frames[j];
        if (!encode_plane(&J.ty[j], f.y, f.W, f.H, f.sy, 64) ||
            !encode_plane(&J.tcb[j], f.cb, f.W / 2, f.H / 2, f.sc, 32) ||
            !encode_plane(&J.tcr[j], f.cr, f.W / 2, f.H / 2, f.sc, 32))
            return cudaErrorInvalidValue;
        J.ctu_off[j] = total;
        J.cols[j] = f.W >> 6;
        J.qp[j] = f.qp;
        total += (f.W >> 6) * (f.H >> 6);
    }
    J.n = m;
    J.ctu_off[m] = total;
    if (total == 0) return cudaSuccess;
    if (threads == 64) deblock_tma_kernel<64><<<total, 64, 0, st>>>(J);
    else if (threads == 256) deblock_tma_kernel<256><<<total, 256, 0, st>>>(J);
    else deblock_tma_kernel<128><<<total, 128, 0, st>>>(J);
    return cudaGetLastError();
}

cudaError_t launch_group_vec(const DeblockFrame *frames, int m, cudaStream_t st, int threads) {
    DeblockJobs J;
    J.n = m;
    int total = 0;
    for (int j = 0; j < m; ++j) {
        J.f[j] = frames[j];
        J.ctu_off[j] = total;
        total += (frames[j].W >> 6) * (frames[j].H >> 6);
    }
    J.ctu_off[m] = total;
    if (total == 0) return cudaSuccess;
    if (threads == 64) deblock_frames_kernel<64><<<total, 64, 0, st>>>(J);
    else if (threads == 256) deblock_frames_kernel<256><<<total, 256, 0, st>>>(J);
    else deblock_frames_kernel<128><<<total, 128, 0, st>>>(J);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_deblock_frames(const DeblockFrame *frames, int n, cudaStream_t st, int variant) {
    // TMA staging when the variant asks for it and every frame of a launch
    // group meets the tensor-map alignment; 16-byte vector loads otherwise
    const bool want_tma = (variant & TCB_STAGING_TMA) != 0;
    const int threads = variant & ~TCB_STAGING_TMA;
    static_assert((int)DeblockJobs::MAX == (int)DeblockTmaJobs::MAX, "one group size");
    for (int i = 0; i < n;) {
        const int m = n - i < DeblockJobs::MAX ? n - i : DeblockJobs::MAX;
        bool tma = want_tma && tensor_map_encoder() != nullptr;
        for (int j = 0; tma && j < m; ++j) tma = tma_ok(frames[i + j]);
        const cudaError_t e = tma ? launch_group_tma(frames + i, m, st, threads)
                                  : launch_group_vec(frames + i, m, st, threads);
        if (e != cudaSuccess) return e;
        i += m;
    }
    return cudaSuccess;
}

cudaError_t launch_sao_frames(const SaoFrame *frames, int n, cudaStream_t st, int threads) {
    for (int i = 0; i < n;) {
        SaoJobs J;
        J.n = 0;
        int total = 0;
        while (i < n && J.n < SaoJobs::MAX) {
            J.f[J.n] = frames[i];
            J.ctu_off[J.n] = total;
            total += ((frames[i].W + 63) >> 6) * ((frames[i].H + 63) >> 6);
            ++J.n;
            ++i;
        }
        J.ctu_off[J.n] = total;
        if (total > 0) {
            if (threads == 64) sao_frames_kernel<64><<<total, 64, 0, st>>>(J);
            else sao_frames_kernel<128><<<total, 128, 0, st>>>(J);
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

}  // namespace tcb

// ---------------------------------------------------------------- C ABI
#include <vector>

#include "../../include/tcodec_b200.h"
#include "tcb_encoder.h"

namespace {

bool frame_ok(const tcb_filter_frame_t &f) {
    return f.width > 0 && f.height > 0 && !(f.width & 1) && !(f.height & 1) && f.width <= TC_MAX_WIDTH &&
           f.height <= TC_MAX_HEIGHT && f.stride_y >= f.width && f.stride_c >= f.width / 2 && f.y && f.cb && f.cr &&
           f.qp >= 0 && f.qp <= 63;
}


}  // namespace

extern "C" {

tc_error_t tcb_deblock_frames(const tcb_filter_frame_t *frames, int n, void *stream) {
    if (n < 0 || (n > 0 && !frames)) return TC_ERR_PARAM;
    std::vector<tcb::DeblockFrame> v(n);
    for (int i = 0; i < n; ++i) {
        const tcb_filter_frame_t &f = frames[i];
        if (!frame_ok(f)) return TC_ERR_PARAM;
        v[i] = {f.y, f.cb, f.cr, f.width, f.height, f.stride_y, f.stride_c, f.qp};
    }
    const int threads = n ? tcb::tuned_threads(TCB_KERNEL_DEBLOCK, frames[0].width, frames[0].height) : 0;
    return tcb::launch_deblock_frames(v.data(), n, (cudaStream_t)stream, threads) == cudaSuccess ? TC_OK
                                                                                               : TC_ERR_INTERNAL;
}

tc_error_t tcb_sao_frames(const tcb_filter_frame_t *frames, int n, void *stream) {
    if (n < 0 || (n > 0 && !frames)) return TC_ERR_PARAM;
    std::vector<tcb::SaoFrame> v(n);
    for (int i = 0; i < n; ++i) {
        const tcb_filter_frame_t &f = frames[i];
        if (!frame_ok(f) || !f.src_y || f.stride_src < f.width) return TC_ERR_PARAM;
        v[i] = {f.y, f.src_y, f.width, f.height, f.stride_y, f.stride_src, (int)tcb::tc_lambda_host(f.qp), f.sao_params};
    }
    const int threads = n ? tcb::tuned_threads(TCB_KERNEL_SAO, frames[0].width, frames[0].height) : 0;
    return tcb::launch_sao_frames(v.data(), n, (cudaStream_t)stream, threads) == cudaSuccess ? TC_OK
                                                                                           : TC_ERR_INTERNAL;
}

}  // extern "C"
