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
// count * 65536 + sum (|sum| <= 32 * 255), which one integer add per pixel
// maintains exactly.  Rows are the 30 inner bands plus the 16 single
// sample values of bands 0 and 31, where an offset can clip; the SSE of
// every band after its offset then follows in closed form, clipping
// included (tcb_sao_decide.cuh), with no second pass over the pixels.
#include <cuda_runtime.h>

#include "tcb_common.cuh"
#include "tcb_deblock_pairs.cuh"
#include "tcb_filters.h"
#include "tcb_pixel.cuh"
#include "tcb_sao_decide.cuh"

namespace tcb {

namespace {

// Threads per CTA (one CTU each).  Small CTAs let many CTUs' loads be in
// flight per SM while other CTUs of the same SM filter.
#ifndef TCB_DEBLOCK_FT
#define TCB_DEBLOCK_FT 128
#endif
#ifndef TCB_SAO_FT
#define TCB_SAO_FT 128
#endif
constexpr int DFT = TCB_DEBLOCK_FT, SFT = TCB_SAO_FT;
static_assert(384 % DFT == 0 && DFT >= 32, "deblock CTA: 384 16-byte pieces per CTU");
static_assert(256 % SFT == 0 && SFT >= 32 && SFT <= 256, "SAO CTA: 256 16-pixel segments per CTU");

__device__ __forceinline__ int find_frame(const int *off, int n, int g) {
    int k = 0;
    while (k + 1 < n && off[k + 1] <= g) ++k;
    return k;
}

__device__ __forceinline__ bool aligned16(const void *p, int stride) {
    return (((uintptr_t)p) & 15) == 0 && (stride & 15) == 0;
}

// ---------------------------------------------------------------- deblock

__global__ void __launch_bounds__(DFT) deblock_frames_kernel(DeblockJobs J) {
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
        uint4 v[384 / DFT];
#pragma unroll
        for (int j = 0; j < 384 / DFT; ++j) {
            const int p = t + j * DFT;
            if (p < 256) {
                v[j] = __ldcs((const uint4 *)(gy + (size_t)(p >> 2) * F.sy + (p & 3) * 16));
            } else {
                const int q = p - 256, c = q >> 6, r = (q >> 1) & 31, sg = q & 1;
                v[j] = __ldcs((const uint4 *)(gc(c) + (size_t)r * F.sc + sg * 16));
            }
        }
#pragma unroll
        for (int j = 0; j < 384 / DFT; ++j) {
            const int p = t + j * DFT;
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
    // ---- vertical edges, then horizontal edges, as independent two-lane
    // items (tcb_deblock_pairs.cuh): 640 vertical items (5 per thread at
    // 128 threads), 296 horizontal
    DeblockQp q;
    q.init(F.qp);
    for (int i = t; i < DEBLOCK_VERT_ITEMS; i += DFT) deblock_vert(ty, tc[0], i, q);
    __syncthreads();
    for (int i = t; i < DEBLOCK_HORIZ_ITEMS; i += DFT) deblock_horiz(ty, tc[0], tc[1], i, q);
    __syncthreads();
    // ---- store
    if (vec) {
#pragma unroll
        for (int j = 0; j < 384 / DFT; ++j) {
            const int p = t + j * DFT;
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

// ---------------------------------------------------------------- SAO

// Byte k (0..3) of w.
__device__ __forceinline__ int byte_k(uint32_t w, int k) { return (int)__byte_perm(w, 0, 0x4440 | k); }
// Byte i (0..15) of v, by selects (an indexed register array would live
// in local memory).
__device__ __forceinline__ int byte_i(const uint4 &v, int i) {
    const uint32_t w = i < 8 ? (i < 4 ? v.x : v.y) : (i < 12 ? v.z : v.w);
    return byte_k(w, i & 3);
}

// One sample pair into the thread's statistics column: the word at
// row_word[r] (the row's offset in the table) gains count 1 and o - r.
__device__ __forceinline__ void sao_count(int *col, const int *row_word, int r, int o) {
    col[row_word[r]] += 65536 + o - r;
}

__global__ void __launch_bounds__(SFT) sao_frames_kernel(SaoJobs J) {
    constexpr int NSEG = 256 / SFT;           // 16-pixel segments per thread
    // Four columns of the table are summed before unpacking: a column
    // holds at most 16 * NSEG pixels, so four columns keep |sum| below
    // 4 * 16 * NSEG * 255 = 32640 for NSEG = 2, inside the 16-bit field.
    static_assert(SFT == 128, "SAO table reduction sized for 128 threads");
    __shared__ __align__(16) int hist[SAO_ROWS][SFT];   // count * 65536 + sum of (org - rec), per thread
    __shared__ int row_word[256];             // sample value -> word offset of its statistics row
    __shared__ int row_cnt[SAO_ROWS], row_sum[SAO_ROWS];
    __shared__ long long red[SFT / 32];
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
#pragma unroll
    for (int j = 0; j < NSEG; ++j) {
        const int sg = t + j * SFT, row = sg >> 2, c0 = (sg & 3) * 16;
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
    for (int i = t; i < 256; i += SFT) row_word[i] = sao_row_of(i) * SFT;
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
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int b = 0; b < 4; ++b) sao_count(col, row_word, byte_k(rw[q], b), byte_k(ow[q], b));
        } else {
            for (int i = 0; i < nvalid[j]; ++i) sao_count(col, row_word, byte_i(rv[j], i), byte_i(ov[j], i));
        }
    }
    long long bsum = base;
    for (int o = 16; o > 0; o >>= 1) bsum += __shfl_xor_sync(0xffffffffu, bsum, o);
    if ((t & 31) == 0) red[t >> 5] = bsum;
    __syncthreads();
    // ---- row totals: two threads per row, each summing 64 columns four at
    // a time (16-byte loads) before unpacking
    if (t < 2 * SAO_ROWS) {
        const int row = t >> 1, half = t & 1;
        const int4 *p = (const int4 *)&hist[row][half * (SFT / 2)];
        int cnt = 0, sum = 0;
#pragma unroll
        for (int i = 0; i < SFT / 8; ++i) {
            const int4 v = p[i];
            const int x = v.x + v.y + v.z + v.w;
            const int sv = (int)(int16_t)(x & 0xffff);
            sum += sv;
            cnt += (x - sv) >> 16;
        }
        cnt += __shfl_xor_sync(0xffffffffu, cnt, 1);
        sum += __shfl_xor_sync(0xffffffffu, sum, 1);
        if (!half) { row_cnt[row] = cnt; row_sum[row] = sum; }
    }
    __syncthreads();
    // ---- decision (warp 0): lane b scores band b; first band with the
    // smallest SSE; rate gate of 6 lambda
    if (t < 32) {
        long long b0 = 0;
        for (int i = 0; i < SFT / 32; ++i) b0 += red[i];
        int cand;
        const long long sse = sao_band_sse(t, b0, row_cnt, row_sum, &cand);
        long long best = cand ? sse : b0;
        int bb = cand ? t : 32;
        for (int o = 16; o > 0; o >>= 1) {
            const long long ob = __shfl_xor_sync(0xffffffffu, best, o);
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

cudaError_t launch_deblock_frames(const DeblockFrame *frames, int n, cudaStream_t st) {
    for (int i = 0; i < n;) {
        DeblockJobs J;
        J.n = 0;
        int total = 0;
        while (i < n && J.n < DeblockJobs::MAX) {
            J.f[J.n] = frames[i];
            J.ctu_off[J.n] = total;
            total += (frames[i].W >> 6) * (frames[i].H >> 6);
            ++J.n;
            ++i;
        }
        J.ctu_off[J.n] = total;
        if (total > 0) {
            deblock_frames_kernel<<<total, DFT, 0, st>>>(J);
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

cudaError_t launch_sao_frames(const SaoFrame *frames, int n, cudaStream_t st) {
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
            sao_frames_kernel<<<total, SFT, 0, st>>>(J);
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
    return tcb::launch_deblock_frames(v.data(), n, (cudaStream_t)stream) == cudaSuccess ? TC_OK : TC_ERR_INTERNAL;
}

tc_error_t tcb_sao_frames(const tcb_filter_frame_t *frames, int n, void *stream) {
    if (n < 0 || (n > 0 && !frames)) return TC_ERR_PARAM;
    std::vector<tcb::SaoFrame> v(n);
    for (int i = 0; i < n; ++i) {
        const tcb_filter_frame_t &f = frames[i];
        if (!frame_ok(f) || !f.src_y || f.stride_src < f.width) return TC_ERR_PARAM;
        v[i] = {f.y, f.src_y, f.width, f.height, f.stride_y, f.stride_src, (int)tcb::tc_lambda_host(f.qp), f.sao_params};
    }
    return tcb::launch_sao_frames(v.data(), n, (cudaStream_t)stream) == cudaSuccess ? TC_OK : TC_ERR_INTERNAL;
}

}  // extern "C"
