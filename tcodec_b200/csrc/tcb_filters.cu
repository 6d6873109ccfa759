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
// Both are HBM-bound byte kernels: one 256-thread CTA per CTU, the tile
// moved with 16-byte loads and stores (a byte path serves unaligned
// planes), each byte read once and written at most once.
//
// SAO statistics without atomics: every thread owns 16 pixels of one row
// (kept in registers for the whole CTU) and a private column of a
// [band][thread] table in shared memory, so its read-modify-writes never
// conflict.  A table word packs count and difference sum as
// count * 65536 + sum (|sum| <= 16 * 255), which one integer add per pixel
// maintains exactly.  The per-band SSE after an offset follows in closed
// form from (count, sum) and the unfiltered SSE; only pixels of bands 0 and
// 31, where the offset can clip, get an exact per-pixel correction.
#include <cuda_runtime.h>

#include "tcb_common.cuh"
#include "tcb_filters.h"
#include "tcb_pixel.cuh"

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
    uint8_t *gc[2] = {F.cb + (size_t)(y0 >> 1) * F.sc + (x0 >> 1), F.cr + (size_t)(y0 >> 1) * F.sc + (x0 >> 1)};
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
                v[j] = __ldcs((const uint4 *)(gc[c] + (size_t)r * F.sc + sg * 16));
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
            tc[c][p] = gc[c][(size_t)(p >> 5) * F.sc + (p & 31)];
        }
    }
    __syncthreads();
    const int qp = F.qp, ltc = clampi(qp / 3, 1, 10);
    const int cqp = clampi(qp - 1, 0, 63), ctc = clampi(cqp / 4, 1, 6);
    // ---- vertical edges: luma x = 4..60 (rows 0..63), Cb x = 4..28; items
    // are (row, edge) on 16 / 8 slots per row so the decode is shifts and
    // slot 0 (no edge) idles
    for (int i = t; i < 16 * 64 + 8 * 32; i += DFT) {
        if (i < 16 * 64) {
            const int r = i >> 4, e = i & 15;
            if (e == 0) continue;
            const int x = e * 4;
            uint8_t *p = &ty[r * 64 + x];
            const int p1 = p[-2], p0 = p[-1], q0 = p[0], q1 = p[1];
            if (edge_strength(p0, q0, qp)) {
                p[-1] = (uint8_t)weak_filter(p1, p0, q0, q1, ltc);
                p[0] = (uint8_t)weak_filter(q1, q0, p0, p1, ltc);
            }
        } else {
            const int j = i - 16 * 64, r = j >> 3, e = j & 7;
            if (e == 0) continue;
            const int x = e * 4;
            uint8_t *p = &tc[0][r * 32 + x];
            const int p0 = p[-1], q0 = p[0];
            if (edge_strength(p0, q0, cqp)) {
                const int d = clampi((q0 - p0 + 1) >> 1, -ctc, ctc);
                p[-1] = (uint8_t)clampi(p0 + d, 0, 255);
                p[0] = (uint8_t)clampi(q0 - d, 0, 255);
            }
        }
    }
    __syncthreads();
    // ---- horizontal edges: luma y = 4..60; chroma rows (4e, 4e+1),
    // e = 1..7, with the Cr strength deciding for both planes
    for (int i = t; i < 15 * 64 + 7 * 32; i += DFT) {
        if (i < 15 * 64) {
            const int y = ((i >> 6) + 1) * 4, c = i & 63;
            uint8_t *p = &ty[y * 64 + c];
            const int p1 = p[-128], p0 = p[-64], q0 = p[0], q1 = p[64];
            if (edge_strength(p0, q0, qp)) {
                p[-64] = (uint8_t)weak_filter(p1, p0, q0, q1, ltc);
                p[0] = (uint8_t)weak_filter(q1, q0, p0, p1, ltc);
            }
        } else {
            const int j = i - 15 * 64, y = ((j >> 5) + 1) * 4, c = j & 31;
            uint8_t *pr = &tc[1][y * 32 + c], *pb = &tc[0][y * 32 + c];
            const int p0 = pr[0], q0 = pr[32], b0 = pb[0], b1 = pb[32];
            if (edge_strength(p0, q0, cqp)) {
                int d = clampi((q0 - p0 + 1) >> 1, -ctc, ctc);
                pr[0] = (uint8_t)clampi(p0 + d, 0, 255);
                pr[32] = (uint8_t)clampi(q0 - d, 0, 255);
                d = clampi((b1 - b0 + 1) >> 1, -ctc, ctc);
                pb[0] = (uint8_t)clampi(b0 + d, 0, 255);
                pb[32] = (uint8_t)clampi(b1 - d, 0, 255);
            }
        }
    }
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
                __stcs((uint4 *)(gc[c] + (size_t)r * F.sc + sg * 16), *(const uint4 *)&tc[c][r * 32 + sg * 16]);
            }
        }
    } else {
        for (int i = t; i < 64 * 64; i += DFT) gy[(size_t)(i >> 6) * F.sy + (i & 63)] = ty[i];
        for (int i = t; i < 2 * 32 * 32; i += DFT) {
            const int c = i >> 10, p = i & 1023;
            gc[c][(size_t)(p >> 5) * F.sc + (p & 31)] = tc[c][p];
        }
    }
}

// ---------------------------------------------------------------- SAO

__device__ __forceinline__ uint8_t byte_of(const uint4 &v, int k) {
    const uint32_t w = k < 8 ? (k < 4 ? v.x : v.y) : (k < 12 ? v.z : v.w);
    return (uint8_t)(w >> ((k & 3) * 8));
}

// Packs bytes b[0..15] into a uint4 (little endian within each word).
__device__ __forceinline__ uint4 pack16(const uint8_t *b) {
    uint4 v;
    v.x = b[0] | b[1] << 8 | b[2] << 16 | (uint32_t)b[3] << 24;
    v.y = b[4] | b[5] << 8 | b[6] << 16 | (uint32_t)b[7] << 24;
    v.z = b[8] | b[9] << 8 | b[10] << 16 | (uint32_t)b[11] << 24;
    v.w = b[12] | b[13] << 8 | b[14] << 16 | (uint32_t)b[15] << 24;
    return v;
}

__global__ void __launch_bounds__(SFT) sao_frames_kernel(SaoJobs J) {
    constexpr int NSEG = 256 / SFT;           // 16-pixel segments per thread
    constexpr int TPB = SFT / 32;             // threads summing one band
    __shared__ int hist[32][SFT];             // count * 65536 + sum, per thread
    __shared__ int band_cnt[32], band_sum[32], corr[32];
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
            uint8_t rb[16] = {0}, ob[16] = {0};
            for (int i = 0; i < nvalid[j]; ++i) { rb[i] = gr[i]; ob[i] = go[i]; }
            rv[j] = pack16(rb);
            ov[j] = pack16(ob);
        }
    }
#pragma unroll
    for (int b = 0; b < 32; ++b) hist[b][t] = 0;
    if (t < 32) corr[t] = 0;
    // ---- pass 1: per-band (count, sum) and the unfiltered SSE (|d|^2
    // four pixels at a time; padding bytes are zero in both vectors)
    int base = 0;
    bool edge_band = false;                   // any pixel in band 0 or 31
#pragma unroll
    for (int j = 0; j < NSEG; ++j) {
        const uint32_t rw[4] = {rv[j].x, rv[j].y, rv[j].z, rv[j].w}, ow[4] = {ov[j].x, ov[j].y, ov[j].z, ov[j].w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint32_t ad = __vabsdiffu4(rw[q], ow[q]);
            base = (int)__dp4a(ad, ad, (unsigned)base);
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            if (i < nvalid[j]) {
                const int r = byte_of(rv[j], i), d = (int)byte_of(ov[j], i) - r;
                hist[r >> 3][t] += 65536 + d;
                edge_band |= (unsigned)(r - 8) >= 240u;
            }
        }
    }
    long long bsum = base;
    for (int o = 16; o > 0; o >>= 1) bsum += __shfl_xor_sync(0xffffffffu, bsum, o);
    if ((t & 31) == 0) red[t >> 5] = bsum;
    const bool any_edge = __syncthreads_or(edge_band);
    // ---- per-band totals: TPB threads per band, SFT / TPB columns each
    {
        const int b = t / TPB, part = t - b * TPB;
        int cnt = 0, sum = 0;
        for (int j = part; j < SFT; j += TPB) {
            const int v = hist[b][j];
            const int sv = (int)(int16_t)(v & 0xffff);
            sum += sv;
            cnt += (v - sv) >> 16;
        }
        for (int o = 1; o < TPB; o <<= 1) {
            cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
            sum += __shfl_xor_sync(0xffffffffu, sum, o);
        }
        if (part == 0) { band_cnt[b] = cnt; band_sum[b] = sum; }
    }
    __syncthreads();
    // ---- pass 2: exact correction where the offset clips (bands 0, 31)
    auto cand_of = [&](int b) {
        const int cnt = band_cnt[b], sum = band_sum[b];
        if (!cnt) return 0;
        return clampi((sum + (sum >= 0 ? cnt / 2 : -(cnt / 2))) / cnt, -7, 7);
    };
    if (any_edge) {
        const int c_lo = cand_of(0), c_hi = cand_of(31);
        int lo = 0, hi = 0;
#pragma unroll
        for (int j = 0; j < NSEG; ++j)
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                if (i < nvalid[j]) {
                    const int r = byte_of(rv[j], i), o = byte_of(ov[j], i), d = o - r;
                    const int cand = r < 8 ? c_lo : (r >= 248 ? c_hi : 0);
                    const int v = r + cand;
                    if (cand && (v < 0 || v > 255)) {
                        const int e = o - clampi(v, 0, 255);
                        const int fix = (e * e - d * d) - (cand * cand - 2 * d * cand);
                        if (r < 8) lo += fix; else hi += fix;
                    }
                }
            }
        if (lo) atomicAdd(&corr[0], lo);
        if (hi) atomicAdd(&corr[31], hi);
    }
    __syncthreads();
    // ---- decision (warp 0): first band with the smallest SSE, rate gate
    if (t < 32) {
        long long b0 = 0;
        for (int i = 0; i < SFT / 32; ++i) b0 += red[i];
        const int cand = cand_of(t);
        long long sse = b0;
        const bool ok = band_cnt[t] > 0 && cand != 0;
        if (ok) sse = b0 - 2LL * cand * band_sum[t] + (long long)band_cnt[t] * cand * cand + corr[t];
        long long best = ok ? sse : b0;
        int bb = ok ? t : 32;
        for (int o = 16; o > 0; o >>= 1) {
            const long long ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int obb = __shfl_xor_sync(0xffffffffu, bb, o);
            if (ob < best || (ob == best && obb < bb)) { best = ob; bb = obb; }
        }
        if (t == 0) {
            int has = bb < 32 && best < b0;
            if (has && best + (long long)F.lambda_sao * 6 >= b0) has = 0;
            dec[0] = has;
            dec[1] = has ? bb : 0;
            dec[2] = has ? cand_of(bb) : 0;
            if (F.params) {
                int16_t *pp = F.params + 3 * local;
                pp[0] = (int16_t)dec[0]; pp[1] = (int16_t)dec[1]; pp[2] = (int16_t)dec[2];
            }
        }
    }
    __syncthreads();
    // ---- apply (only segments holding pixels of the chosen band are written)
    if (dec[0]) {
        const int band = dec[1], off = dec[2];
#pragma unroll
        for (int j = 0; j < NSEG; ++j) {
            if (nvalid[j] <= 0) continue;
            const int sg = t + j * SFT, row = sg >> 2, c0 = (sg & 3) * 16;
            uint8_t *gr = F.rec + (size_t)(y0 + row) * F.sr + x0 + c0;
            uint8_t nb[16];
            bool any = false;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int r = byte_of(rv[j], i);
                const bool hit = i < nvalid[j] && (r >> 3) == band;
                nb[i] = hit ? (uint8_t)clampi(r + off, 0, 255) : (uint8_t)r;
                any |= hit;
            }
            if (!any) continue;
            if (vec[j]) __stcs((uint4 *)gr, pack16(nb));
            else for (int i = 0; i < nvalid[j]; ++i) gr[i] = nb[i];
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
