// CPU check of the packed 16-bit lane routines that the frame kernels run
// (they are __host__ __device__), against the oracle's C restatement:
//   * MC: mc_luma_six_tap with the run-time phase selector and with each
//     of the 15 compile-time phases, mc_chroma_bilinear, on row strides that
//     are multiples of 4 (the kernels' condition for the packed path),
//     against or_pred_luma / or_pred_chroma;
//   * deblocking: every vertical and horizontal work item of a CTU (the
//     vertical ones also as whole rows), run in a random order, against
//     or_deblock_ctu;
//   * SAO: the closed-form band SSE (sao_band_sse) against a brute-force
//     SSE of the offset, clipped CTU, and the word-level statistics
//     helpers (sao_rows4, sao_incr4, sao_unpack) exhaustively.
// Built for the host only by tests/test_packed_lanes.py; exit status 0 when
// every case matches.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "../oracle/tcoracle.h"
#include "../tcodec_b200/csrc/tcb_deblock_pairs.cuh"
#include "../tcodec_b200/csrc/tcb_mc_pairs.cuh"
#include "../tcodec_b200/csrc/tcb_sao_decide.cuh"

using namespace tcb;

namespace {

template <int DX, int DY>
void luma_fixed(const uint8_t *r, int s, int fx, int fy, int h, uint32_t *o) {
    mc_luma_six_tap(r, s, fx, fy, h, PairPhaseFixed<DX, DY>(), o);
}
void luma_phase(int phase, const uint8_t *r, int s, int fx, int fy, int h, uint32_t *o) {
    switch (phase) {
        case 1: luma_fixed<0, 1>(r, s, fx, fy, h, o); break;
        case 2: luma_fixed<0, 2>(r, s, fx, fy, h, o); break;
        case 3: luma_fixed<0, 3>(r, s, fx, fy, h, o); break;
        case 4: luma_fixed<1, 0>(r, s, fx, fy, h, o); break;
        case 5: luma_fixed<1, 1>(r, s, fx, fy, h, o); break;
        case 6: luma_fixed<1, 2>(r, s, fx, fy, h, o); break;
        case 7: luma_fixed<1, 3>(r, s, fx, fy, h, o); break;
        case 8: luma_fixed<2, 0>(r, s, fx, fy, h, o); break;
        case 9: luma_fixed<2, 1>(r, s, fx, fy, h, o); break;
        case 10: luma_fixed<2, 2>(r, s, fx, fy, h, o); break;
        case 11: luma_fixed<2, 3>(r, s, fx, fy, h, o); break;
        case 12: luma_fixed<3, 0>(r, s, fx, fy, h, o); break;
        case 13: luma_fixed<3, 1>(r, s, fx, fy, h, o); break;
        case 14: luma_fixed<3, 2>(r, s, fx, fy, h, o); break;
        default: luma_fixed<3, 3>(r, s, fx, fy, h, o); break;
    }
}

// Sample content: uniform noise, binary extremes (the lane ranges' worst
// cases), or a flat area with small noise.
void fill(std::vector<uint8_t> &f, int kind, std::mt19937 &rng) {
    for (auto &v : f)
        v = kind == 0 ? rng() & 255 : (kind == 1 ? ((rng() & 1) ? 255 : 0) : 128 + (int)(rng() % 5));
}

long check_mc(std::mt19937 &rng, long &blocks) {
    long bad = 0;
    for (int it = 0; it < 60; ++it) {
        const int W = 40 + rng() % 100, H = 30 + rng() % 80, s = ((W + 3) & ~3) + 4 * (rng() % 3);
        std::vector<uint8_t> f((size_t)s * H + 64);
        fill(f, it % 3, rng);
        for (int k = 0; k < 64; ++k) {
            const int fx = 2 + rng() % (W - 12), fy = 2 + rng() % (H - 12), phase = 1 + rng() % 15;
            const int dx = phase >> 2, dy = phase & 3;
            uint8_t want[64];
            or_pred_luma(f.data(), s, W, H, fx * 4 + dx, fy * 4 + dy, want, 8, 8);
            PairPhase ph;
            ph.init(dx, dy);
            for (int v = 0; v < 4; ++v) {           // halves 0, 1: selector; 2, 3: fixed phase
                uint32_t out[8];
                if (v < 2) mc_luma_six_tap(f.data(), s, fx, fy, v, ph, out);
                else luma_phase(phase, f.data(), s, fx, fy, v - 2, out);
                for (int y = 0; y < 8; ++y)
                    for (int x = 0; x < 4; ++x)
                        bad += ((out[y] >> (8 * x)) & 255) != want[y * 8 + 4 * (v & 1) + x];
            }
            ++blocks;
            const int mvx = rng() % (8 * (W - 6)), mvy = rng() % (8 * (H - 6)), xi = mvx >> 3, yi = mvy >> 3;
            if (xi + 4 < W && yi + 4 < H) {
                uint8_t wc[16];
                or_pred_chroma(f.data(), s, W, H, mvx, mvy, wc, 4, 4);
                uint32_t out[4];
                mc_chroma_bilinear(f.data(), s, xi, yi, mvx & 7, mvy & 7, out);
                for (int y = 0; y < 4; ++y)
                    for (int x = 0; x < 4; ++x) bad += ((out[y] >> (8 * x)) & 255) != wc[y * 4 + x];
            }
        }
    }
    return bad;
}

long check_deblock(std::mt19937 &rng, long &ctus) {
    long bad = 0;
    for (int it = 0; it < 600; ++it) {
        alignas(16) uint8_t ty[64 * 64], tb[32 * 32], tr[32 * 32];
        const int kind = it % 4, qp = rng() % 64, base = rng() % 256, amp = 1 + rng() % 60;
        auto near = [&]() { return (uint8_t)std::min(255, std::max(0, base + (int)(rng() % (2 * amp + 1)) - amp)); };
        for (int i = 0; i < 64 * 64; ++i)
            ty[i] = kind == 0 ? rng() & 255
                    : kind == 1 ? near()
                    : kind == 2 ? ((rng() & 1) ? 255 : 0)
                                : (uint8_t)(base + ((i & 63) / 4) * 3 + (i >> 8));
        for (int i = 0; i < 32 * 32; ++i) {
            tb[i] = kind == 2 ? ((rng() & 1) ? 250 : 3) : near();
            tr[i] = kind == 0 ? rng() & 255 : near();
        }
        uint8_t wy[64 * 64], wb[32 * 32], wr[32 * 32];
        memcpy(wy, ty, sizeof wy);
        memcpy(wb, tb, sizeof wb);
        memcpy(wr, tr, sizeof wr);
        or_deblock_ctu(wy, 64, wb, 32, wr, 32, 0, 0, qp);
        DeblockQp q;
        q.init(qp);
        // vertical phase as single items (even iterations) or as whole
        // rows (odd), both in a random order
        const int nv = (it & 1) ? DEBLOCK_VERT_ROWS : DEBLOCK_VERT_ITEMS;
        std::vector<int> ord(nv);
        for (int i = 0; i < nv; ++i) ord[i] = i;
        std::shuffle(ord.begin(), ord.end(), rng);
        for (int i : ord) {
            if (it & 1) deblock_vert_rows(ty, tb, i, q);
            else deblock_vert(ty, tb, i, q);
        }
        // horizontal phase with luma items 1, 2 or 4 words wide
        const int wpi = 1 << (it % 3);
        const int nh = wpi == 1 ? deblock_horiz_wide_items<1>() : wpi == 2 ? deblock_horiz_wide_items<2>()
                                                                         : deblock_horiz_wide_items<4>();
        ord.resize(nh);
        for (int i = 0; i < nh; ++i) ord[i] = i;
        std::shuffle(ord.begin(), ord.end(), rng);
        for (int i : ord) {
            if (wpi == 1) deblock_horiz_wide<1>(ty, tb, tr, i, q);
            else if (wpi == 2) deblock_horiz_wide<2>(ty, tb, tr, i, q);
            else deblock_horiz_wide<4>(ty, tb, tr, i, q);
        }
        bad += memcmp(ty, wy, sizeof wy) != 0 || memcmp(tb, wb, sizeof wb) != 0 || memcmp(tr, wr, sizeof wr) != 0;
        ++ctus;
    }
    return bad;
}

long check_sao(std::mt19937 &rng, long &bands) {
    long bad = 0;
    for (int it = 0; it < 200; ++it) {
        int org[64 * 64], rec[64 * 64];
        const int kind = it % 3;
        for (int i = 0; i < 64 * 64; ++i) {
            // values crowd the clipped ends (0..7, 248..255) in two of three cases
            rec[i] = kind == 0 ? rng() & 255 : kind == 1 ? rng() % 16 : 240 + rng() % 16;
            org[i] = std::min(255, std::max(0, rec[i] + (int)(rng() % 31) - 15));
        }
        int cnt[SAO_ROWS] = {}, sum[SAO_ROWS] = {};
        int base = 0;
        for (int i = 0; i < 64 * 64; ++i) {
            const int r = sao_row_of(rec[i]);
            ++cnt[r];
            sum[r] += org[i] - rec[i];
            base += (org[i] - rec[i]) * (org[i] - rec[i]);
        }
        for (int b = 0; b < 32; ++b) {
            int c = 0;
            const long long got = sao_band_sse(b, base, cnt, sum, &c);
            long long want = 0;
            for (int i = 0; i < 64 * 64; ++i) {
                const int v = (rec[i] >> 3) == b ? std::min(255, std::max(0, rec[i] + c)) : rec[i];
                want += (long long)(org[i] - v) * (org[i] - v);
            }
            bad += got != want;
            ++bands;
        }
    }
    return bad;
}

// The word-level statistics helpers of the SAO kernel: sao_rows4 against
// sao_row_of for every sample value in every byte, sao_incr4 for every
// (reconstruction, source) pair, and sao_unpack at the largest counts a
// word can hold with the most negative and positive sums.
long check_sao_words() {
    long bad = 0;
    for (uint32_t v = 0; v < 256; ++v)
        for (int k = 0; k < 4; ++k) {
            const uint32_t w = (0x5A3C81F0u & ~(0xFFu << (8 * k))) | v << (8 * k);
            const uint32_t rows = sao_rows4(w);
            for (int i = 0; i < 4; ++i) bad += (int)((rows >> (8 * i)) & 0xFF) != sao_row_of((w >> (8 * i)) & 0xFF);
        }
    for (uint32_t r = 0; r < 256; ++r)
        for (uint32_t o = 0; o < 256; ++o) {
            const uint32_t rw = r | (255 - r) << 8 | ((r * 7) & 255) << 16 | ((r + 128) & 255) << 24;
            const uint32_t ow = o | ((o * 3) & 255) << 8 | (255 - o) << 16 | ((o + 77) & 255) << 24;
            uint32_t even, odd;
            sao_incr4(rw, ow, even, odd);
            const uint32_t inc[4] = {sao_lane_lo(even), sao_lane_lo(odd), sao_lane_hi(even), sao_lane_hi(odd)};
            for (int i = 0; i < 4; ++i)
                bad += (int)inc[i] != 65536 + (int)SAO_BIAS + (int)((ow >> (8 * i)) & 0xFF) -
                                          (int)((rw >> (8 * i)) & 0xFF);
        }
    for (int n = 0; n <= 128; ++n)
        for (int d : {-255, -1, 0, 1, 255}) {
            int cnt = 0, bsum = 0;
            sao_unpack((uint32_t)n * (65536u + SAO_BIAS + d), cnt, bsum);
            bad += cnt != n || bsum - (int)SAO_BIAS * cnt != n * d;
        }
    return bad;
}

}  // namespace

int main() {
    std::mt19937 rng(5);
    long blocks = 0, ctus = 0, bands = 0;
    const long mc = check_mc(rng, blocks), db = check_deblock(rng, ctus), sao = check_sao(rng, bands);
    printf("mc blocks %ld mismatching samples %ld\n", blocks, mc);
    printf("deblock ctus %ld mismatching %ld\n", ctus, db);
    const long saow = check_sao_words();
    printf("sao bands %ld mismatching %ld\n", bands, sao);
    printf("sao word helpers mismatching %ld\n", saow);
    return (mc || db || sao || saow) ? 1 : 0;
}
