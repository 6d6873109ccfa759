// legacy_emu.cpp — CPU check of the legacy (v0 / v1) 8x8 block path.
//
// Test infrastructure: compiles the device source of the legacy block path
// (tcodec_b200/csrc/tcb_legacy.cuh) as plain C++ with a team of one lane,
// drives it with a minimal P-frame sequence loop (constant QP, key frames
// at the interval, DPB of four), writes packets with the library's host
// syntax writer (tcb_entropy.cpp), and compares every packet and the final
// reconstruction with the reference encoder linked in from its own
// sources.  Each reference packet is also decoded by the library's host
// parser (tcb_parse.h) and the same device source's reconstruction
// (decode_block) and compared with the reference decoder's picture.  The
// last packet of a raw Exp-Golomb stream is decoded cut short by a quarter
// (reads past the end of a legacy frame give zero bits in both decoders);
// range-coded packets are not cut, because on its error paths the
// reference's coefficient decoder returns without writing the block's
// (uninitialised) coefficient array, so its picture is not defined.
// Usage: legacy_emu W H frames qp preset version entropy crc
// threads profile [seed [input.yuv|- [output]]]: frames come from the
// synthetic clip, or from a planar 4:2:0 file; `output` receives the
// stream as length-prefixed packets (4-byte little-endian size, then the
// packet).  Prints one line; exit code 0 when identical.
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#include <vector>

extern "C" {
#include "../include/tcodec.h"
}

#define __device__
#define __forceinline__ inline
#define __constant__
#define __noinline__
static inline int __ffs(int x) { return __builtin_ffs(x); }

namespace tcb {
namespace legacy {
static int g_d4[4][4], g_d8[8][8];
inline int ldct4(int k, int n) { return g_d4[k][n]; }
inline int ldct8(int k, int n) { return g_d8[k][n]; }
}  // namespace legacy
}  // namespace tcb

#include "../tcodec_b200/csrc/tcb_legacy.cuh"
#include "../tcodec_b200/csrc/tcb_entropy.h"
#include "../tcodec_b200/csrc/tcb_parse.h"

using namespace tcb;
using namespace tcb::legacy;

// Prefix of the reference's encoder handle: its configuration, the current
// input and the reconstruction.
struct RefEncPrefix {
    tc_config_t cfg;
    tc_frame_buf_t *cur;
    tc_frame_buf_t *recon;
};

static void init_tables() {
    const double pi = 3.14159265358979323846;
    for (int N = 4; N <= 8; N += 4)
        for (int k = 0; k < N; ++k)
            for (int m = 0; m < N; ++m) {
                const double s = k == 0 ? sqrt(1.0 / N) : sqrt(2.0 / N);
                const int v = (int)lround(16384.0 * s * cos((2 * m + 1) * k * pi / (2.0 * N)));
                if (N == 4) g_d4[k][m] = v; else g_d8[k][m] = v;
            }
}

struct Plane3 {
    std::vector<uint8_t> y, cb, cr;
};

// Synthetic clip: a textured pattern drifting by a fractional amount per
// frame, a flat region, a noisy region and a moving bright square.
static void make_frame(int W, int H, int t, unsigned seed, std::vector<uint8_t> &y, std::vector<uint8_t> &cb,
                       std::vector<uint8_t> &cr) {
    y.assign((size_t)W * H, 0);
    cb.assign((size_t)(W / 2) * (H / 2), 0);
    cr.assign((size_t)(W / 2) * (H / 2), 0);
    unsigned r = seed * 2654435761u + 12345u;
    for (int j = 0; j < H; ++j)
        for (int i = 0; i < W; ++i) {
            const double x = i + 0.75 * t, yy = j + 0.5 * t;
            double v = 128 + 60 * sin(x * 0.11 + seed) * cos(yy * 0.07) + 30 * sin((x + yy) * 0.31);
            if (i < W / 4 && j < H / 3) v = 90 + (seed % 7);
            if (i > W / 2 && j > H / 2) {
                r = r * 1103515245u + 12345u;
                v += (int)((r >> 16) % 41) - 20;
            }
            const int sx = (7 * t + (int)(seed % 13)) % (W > 16 ? W - 16 : 1), sy = (3 * t) % (H > 16 ? H - 16 : 1);
            if (i >= sx && i < sx + 16 && j >= sy && j < sy + 16) v = 230;
            y[(size_t)j * W + i] = (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v);
        }
    for (int j = 0; j < H / 2; ++j)
        for (int i = 0; i < W / 2; ++i) {
            cb[(size_t)j * (W / 2) + i] = (uint8_t)(128 + 40 * sin((i + 0.3 * t) * 0.2 + seed));
            cr[(size_t)j * (W / 2) + i] = (uint8_t)(128 + 30 * cos((j - 0.2 * t) * 0.15));
        }
}

static long long lambda_of(int qp) {
    const long long s = lg_qscale[qp < 0 ? 0 : qp > 63 ? 63 : qp];
    long long l = (s * s * 200) >> 10;
    if (l < 1) l = 1;
    if (l > (1ll << 30)) l = 1ll << 30;
    return l;
}

int main(int argc, char **argv) {
    if (argc < 11) { fprintf(stderr, "usage\n"); return 2; }
    const int W = atoi(argv[1]), H = atoi(argv[2]), nf = atoi(argv[3]), qp = atoi(argv[4]);
    const int preset = atoi(argv[5]), version = atoi(argv[6]), entropy = atoi(argv[7]), crc = atoi(argv[8]);
    const int threads = atoi(argv[9]), profile = atoi(argv[10]);
    const unsigned seed = argc > 11 ? (unsigned)atoi(argv[11]) : 1u;
    const char *in_path = argc > 12 && strcmp(argv[12], "-") != 0 ? argv[12] : nullptr;
    FILE *out_file = argc > 13 ? fopen(argv[13], "wb") : nullptr;
    FILE *in_file = in_path ? fopen(in_path, "rb") : nullptr;
    if (in_path && !in_file) { printf("cannot open %s\n", in_path); return 2; }
    init_tables();

    tc_config_t cfg;
    tc_config_defaults(&cfg, W, H);
    cfg.qp = qp;
    cfg.preset = (tc_preset_t)preset;
    cfg.bitstream_version = (uint8_t)version;
    cfg.enable_entropy_coded = entropy;
    cfg.enable_crc = crc;
    cfg.threads = threads;
    cfg.profile = (uint8_t)profile;
    cfg.use_v2 = 0;
    tc_encoder_t *ref = tc_encoder_create(&cfg);
    if (!ref) { printf("reference encoder create failed\n"); return 2; }
    tc_decoder_t *rdec = tc_decoder_create(W, H);
    if (!rdec) { printf("reference decoder create failed\n"); return 2; }

    const int sy = ((W + 63) / 64) * 64, sc = ((W / 2 + 63) / 64) * 64;
    const int cols = (W + 63) / 64, rows = (H + 63) / 64;
    const int nthr = threads <= 0 ? 4 : threads;
    const bool wpp = rows > 1 && nthr > 1 && !entropy;
    const int kint = cfg.keyframe_interval > 0 ? cfg.keyframe_interval : 30;
    // Padded planes: the reconstruction persists across frames (the
    // reference encodes in place), the DPB holds copies.
    std::vector<uint8_t> cy((size_t)sy * H + 64), ccb((size_t)sc * (H / 2) + 64), ccr(ccb.size());
    std::vector<uint8_t> ry(cy.size(), 0), rcb(ccb.size(), 0), rcr(ccb.size(), 0);
    std::vector<Plane3> dpb(4);
    int dpb_poc[4] = {-1, -1, -1, -1};
    bool dpb_ok[4] = {false, false, false, false};
    std::vector<LBlock> blocks((size_t)cols * rows * BLOCKS);
    std::vector<uint8_t> pkt((size_t)W * H * 3), scratch;
    // Decoder side: persistent picture, DPB copies with their POCs.
    std::vector<uint8_t> dy(cy.size(), 0), dcb(ccb.size(), 0), dcr(ccb.size(), 0);
    std::vector<Plane3> ddpb(4);
    int ddpb_poc[4] = {-1, -1, -1, -1};
    bool ddpb_ok[4] = {false, false, false, false};
    std::vector<LBlock> dblocks((size_t)cols * rows * BLOCKS);
    LState S;
    int mismatch = 0, pictures = 0;
    size_t total = 0;
    for (int f = 0; f < nf; ++f) {
        std::vector<uint8_t> y, cb, cr;
        if (in_file) {
            y.resize((size_t)W * H);
            cb.resize((size_t)(W / 2) * (H / 2));
            cr.resize(cb.size());
            if (fread(y.data(), 1, y.size(), in_file) != y.size() || fread(cb.data(), 1, cb.size(), in_file) != cb.size() ||
                fread(cr.data(), 1, cr.size(), in_file) != cr.size()) {
                printf("short input at frame %d\n", f);
                return 2;
            }
        } else {
            make_frame(W, H, f, seed, y, cb, cr);
        }
        tc_packet_t rp;
        memset(&rp, 0, sizeof(rp));
        if (tc_encoder_encode(ref, y.data(), W, cb.data(), W / 2, cr.data(), W / 2, &rp) != TC_OK) {
            printf("reference encode failed at frame %d\n", f);
            return 2;
        }
        for (int j = 0; j < H; ++j) memcpy(&cy[(size_t)j * sy], &y[(size_t)j * W], W);
        for (int j = 0; j < H / 2; ++j) {
            memcpy(&ccb[(size_t)j * sc], &cb[(size_t)j * (W / 2)], W / 2);
            memcpy(&ccr[(size_t)j * sc], &cr[(size_t)j * (W / 2)], W / 2);
        }
        const int is_key = f == 0 || f % kint == 0;
        const int ftype = is_key ? 0 : 1;
        if (is_key && f > 0)
            for (int i = 0; i < 4; ++i) { dpb_ok[i] = false; dpb_poc[i] = -1; }
        LFrame F;
        memset(&F, 0, sizeof(F));
        F.W = W; F.H = H; F.sy = sy; F.sc = sc; F.ctu_cols = cols; F.ctu_rows = rows;
        F.cur_y = cy.data(); F.cur_cb = ccb.data(); F.cur_cr = ccr.data();
        F.rec_y = ry.data(); F.rec_cb = rcb.data(); F.rec_cr = rcr.data();
        const int max_refs = (preset == TC_PRESET_SLOW && profile >= TC_PROFILE_STREAMING_MAIN) ? 4 : 1;
        for (int ri = 0; ri < max_refs && F.n_cand < 2; ++ri)
            if (dpb_ok[ri]) { F.cand_y[F.n_cand] = dpb[ri].y.data(); F.cand_sel[F.n_cand] = ri; F.n_cand++; }
        for (int i = 0; i < 4; ++i) F.dpb_y[i] = dpb_ok[i] ? dpb[i].y.data() : nullptr;
        F.frame_type = ftype; F.qp = qp;
        F.search_range = preset == TC_PRESET_ULTRAFAST ? 16 : preset == TC_PRESET_SLOW ? 64 : 32;
        F.lambda = lambda_of(qp);
        F.blocks = blocks.data();
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < cols; ++c) code_ctu(S, F, r, c, true);
        const LegacyFrameSyntax h = legacy_frame_syntax(cfg, is_key, ftype, qp, f, false, wpp);
        const size_t n = write_legacy_frame(pkt.data(), pkt.size(), h, blocks.data(), cols, rows, scratch);
        total += n;
        if (out_file) {
            const uint8_t len[4] = {(uint8_t)n, (uint8_t)(n >> 8), (uint8_t)(n >> 16), (uint8_t)(n >> 24)};
            fwrite(len, 1, 4, out_file);
            fwrite(pkt.data(), 1, n, out_file);
        }
        if (n != rp.size || memcmp(pkt.data(), rp.data, n) != 0) {
            size_t k = 0;
            while (k < n && k < rp.size && pkt[k] == rp.data[k]) ++k;
            printf("frame %d: packet differs (ours %zu bytes, reference %zu, first difference at byte %zu)\n", f, n,
                   rp.size, k);
            mismatch = 1;
            break;
        }
        const tc_frame_buf_t *rr = ((RefEncPrefix *)ref)->recon;
        int bad = 0;
        for (int j = 0; j < H && !bad; ++j)
            if (memcmp(&ry[(size_t)j * sy], rr->y + (size_t)j * rr->stride_y, W)) bad = 1 + j;
        for (int j = 0; j < H / 2 && !bad; ++j)
            if (memcmp(&rcb[(size_t)j * sc], rr->cb + (size_t)j * rr->stride_c, W / 2) ||
                memcmp(&rcr[(size_t)j * sc], rr->cr + (size_t)j * rr->stride_c, W / 2))
                bad = 10000 + j;
        if (bad) {
            printf("frame %d: reconstruction differs (row code %d)\n", f, bad);
            mismatch = 1;
            break;
        }
        // ---- decode the reference packet both ways
        {
            const tc_pixel_t *oy, *ocb, *ocr;
            int osy, oscb, oscr;
            const size_t dsz = f == nf - 1 && !entropy ? rp.size - rp.size / 4 : rp.size;
            const tc_error_t rerr = tc_decoder_decode(rdec, rp.data, dsz, &oy, &osy, &ocb, &oscb, &ocr, &oscr);
            tcb::parse::Reader bs;
            bs.init(rp.data, dsz);
            tcb::parse::Header hd;
            if (tcb::parse::read_header(bs, hd) != TC_OK) { printf("frame %d: header rejected\n", f); mismatch = 1; break; }
            bs.align();
            const int ent = hd.version != 0 && (hd.tools & TC_TOOL_ENTROPY_CODED);
            if (hd.frame_type == 0 && hd.frame_num > 0)
                for (int i = 0; i < 4; ++i) { ddpb_ok[i] = false; ddpb_poc[i] = -1; }
            const tc_error_t perr = tcb::parse::parse_legacy_frame(rp.data, dsz, bs, hd, ent, W, H, cols, rows, dblocks.data());
            if (rerr != TC_OK || perr != TC_OK) {
                if (rerr == TC_OK || perr == TC_OK || f != nf - 1) {
                    printf("frame %d: decode status differs (reference %d, parser %d)\n", f, (int)rerr, (int)perr);
                    mismatch = 1;
                }
                break;   // both rejected the cut-short last frame
            }
            LFrame D;
            memset(&D, 0, sizeof(D));
            D.W = W; D.H = H; D.sy = sy; D.sc = sc; D.ctu_cols = cols; D.ctu_rows = rows;
            D.rec_y = dy.data(); D.rec_cb = dcb.data(); D.rec_cr = dcr.data();
            for (int i = 0; i < 4; ++i) D.dpb_y[i] = ddpb_ok[i] ? ddpb[i].y.data() : nullptr;
            D.frame_type = hd.frame_type; D.qp = hd.qp; D.blocks = dblocks.data();
            for (int r = 0; r < rows; ++r)
                for (int c = 0; c < cols; ++c) code_ctu(S, D, r, c, false);
            int dbad = 0;
            for (int j = 0; j < H && !dbad; ++j) if (memcmp(&dy[(size_t)j * sy], oy + (size_t)j * osy, W)) dbad = 1 + j;
            for (int j = 0; j < H / 2 && !dbad; ++j)
                if (memcmp(&dcb[(size_t)j * sc], ocb + (size_t)j * oscb, W / 2) ||
                    memcmp(&dcr[(size_t)j * sc], ocr + (size_t)j * oscr, W / 2))
                    dbad = 10000 + j;
            if (dbad) { printf("frame %d: decoded picture differs (row code %d)\n", f, dbad); mismatch = 1; break; }
            ++pictures;
            for (int i = 3; i > 0; --i) { ddpb[i] = ddpb[i - 1]; ddpb_ok[i] = ddpb_ok[i - 1]; ddpb_poc[i] = ddpb_poc[i - 1]; }
            ddpb[0].y = dy; ddpb[0].cb = dcb; ddpb[0].cr = dcr;
            ddpb_ok[0] = true; ddpb_poc[0] = hd.frame_num;
        }
        for (int i = 3; i > 0; --i) { dpb[i] = dpb[i - 1]; dpb_ok[i] = dpb_ok[i - 1]; dpb_poc[i] = dpb_poc[i - 1]; }
        dpb[0].y = ry; dpb[0].cb = rcb; dpb[0].cr = rcr;
        dpb_ok[0] = true; dpb_poc[0] = f;
    }
    tc_encoder_destroy(ref);
    tc_decoder_destroy(rdec);
    if (out_file) fclose(out_file);
    if (in_file) fclose(in_file);
    if (!mismatch)
        printf("identical: %d frames, %zu bytes (encoder packets and reconstruction), %d decoded pictures\n", nf, total,
               pictures);
    return mismatch;
}
