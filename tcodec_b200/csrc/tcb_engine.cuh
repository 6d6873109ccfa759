// tcb_engine.cuh — shared-memory layout and launch constants of the CTU
// rate-distortion engine (one 512-thread CTA per 64x64 CTU).
#pragma once
#include "tcb_common.cuh"
#include "tcb_resid.cuh"

namespace tcb {

constexpr int NT = 512;             // threads per CTA (one CTU)
constexpr int CTAS_PER_SM = 1;      // CTUs resident per SM
constexpr int NW = NT / 32;         // warps per CTA
constexpr int NGROUP = 4;           // motion-search warp groups
constexpr int GT = NT / NGROUP;     // threads per motion-search group
static_assert(GT == 128, "the motion-search work split assumes 4-warp groups");

// Recon tile: luma rows -1..63 and columns -8..63 of the CTU, chroma rows
// -1..31 and columns -4..31.  Column offsets keep the interior aligned.
constexpr int RY_W = 72, RY_OX = 8, RY_OY = 1, RY_H = 65;
constexpr int RC_W = 36, RC_OX = 4, RC_OY = 1, RC_H = 33;

// Candidate slots of one leaf.
enum {
    K_ME0 = 0,      // explicit inter, MVP-centred search on the first reference
    K_ME1 = 1,      // explicit inter on the second reference (multiref)
    K_GLB = 2,      // explicit inter, global-motion centre
    K_TMP = 3,      // explicit inter, temporal centre
    K_MRG = 4,      // merge at the MVP
    K_B0 = 0,       // B: forward / backward / average / single merges (0..4;
                    // B frames use no P slot, so the two sets share buffers)
    K_INTRA = 5,    // intra modes 0..17 -> slots 5..22
    NCAND = 23
};
constexpr int NPRED = 5;
#ifndef TCB_IPRED_MAX
#define TCB_IPRED_MAX 32
#endif
constexpr int IPRED_MAX = TCB_IPRED_MAX;   // largest leaf whose intra predictions are kept            // inter prediction buffers (slots 0..4)

struct MeGroup {
    int part[2][32];    // per-warp partial sums, double-buffered (see group_int_sads)
    int mvx, mvy, best;
};

struct Smem {
    uint8_t cur_y[64 * 64];
    uint8_t cur_c[2][32 * 32];
    uint8_t rec_y[RY_H * RY_W];
    uint8_t rec_c[2][RC_H * RC_W];
    // qt_split snapshots, per depth: luma, cb, cr, grid (pre / parent).
    uint8_t snap_y0[2][64 * 64], snap_c0[2][2][32 * 32];
    uint8_t snap_y1[2][32 * 32], snap_c1[2][2][16 * 16];
    uint8_t snap_y2[2][16 * 16], snap_c2[2][2][8 * 8];
    MvCell snap_g[3][2][64];
    MvCell grid[64];
    Node nodes[QT_NODES];
    long long node_cost[QT_NODES];
    uint8_t pred[NPRED][64 * 64];
    uint8_t cpred[4][32 * 32];
    uint8_t ra[2 * 64 + 4], rl[2 * 64 + 4];     // index i+1 holds ref[i], i in -1..2N
    uint8_t ipred[18][IPRED_MAX * IPRED_MAX];    // intra predictions of the current leaf (<= IPRED_MAX)
    uint32_t ipred_ok;                           // modes held in ipred
    int scratch[NW][288];     // per warp: 4 octets x 72 or 8 quads x 20 ints (padded rows)
    MeGroup me[NGROUP];
    QuantParams qparam[2];     // luma, chroma quantiser of the current CTU
    // Luma reconstruction of every scored candidate of the current leaf
    // (leaves up to 16x16), [slot][8x8 TUs, 4x4 TUs]: the replay of the
    // winner copies it instead of coding the winner again.
    uint8_t crec[NCAND][2][16 * 16];
    int win_slot;              // candidate slot of the last scan's winner (-1: skip)
    int acc_sse[NCAND][2];
    int acc_bits[NCAND][2];
    long long acc64[4];
    int cl[NCAND];             // candidate list for job loops
    int cl2[8];                // 8x8-only candidates (merges)
    int cand_mvx[NPRED], cand_mvy[NPRED], cand_ref[NPRED], cand_ref2[NPRED];
    int ncl, dc, flag;
    uint8_t dc_u8;             // S.dc as a one-byte prediction source (PredSrc)
    long long best_cost;
    int sao[3];
    int band_sum[32], band_cnt[32], band_sq[32], band_new[32], band_cand[32];
    int ncoef;
    unsigned long long tu8mask;
};

}  // namespace tcb
