// tcb_pixel.cuh — per-sample device functions of the v2 pixel pipeline:
// six-tap / bilinear luma interpolation with the reference's exact edge
// fallbacks, 1/8-pel chroma interpolation, the 18 intra predictors, the
// chroma DC predictor and the deblocking edge filter.  Each function returns
// the one sample the reference's block routine writes at that position, so
// kernels can evaluate any subset of a block in any thread order.
#pragma once
#include "tcb_common.cuh"

namespace tcb {

// ---------------------------------------------------------------- luma MC

// Six-tap [1,-5,20,20,-5,1]/32 half-sample filters, unclipped
// (reference src/motion.c:70-107).
__device__ __forceinline__ int f6h(const uint8_t *row, int x) {
    return (row[x - 2] - 5 * row[x - 1] + 20 * row[x] + 20 * row[x + 1] -
            5 * row[x + 2] + row[x + 3] + 16) >> 5;
}
__device__ __forceinline__ int f6v(const uint8_t *ref, int s, int x, int y) {
    const uint8_t *p = ref + (size_t)y * s + x;
    return (p[-2 * s] - 5 * p[-s] + 20 * p[0] + 20 * p[s] - 5 * p[2 * s] +
            p[3 * s] + 16) >> 5;
}
__device__ __forceinline__ int f6hv(const uint8_t *ref, int s, int x, int y) {
    const uint8_t *r = ref + (size_t)y * s;
    int h0 = f6h(r - 2 * s, x), h1 = f6h(r - s, x), h2 = f6h(r, x);
    int h3 = f6h(r + s, x), h4 = f6h(r + 2 * s, x), h5 = f6h(r + 3 * s, x);
    return (h0 - 5 * h1 + 20 * h2 + 20 * h3 - 5 * h4 + h5 + 16) >> 5;
}

// Horizontal-only quarter-pel (reference src/motion.c:133-160).
__device__ __forceinline__ int luma_h(const uint8_t *ref, int s, int x, int y, int dx) {
    const uint8_t *row = ref + (size_t)y * s;
    if (dx == 0) return row[x];
    int h = f6h(row, x);
    if (dx == 2) return clampi(h, 0, 255);
    if (dx == 1) return clampi((row[x] + h + 1) / 2, 0, 255);
    return clampi((h + row[x + 1] + 1) / 2, 0, 255);
}
// Vertical-only quarter-pel (reference src/motion.c:162-188).
__device__ __forceinline__ int luma_v(const uint8_t *ref, int s, int x, int y, int dy) {
    const uint8_t *p = ref + (size_t)y * s + x;
    if (dy == 0) return p[0];
    int v = f6v(ref, s, x, y);
    if (dy == 2) return clampi(v, 0, 255);
    if (dy == 1) return clampi((p[0] + v + 1) / 2, 0, 255);
    return clampi((v + p[s] + 1) / 2, 0, 255);
}
// Nine-anchor diagonal quarter-pel, valid for all 16 phases
// (reference src/motion.c:190-260).
__device__ __forceinline__ int luma_hv(const uint8_t *ref, int s, int x, int y, int dx, int dy) {
    const uint8_t *p = ref + (size_t)y * s + x;
    int a00 = p[0], a10 = p[1], a01 = p[s], a11 = p[s + 1];
    int top, mid, bot;
    // Only the anchors this phase uses are evaluated (reads have no side
    // effects, so skipping the others cannot change the result).
    int b = 0, e = 0, c = 0, f = 0, d = 0;
    if (dx != 0) { b = f6h(p - x, x); e = f6h(p - x + s, x); }
    if (dy != 0) {
        c = f6v(ref, s, x, y);
        if (dx != 0) { f = f6v(ref, s, x + 1, y); d = f6hv(ref, s, x, y); }
    }
    switch (dx) {
        case 0:  top = a00;               mid = c;               bot = a01; break;
        case 1:  top = (a00 + b + 1) >> 1; mid = (c + d + 1) >> 1; bot = (a01 + e + 1) >> 1; break;
        case 2:  top = b;                 mid = d;               bot = e; break;
        default: top = (b + a10 + 1) >> 1; mid = (d + f + 1) >> 1; bot = (e + a11 + 1) >> 1; break;
    }
    int r;
    switch (dy) {
        case 0:  r = top; break;
        case 1:  r = (top + mid + 1) >> 1; break;
        case 2:  r = mid; break;
        default: r = (mid + bot + 1) >> 1; break;
    }
    return clampi(r, 0, 255);
}

// Bilinear quarter-pel blend (reference src/motion.c:111-116).
__device__ __forceinline__ int interp_qpel(int a, int b, int frac) {
    return clampi((a * (4 - frac) + b * frac + 2) / 4, 0, 255);
}

// Per-sample luma interpolation with edge fallbacks: six-tap where the
// whole six-tap support is inside, else bilinear, else nearest
// (reference src/motion.c:269-304 get_interp_luma).
__device__ __forceinline__ int interp_luma_safe(const uint8_t *ref, int s, int W, int H,
                                                int fx, int fy, int dx, int dy) {
    if (fx >= 2 && fx + 3 < W && fy >= 2 && fy + 3 < H) {
        if (dx == 0 && dy == 0) return ref[(size_t)fy * s + fx];
        if (dy == 0) return luma_h(ref, s, fx, fy, dx);
        if (dx == 0) return luma_v(ref, s, fx, fy, dy);
        return luma_hv(ref, s, fx, fy, dx, dy);
    }
    if (fx >= 0 && fy >= 0 && fx + 1 < W && fy + 1 < H) {
        const uint8_t *p = ref + (size_t)fy * s + fx;
        int top = interp_qpel(p[0], p[1], dx);
        int bot = interp_qpel(p[s], p[s + 1], dx);
        return interp_qpel(top, bot, dy);
    }
    int nx = clampi(fx + (dx >= 2 ? 1 : 0), 0, W - 1);
    int ny = clampi(fy + (dy >= 2 ? 1 : 0), 0, H - 1);
    return ref[(size_t)ny * s + nx];
}

// Block-level luma MC path selection (reference src/motion.c:493-584
// tc_inter_predict): decided once per block from the MV and block size.
struct LumaMC {
    const uint8_t *ref;
    int s, W, H, fx, fy, dx, dy;
    int mode;   // 0 integer in-frame copy, 1 full six-tap block, 2 per-sample safe
    __device__ __forceinline__ void init(const uint8_t *r, int stride, int w, int h,
                                         int mvx, int mvy, int blk) {
        ref = r; s = stride; W = w; H = h;
        fx = mvx >> 2; fy = mvy >> 2; dx = mvx & 3; dy = mvy & 3;
        if (dx == 0 && dy == 0 && fx >= 0 && fy >= 0 && fx + blk <= W && fy + blk <= H)
            mode = 0;
        else if ((dx | dy) != 0 && fx >= 2 && fx + blk + 2 < W && fy >= 2 && fy + blk + 2 < H)
            mode = 1;
        else
            mode = 2;
    }
    __device__ __forceinline__ int at(int x, int y) const {
        if (mode == 0) return ref[(size_t)(fy + y) * s + fx + x];
        if (mode == 1) {
            if (dy == 0) return luma_h(ref, s, fx + x, fy + y, dx);
            if (dx == 0) return luma_v(ref, s, fx + x, fy + y, dy);
            return luma_hv(ref, s, fx + x, fy + y, dx, dy);
        }
        return interp_luma_safe(ref, s, W, H, fx + x, fy + y, dx, dy);
    }
};

// 1/8-pel bilinear chroma MC with clamped coordinates
// (reference src/motion.c:597-632).  The integer in-frame copy path of the
// reference produces the same value as this formula.
__device__ __forceinline__ int chroma_mc_at(const uint8_t *ref, int s, int W, int H,
                                            int mvx, int mvy, int x, int y) {
    int xi = mvx >> 3, yi = mvy >> 3, fx = mvx & 7, fy = mvy & 7;
    int y0 = clampi(yi + y, 0, H - 1), y1 = clampi(yi + y + 1, 0, H - 1);
    int x0 = clampi(xi + x, 0, W - 1), x1 = clampi(xi + x + 1, 0, W - 1);
    const uint8_t *r0 = ref + (size_t)y0 * s, *r1 = ref + (size_t)y1 * s;
    return ((8 - fx) * (8 - fy) * r0[x0] + fx * (8 - fy) * r0[x1] +
            (8 - fx) * fy * r1[x0] + fx * fy * r1[x1] + 32) >> 6;
}

// ---------------------------------------------------------------- intra

// Angular displacement in 1/32 sample per row (modes 2..8) or column
// (modes 9..17) (reference src/predict.c:180-188 and 247-257), indexed by
// mode.  A file-scope constant table: a function-local array indexed at run
// time would be rebuilt in local memory on every call.
static __constant__ int8_t c_ang_disp[18] = {0, 0, 32, 16, 6, 0, -6, -16, -32,
                                             32, 16, 6, 0, -6, -16, -32, -48, 48};
__device__ __forceinline__ int ang_disp_vert(int mode) { return c_ang_disp[mode]; }
__device__ __forceinline__ int ang_disp_horiz(int mode) { return c_ang_disp[mode]; }

// Intra prediction sample (x, y) of an N x N block.  `ra` and `rl` point at
// index 0 of the above / left reference runs built by the v2 reference
// builder; index -1 is the corner and 2N the interpolation guard
// (reference src/predict.c:117-340, called with ra+1 / rl+1 as in
// src/encoder.c:604-605).  `dc` is the block's DC value.
__device__ __forceinline__ int intra_at(const uint8_t *ra, const uint8_t *rl, int N,
                                        int mode, int dc, int x, int y) {
    if (mode == 0) {
        // every term is non-negative and 2N a power of two: the division is a shift
        int v = (ra[x + 1] * (N - 1 - y) + rl[y + 1] * (N - 1 - x) + ra[0] * (x + y) + N) >> (__ffs(N));
        return clampi(v, 0, 255);
    }
    if (mode == 1 || mode < 0 || mode > 17) return dc;
    const int maxi_ = 2 * N;
    int disp, pos;
    const uint8_t *pri, *sec;
    if (mode < 9) { disp = ang_disp_vert(mode); pos = (x << 5) + y * disp; pri = ra; sec = rl; }
    else          { disp = ang_disp_horiz(mode); pos = (y << 5) + x * disp; pri = rl; sec = ra; }
    const uint8_t *src = pri;
    if (!(disp >= 0 || pos >= 0)) { src = sec; pos = -pos; }
    int i0 = (pos >> 5) + 1, fr = pos & 31;
    int p0 = src[clampi(i0, 0, maxi_)], p1 = src[clampi(i0 + 1, 0, maxi_)];
    return clampi(p0 + (((p1 - p0) * fr + 16) >> 5), 0, 255);
}

// ---------------------------------------------------------------- deblock

// Edge strength (reference src/filter.c:23-38): 2 / 1 for likely blocking
// artefacts, 0 for likely real edges.
__device__ __forceinline__ int edge_strength(int p0, int q0, int qp) {
    int diff = absi(p0 - q0);
    int t1 = clampi(qp / 4, 2, 16), t3 = clampi(qp, 8, 48);
    if (diff < t1) return 2;
    if (diff < t3) return 1;
    return 0;
}
// Weak filter on the sample p0 of a p1 p0 | q0 q1 edge (reference
// src/filter.c:49-57).
__device__ __forceinline__ int weak_filter(int p1, int p0, int q0, int q1, int tc) {
    int delta = (9 * (q0 - p0) - 3 * (q1 - p1) + 8) >> 4;
    delta = clampi(delta, -tc, tc);
    return clampi(p0 + delta, 0, 255);
}

}  // namespace tcb
