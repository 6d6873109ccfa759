/*
 * tcoracle.h — CPU restatement of the TCodec v2 pixel-pipeline kernels.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the GPU kernels are
 * compared against; nothing in the product library links it.  Every
 * function restates the reference algorithm it names (file:line in the
 * reference tree) in plain C with scalar loops, and is itself pinned
 * against the reference library built by oracle/Makefile (tests/
 * test_oracle.py).  Planes are 8-bit with explicit strides; coefficient
 * blocks are int16 raster order.
 */
#ifndef TCORACLE_H
#define TCORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { int16_t dx, dy; uint8_t intra, pad; } or_mvcell_t;

/* Tables and scalar helpers (reference src/quantize.c:30-85,286-293,
 * tcodec_common.h:226-246, src/entropy.c:72-79). */
int  or_qscale(int qp);
int  or_eff_scale(int qp, int band);
int  or_lambda(int qp);
int  or_freq_band(int pos, int n);
int  or_quant(int c, int eff);
int  or_dequant(int q, int eff);
void or_dct_matrix(int n, int *m);

/* Motion (reference src/motion.c). */
int  or_sad(const uint8_t *a, int sa, const uint8_t *b, int sb, int n);
void or_motion_est(const uint8_t *ref, int rs, int w, int h, const uint8_t *org, int os,
                   int cx, int cy, int blk, int sr, int *mvx, int *mvy, int *sad);
void or_pred_luma(const uint8_t *ref, int rs, int w, int h, int mvx, int mvy,
                  uint8_t *dst, int ds, int blk);
void or_pred_chroma(const uint8_t *ref, int rs, int w, int h, int mvx, int mvy,
                    uint8_t *dst, int ds, int blk);
void or_mvp(const or_mvcell_t *grid, int cx, int cy, int *mx, int *my);

/* Intra (reference src/predict.c). ra/rl: index 0 = corner, 1 + i = ref[i]. */
void or_intra_refs(const uint8_t *rec, int s, int x, int y, int n, int w, int h,
                   uint8_t *ra, uint8_t *rl);
void or_intra_pred(uint8_t *dst, int ds, const uint8_t *ra, const uint8_t *rl, int n, int mode);
void or_chroma_dc(const uint8_t *rec, int s, int cx, int cy, int cs, uint8_t *dst, int ds);
void or_cfl_blend(uint8_t *dst, int ds, const uint8_t *ry, int sy, const uint8_t *rc, int sc,
                  int lx, int ly, int cx, int cy, int cw, int ch);

/* Transforms (reference src/transform.c:313-636). */
void or_fdct(int n, const int16_t *in, int is, int16_t *out);
void or_idct(int n, const int16_t *in, int16_t *out, int os);
void or_fwht(int n, const int16_t *in, int is, int16_t *out);
void or_iwht(int n, const int16_t *in, int16_t *out, int os);

/* Fused residual coding of one TU (reference src/encoder.c:477-543 per-TU
 * body, 333-385 rdoq/bit model).  n = 4 or 8.  Returns SSE; writes the
 * quantised levels, reconstructed samples and the bit estimate. */
long long or_code_tu(int n, const uint8_t *org, int os, const uint8_t *pred, int ps, int qp,
                     long long lambda, int16_t *levels, uint8_t *rec, int rs, int *bits);

/* In-loop filters (reference src/filter.c). */
void or_deblock_ctu(uint8_t *y, int sy, uint8_t *cb, int scb, uint8_t *cr, int scr,
                    int ctu_x, int ctu_y, int qp);
int  or_sao_choose(const uint8_t *org, int os, const uint8_t *rec, int rs, int x, int y,
                   int w, int h, int *band, int *offset);
void or_sao_apply(uint8_t *y, int s, int x, int y0, int w, int h, int band, int offset);
int  or_sao_decide(const uint8_t *org, int os, const uint8_t *rec, int rs, int x, int y,
                   int w, int h, int qp, int *band, int *offset);

/* Encoder-only global motion hint (reference src/encoder.c:171-202). */
void or_global_mv(const uint8_t *cur, const uint8_t *ref, int w, int h, int s, int *gx, int *gy);

#ifdef __cplusplus
}
#endif
#endif
