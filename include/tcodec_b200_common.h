/*
 * tcodec_b200_common.h — host entry points below include/tcodec.h that the
 * reference's C regression suite (test/test_tcodec.c) links against
 * directly: the bitstream writer / reader, the context-modelled binary
 * range coder and its coefficient coding, the residual DCT and WHT, and
 * the luma SAO / deblocking filters.  libtcodec_b200 exports them with the
 * reference's names, argument meanings and struct layouts (reference
 * include/tcodec_common.h), so that suite links against this library
 * unchanged.  They run on the host on host memory; the device versions of
 * the same arithmetic are the CTU engine and the tcb_* frame kernels.
 */
#ifndef TCODEC_B200_COMMON_H
#define TCODEC_B200_COMMON_H

#include <stddef.h>
#include <stdint.h>

#include "tcodec_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Bitstream writer / reader (reference include/tcodec_common.h:51-78,
 * src/bitstream.c:38-172).  Bits are written MSB first; a writer zeroes
 * each byte as it enters it.  Writes past `capacity` are dropped. */
typedef struct tc_bs_writer {
    uint8_t *buf;
    size_t   capacity;
    size_t   byte_pos;
    int      bit_pos;
} tc_bs_writer_t;

typedef struct tc_bs_reader {
    const uint8_t *buf;
    size_t         size;
    size_t         byte_pos;
    int            bit_pos;
    int            error;       /* set when a read runs past the buffer */
} tc_bs_reader_t;

void     tc_bs_writer_init(tc_bs_writer_t *w, uint8_t *buf, size_t capacity);
void     tc_bs_writer_write_bits(tc_bs_writer_t *w, uint32_t val, int nbits);
void     tc_bs_writer_write_ue(tc_bs_writer_t *w, uint32_t val);
void     tc_bs_writer_write_se(tc_bs_writer_t *w, int32_t val);
int      tc_bs_se_bits(int32_t val);
void     tc_bs_writer_byte_align(tc_bs_writer_t *w);
size_t   tc_bs_writer_bytes(tc_bs_writer_t *w);
void     tc_bs_reader_init(tc_bs_reader_t *r, const uint8_t *buf, size_t size);
uint32_t tc_bs_reader_read_bits(tc_bs_reader_t *r, int nbits);
uint32_t tc_bs_reader_read_ue(tc_bs_reader_t *r);
int32_t  tc_bs_reader_read_se(tc_bs_reader_t *r);
int      tc_bs_reader_eof(tc_bs_reader_t *r);
uint16_t tc_crc16(const uint8_t *data, size_t len);

/* Binary range coder (reference include/tcodec_common.h:317-375,
 * src/range_coder.c:77-497): one byte per context (bits 0-5 state, bit 7
 * most probable symbol), 32-bit low with cache byte / outstanding count
 * for carries, 5 flush bytes; the decoder reads 4 bytes at init. */
typedef uint8_t tc_rc_ctx_t;

typedef struct tc_rc_enc {
    tc_bs_writer_t *bs;
    uint32_t        low;
    uint32_t        range;
    int             cache_byte;   /* -1 when empty */
    int             outstanding;  /* deferred 0xFF bytes */
} tc_rc_enc_t;

typedef struct tc_rc_dec {
    tc_bs_reader_t *bs;
    uint32_t        low;
    uint32_t        range;
} tc_rc_dec_t;

void     tc_rc_enc_init(tc_rc_enc_t *rc, tc_bs_writer_t *bs);
void     tc_rc_enc_flush(tc_rc_enc_t *rc);
void     tc_rc_dec_init(tc_rc_dec_t *rc, tc_bs_reader_t *bs);
void     tc_rc_ctx_init(tc_rc_ctx_t *ctx, int num_ctx);
void     tc_rc_ctx_copy(tc_rc_ctx_t *dst, const tc_rc_ctx_t *src, int num_ctx);
void     tc_rc_enc_bit(tc_rc_enc_t *rc, tc_rc_ctx_t *ctx, int bit);
int      tc_rc_dec_bit(tc_rc_dec_t *rc, tc_rc_ctx_t *ctx);
void     tc_rc_enc_bits(tc_rc_enc_t *rc, tc_rc_ctx_t *ctx, int base_ctx, uint32_t val, int nbits);
uint32_t tc_rc_dec_bits(tc_rc_dec_t *rc, tc_rc_ctx_t *ctx, int base_ctx, int nbits);
uint32_t tc_rc_enc_ue(tc_rc_enc_t *rc, tc_rc_ctx_t *ctx, int base_ctx, uint32_t val);
uint32_t tc_rc_dec_ue(tc_rc_dec_t *rc, tc_rc_ctx_t *ctx, int base_ctx);
/* Coefficients of one TU (n = 16 or 64, raster order): last-position
 * prefix, then significance / greater-than-1 / greater-than-2 / level /
 * sign from the last nonzero back to DC; is_chroma selects the chroma
 * context bank.  dct_size is accepted for interface compatibility. */
void     tc_rc_enc_coeffs(tc_rc_enc_t *rc, tc_rc_ctx_t *ctx, const tc_coeff_t *coeffs, int n,
                          tc_block_size_t dct_size, int is_chroma);
void     tc_rc_dec_coeffs(tc_rc_dec_t *rc, tc_rc_ctx_t *ctx, tc_coeff_t *coeffs, int n,
                          tc_block_size_t dct_size, int is_chroma);

/* Residual transforms (reference include/tcodec_common.h:133-176,
 * src/transform.c:313-636).  Forward: `in` strided residual, `out` 16 / 64
 * raster coefficients; inverse: raster coefficients in, strided out. */
void tc_fdct4x4_res(const tc_coeff_t *in, int stride, tc_coeff_t *out);
void tc_idct4x4_res(const tc_coeff_t *in, tc_coeff_t *out, int stride);
void tc_fdct8x8_res(const tc_coeff_t *in, int stride, tc_coeff_t *out);
void tc_idct8x8_res(const tc_coeff_t *in, tc_coeff_t *out, int stride);

/* Every output sample of tc_idct4x4_res / tc_idct8x8_res when only the DC
 * coefficient is non-zero (reference include/tcodec_common.h:150-163, the
 * decoder's DC-only path): both rounded 14-bit passes with the DC basis
 * value round(2^14 * sqrt(1/N)), 8192 for N = 4 and 5793 for N = 8. */
static inline int tc_idct_dc4_res(int dc) {
    const int basis = 8192, half = 1 << 13;
    const int row = (dc * basis + half) >> 14;
    return (row * basis + half) >> 14;
}
static inline int tc_idct_dc8_res(int dc) {
    const int basis = 5793, half = 1 << 13;
    const int row = (dc * basis + half) >> 14;
    return (row * basis + half) >> 14;
}

void tc_fwht4x4(const tc_coeff_t *in, int stride, tc_coeff_t *out);
void tc_iwht4x4(const tc_coeff_t *in, tc_coeff_t *out, int stride);
void tc_fwht8x8(const tc_coeff_t *in, int stride, tc_coeff_t *out);
void tc_iwht8x8(const tc_coeff_t *in, tc_coeff_t *out, int stride);

/* In-loop filters on host planes (reference include/tcodec_common.h:
 * 530-549, src/filter.c:23-319). */
void tc_deblock_ctu(tc_pixel_t *y, int stride_y, tc_pixel_t *cb, int stride_cb, tc_pixel_t *cr, int stride_cr,
                    int ctu_x, int ctu_y, int qp);
void tc_sao_ctu_luma(tc_pixel_t *y, int stride_y, int x, int y0, int width, int height, int band, int offset);
int  tc_sao_choose_bo(const tc_pixel_t *orig, int orig_stride, const tc_pixel_t *recon, int recon_stride,
                      int x, int y, int width, int height, int *band, int *offset);

#ifdef __cplusplus
}
#endif

#endif /* TCODEC_B200_COMMON_H */
