/*
 * tcodec.h — public C API of the B200 TCodec implementation.
 *
 * The entry points, argument meanings and error behaviour are those of the
 * reference include/tcodec.h:27-142 (each declaration cites its line).  The
 * v2 encoder (use_v2 = 1) runs its per-frame pixel pipeline — motion search,
 * interpolation, intra prediction, transform/quant/recon, quadtree RDO,
 * deblocking and SAO — as sm_100a CUDA kernels on the current CUDA device;
 * range coding stays on the host.  There is no CPU fallback: without a
 * usable CUDA device tc_encoder_create returns NULL and encode calls return
 * TC_ERR_INTERNAL.
 *
 * Both bitstreams of the reference are implemented: v2 (use_v2 = 1,
 * bitstream_version forced to 2) and the legacy fixed 8x8 block syntax
 * (use_v2 = 0, bitstream_version 0 or 1), whose block decisions and
 * reconstruction also run on the device.  Frame sizes must be even.
 */
#ifndef TCODEC_H
#define TCODEC_H

#include "tcodec_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define TCODEC_VERSION_MAJOR  0
#define TCODEC_VERSION_MINOR  1
#define TCODEC_VERSION_PATCH  0
#define TCODEC_VERSION_INT    ((0 << 16) | (1 << 8) | 0)
#define TCODEC_VERSION_STRING "0.1.0"

typedef struct tc_encoder tc_encoder_t;
typedef struct tc_decoder tc_decoder_t;

/* reference tcodec.h:31 — NULL on invalid config or device failure. */
tc_encoder_t *tc_encoder_create(const tc_config_t *config);
/* reference tcodec.h:34 */
void tc_encoder_destroy(tc_encoder_t *enc);
/* reference tcodec.h:39-43 — packet_out->data stays valid until the next
 * encode call or destroy.  TC_ERR_NEED_MORE while a B-frame GOP fills. */
tc_error_t tc_encoder_encode(tc_encoder_t *enc,
                             const tc_pixel_t *y,  int stride_y,
                             const tc_pixel_t *cb, int stride_cb,
                             const tc_pixel_t *cr, int stride_cr,
                             tc_packet_t *packet_out);
/* reference tcodec.h:46 */
void tc_encoder_force_keyframe(tc_encoder_t *enc);
/* reference tcodec.h:49-52 */
void tc_encoder_get_stats(tc_encoder_t *enc, int64_t *total_bytes,
                          int32_t *total_frames, double *avg_psnr);
/* reference tcodec.h:57 — TC_OK while buffered packets remain, else
 * TC_ERR_EOF. */
tc_error_t tc_encoder_flush_tail(tc_encoder_t *enc, tc_packet_t *packet_out);

/* reference tcodec.h:64 */
tc_decoder_t *tc_decoder_create(int32_t width, int32_t height);
/* reference tcodec.h:67 */
void tc_decoder_destroy(tc_decoder_t *dec);
/* reference tcodec.h:72-76 */
tc_error_t tc_decoder_decode(tc_decoder_t *dec, const uint8_t *data,
                             size_t size,
                             const tc_pixel_t **y,  int *stride_y,
                             const tc_pixel_t **cb, int *stride_cb,
                             const tc_pixel_t **cr, int *stride_cr);
/* reference tcodec.h:79-80 */
void tc_decoder_get_info(tc_decoder_t *dec, int32_t *width, int32_t *height);
/* reference tcodec.h:85-88 */
tc_error_t tc_decoder_flush_tail(tc_decoder_t *dec,
                                 const tc_pixel_t **y,  int *stride_y,
                                 const tc_pixel_t **cb, int *stride_cb,
                                 const tc_pixel_t **cr, int *stride_cr);
/* reference tcodec.h:93 */
int tc_decoder_crc_valid(tc_decoder_t *dec);
/* reference tcodec.h:98 */
int tc_decoder_entropy_coded(tc_decoder_t *dec);
/* reference tcodec.h:102-108 */
void tc_decoder_set_profile(tc_decoder_t *dec, int enabled);
void tc_decoder_reset_profile(tc_decoder_t *dec);
void tc_decoder_get_profile(tc_decoder_t *dec,
                            uint64_t *parse_ns, uint64_t *coeff_ns,
                            uint64_t *transform_ns, uint64_t *motion_ns,
                            uint64_t *chroma_ns, uint64_t *deblock_ns,
                            uint64_t *copy_ns);
/* reference tcodec.h:111 */
void tc_decoder_set_threads(tc_decoder_t *dec, int nthreads);

/* reference tcodec.h:116 */
const char *tc_error_string(tc_error_t err);
/* reference tcodec.h:119-120 */
int tc_version(void);
const char *tc_version_string(void);
/* reference tcodec.h:123 */
void tc_config_defaults(tc_config_t *cfg, int32_t width, int32_t height);
/* reference tcodec.h:126-128 */
double tc_psnr(const tc_pixel_t *a, int stride_a,
               const tc_pixel_t *b, int stride_b, int width, int height);

/* Packed RGB (3 bytes per pixel) to planar YCbCr 4:2:0 and back, BT.601
 * full-range in 14-bit fixed point, chroma as the 2x2 box average
 * (reference include/tcodec.h:130-142, src/color.c).  Host memory. */
tc_error_t tc_rgb_to_ycbcr(const uint8_t *rgb, int rgb_stride,
                           tc_pixel_t *y, int stride_y, tc_pixel_t *cb, int stride_cb,
                           tc_pixel_t *cr, int stride_cr, int width, int height);
tc_error_t tc_ycbcr_to_rgb(const tc_pixel_t *y, int stride_y, const tc_pixel_t *cb, int stride_cb,
                           const tc_pixel_t *cr, int stride_cr, uint8_t *rgb, int rgb_stride,
                           int width, int height);

#ifdef __cplusplus
}
#endif

#endif /* TCODEC_H */
