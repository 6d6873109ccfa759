/*
 * tcodec_types.h — value types of the TCodec public API.
 *
 * Drop-in contract: every constant, enum value and struct layout here is
 * identical to the reference's include/tcodec_types.h (lines cited per
 * block), so programs compiled against the reference header link against
 * libtcodec_b200.so unchanged.  Only declarations that the public API or
 * the bitstream needs are kept.
 */
#ifndef TCODEC_TYPES_H
#define TCODEC_TYPES_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Geometry / limits (reference tcodec_types.h:44-63). */
#define TC_CTU_SIZE         64
#define TC_BLOCK_4x4        4
#define TC_BLOCK_8x8        8
#define TC_MAX_WIDTH        4096
#define TC_MAX_HEIGHT       4096
#define TC_MIN_BLOCK        4
#define TC_INTRA_MODES      18
#define TC_REF_FRAMES       4
#define TC_MV_PREC          4
#define TC_QP_MIN           0
#define TC_QP_MAX           63
#define TC_QP_DEFAULT       32
#define TC_NUM_CONTEXTS_RC  119

/* Bitstream identification (reference tcodec_types.h:65-80). */
#define TC_MAGIC_0  0x54
#define TC_MAGIC_1  0x43
#define TC_MAGIC_2  0x56
#define TC_VERSION_V0  0
#define TC_VERSION_V1  1
#define TC_VERSION_V2  2
#define TC_VERSION     TC_VERSION_V1
#define TC_FRAME_HEADER_SIZE_V0  12
#define TC_FRAME_HEADER_SIZE_V1  14

/* Sample types (reference tcodec_types.h:84-88). */
typedef uint8_t  tc_pixel_t;
typedef int16_t  tc_coeff_t;
typedef int16_t  tc_pred_t;
typedef int32_t  tc_mv_t;
typedef int32_t  tc_sad_t;

/* Frame types (reference tcodec_types.h:92-96). */
typedef enum {
    TC_FRAME_KEY   = 0,
    TC_FRAME_INTER = 1,
    TC_FRAME_BIDIR = 2
} tc_frame_type_t;

/* Profiles (reference tcodec_types.h:100-107). */
typedef enum {
    TC_PROFILE_BASELINE_MOBILE = 0,
    TC_PROFILE_STREAMING_MAIN  = 1,
    TC_PROFILE_ARCHIVE_HIGH    = 2,
    TC_PROFILE_GRAIN_CINEMA    = 3
} tc_profile_t;
#define TC_PROFILE_MAX  3

/* Levels (reference tcodec_types.h:111-121). */
#define TC_LEVEL_AUTO   0
#define TC_LEVEL_MAX    8

typedef enum { TC_BLOCK_4x4_ID = 0, TC_BLOCK_8x8_ID = 1 } tc_block_size_t;

/* Intra modes (reference tcodec_types.h:128-146). */
typedef enum {
    TC_INTRA_PLANAR = 0,
    TC_INTRA_DC     = 1,
    TC_INTRA_ANGULAR_START       = 2,
    TC_INTRA_ANGULAR_VERT_END    = 9,
    TC_INTRA_ANGULAR_HORIZ_START = 9,
    TC_INTRA_MAX    = 18
} tc_intra_mode_t;

/* Presets (reference tcodec_types.h:148-153). */
typedef enum {
    TC_PRESET_ULTRAFAST = 0,
    TC_PRESET_FAST      = 1,
    TC_PRESET_MEDIUM    = 2,
    TC_PRESET_SLOW      = 3
} tc_preset_t;

/* Rate control (reference tcodec_types.h:155-159). */
typedef enum {
    TC_RC_CQP = 0,
    TC_RC_CBR = 1,
    TC_RC_VBR = 2
} tc_ratectrl_t;

/* Error codes (reference tcodec_types.h:156-164). */
typedef enum {
    TC_OK            =  0,
    TC_ERR_MEMORY    = -1,
    TC_ERR_PARAM     = -2,
    TC_ERR_BITSTREAM = -3,
    TC_ERR_EOF       = -4,
    TC_ERR_INTERNAL  = -5,
    TC_ERR_NEED_MORE = -6
} tc_error_t;

/* Quarter-pel motion vector (reference tcodec_types.h:168-171). */
typedef struct tc_mv { tc_mv_t x; tc_mv_t y; } tc_mv_s;

/* Frame header flag bits (reference tcodec_types.h:250-256). */
#define TC_FLAG_KEY_FRAME    0x80
#define TC_FLAG_WPP          0x40
#define TC_FLAG_RAP          0x20
#define TC_FLAG_CRC          0x10
#define TC_FLAG_EXT_HEADER   0x08

/* Tool flags, 16-bit v1 header field (reference tcodec_types.h:263-297). */
#define TC_TOOL_SKIP_MERGE        (1u << 0)
#define TC_TOOL_CFL_CHROMA        (1u << 1)
#define TC_TOOL_JND_WEIGHTING     (1u << 2)
#define TC_TOOL_MEDIAN_MV_PRED    (1u << 3)
#define TC_TOOL_MULTI_REF         (1u << 4)
#define TC_TOOL_SIX_TAP_INTERP    (1u << 5)
#define TC_TOOL_ENTROPY_CODED     (1u << 6)
#define TC_TOOL_ENTRY_POINTS      (1u << 7)
#define TC_TOOL_SAO               (1u << 8)
#define TC_TOOL_GRAIN_SYNTHESIS   (1u << 9)
#define TC_TOOL_BIPRED            (1u << 10)
#define TC_TOOL_CONTEXT_RESET     (1u << 14)
#define TC_TOOL_FRESH_SKIP        (1u << 15)
#define TC_TOOLS_IMPLEMENTED (TC_TOOL_SKIP_MERGE | TC_TOOL_CFL_CHROMA | \
    TC_TOOL_JND_WEIGHTING | TC_TOOL_MEDIAN_MV_PRED | TC_TOOL_MULTI_REF | \
    TC_TOOL_SIX_TAP_INTERP | TC_TOOL_ENTROPY_CODED | TC_TOOL_ENTRY_POINTS | \
    TC_TOOL_SAO | TC_TOOL_BIPRED | TC_TOOL_CONTEXT_RESET | TC_TOOL_FRESH_SKIP)

/* Host frame buffer (reference tcodec_types.h:309-320): same layout, so
 * callers that read encoder->recon planes keep working. */
typedef struct tc_frame_buf {
    tc_pixel_t *y;
    tc_pixel_t *cb;
    tc_pixel_t *cr;
    int32_t     stride_y;
    int32_t     stride_c;
    int32_t     width;
    int32_t     height;
    int32_t     poc;
    uint8_t     qp_avg;
    int         owned;
} tc_frame_buf_t;

/* Encoded packet (reference tcodec_types.h:324-329). */
typedef struct tc_packet {
    uint8_t *data;
    size_t   size;
    int64_t  pts;
    int      key_frame;
} tc_packet_t;

/* Encoder configuration (reference tcodec_types.h:333-355). */
typedef struct tc_config {
    int32_t       width;
    int32_t       height;
    tc_preset_t   preset;
    tc_ratectrl_t rc_method;
    int32_t       qp;
    int32_t       target_bitrate;
    int32_t       fps_num;
    int32_t       fps_den;
    int32_t       keyframe_interval;
    int32_t       threads;
    int32_t       tile_cols;
    int32_t       tile_rows;
    uint8_t       bitstream_version;
    uint8_t       profile;
    uint8_t       level_idx;
    int           enable_crc;
    int           enable_entropy_coded;
    int           enable_b_frames;
    int           use_v2;
} tc_config_t;

#ifdef __cplusplus
}
#endif

#endif /* TCODEC_TYPES_H */
