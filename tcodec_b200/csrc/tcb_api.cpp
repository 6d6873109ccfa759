// tcb_api.cpp — utility entry points of include/tcodec.h (reference
// src/tcodec.c:12-98, src/frame.c:12-89) and host frame buffers.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime.h>

#include "../../include/tcodec.h"
#include "tcb_encoder.h"

namespace tcb {
std::atomic<long long> g_alloc_countdown{-1};
}  // namespace tcb

extern "C" {

// Arms the allocation fault injector (tcb_alloc.h): the next n device or
// pinned-host allocations of the library succeed and the one after fails
// (once); n < 0 disarms it.  Returns the count that was left, negative when
// nothing was pending, so a caller can tell whether the failure happened.
long long tcb_debug_fail_allocations_after(long long n) {
    return tcb::g_alloc_countdown.exchange(n < 0 ? -1 : n);
}

// Host frame with 64-byte aligned strides (reference src/frame.c:19-43).
// Pinned frames are used for the per-frame reconstruction copy.
tc_frame_buf_t *tcb_host_frame_alloc(int width, int height, int pinned) {
    tc_frame_buf_t *f = (tc_frame_buf_t *)calloc(1, sizeof(tc_frame_buf_t));
    if (!f) return nullptr;
    f->width = width;
    f->height = height;
    f->stride_y = ((width + 63) / 64) * 64;
    f->stride_c = ((width / 2 + 63) / 64) * 64;
    f->qp_avg = TC_QP_DEFAULT;
    f->owned = pinned ? 2 : 1;
    const size_t ys = (size_t)f->stride_y * height, cs = (size_t)f->stride_c * (height / 2);
    if (pinned) {
        if (tcb::pinned_alloc(&f->y, ys ? ys : 1) != cudaSuccess || tcb::pinned_alloc(&f->cb, cs ? cs : 1) != cudaSuccess ||
            tcb::pinned_alloc(&f->cr, cs ? cs : 1) != cudaSuccess) {
            tcb_host_frame_free(f);
            return nullptr;
        }
        memset(f->y, 0, ys); memset(f->cb, 0, cs); memset(f->cr, 0, cs);
    } else {
        f->y = (tc_pixel_t *)calloc(ys ? ys : 1, 1);
        f->cb = (tc_pixel_t *)calloc(cs ? cs : 1, 1);
        f->cr = (tc_pixel_t *)calloc(cs ? cs : 1, 1);
        if (!f->y || !f->cb || !f->cr) { tcb_host_frame_free(f); return nullptr; }
    }
    return f;
}

void tcb_host_frame_free(tc_frame_buf_t *f) {
    if (!f) return;
    if (f->owned == 2) { cudaFreeHost(f->y); cudaFreeHost(f->cb); cudaFreeHost(f->cr); }
    else if (f->owned == 1) { free(f->y); free(f->cb); free(f->cr); }
    free(f);
}

const char *tc_error_string(tc_error_t err) {
    switch (err) {
        case TC_OK: return "OK";
        case TC_ERR_MEMORY: return "Out of memory";
        case TC_ERR_PARAM: return "Invalid parameter";
        case TC_ERR_BITSTREAM: return "Bitstream error";
        case TC_ERR_EOF: return "End of bitstream";
        case TC_ERR_INTERNAL: return "Internal error";
        default: return "Unknown error";
    }
}

int tc_version(void) { return TCODEC_VERSION_INT; }
const char *tc_version_string(void) { return TCODEC_VERSION_STRING; }

void tc_config_defaults(tc_config_t *cfg, int32_t width, int32_t height) {
    if (!cfg) return;
    memset(cfg, 0, sizeof(*cfg));
    cfg->width = width;
    cfg->height = height;
    cfg->preset = TC_PRESET_MEDIUM;
    cfg->rc_method = TC_RC_CQP;
    cfg->qp = TC_QP_DEFAULT;
    cfg->fps_num = 60;
    cfg->fps_den = 1;
    cfg->keyframe_interval = 30;
    cfg->bitstream_version = TC_VERSION_V1;
    cfg->profile = TC_PROFILE_BASELINE_MOBILE;
    cfg->level_idx = TC_LEVEL_AUTO;
}

double tc_psnr(const tc_pixel_t *a, int stride_a, const tc_pixel_t *b, int stride_b, int width,
               int height) {
    if (!a || !b || width <= 0 || height <= 0) return 0.0;
    int64_t sse = 0;
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) {
            const int d = (int)a[(size_t)y * stride_a + x] - (int)b[(size_t)y * stride_b + x];
            sse += d * d;
        }
    if (sse == 0) return 100.0;
    const double mse = (double)sse / ((double)width * (double)height);
    return 10.0 * log10(255.0 * 255.0 / mse);
}

// Colour conversion, BT.601 full range with 14-bit constants: the
// format's colour matrix (reference src/color.c:20-40).
namespace {
inline uint8_t clip8(int v) { return (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v)); }
constexpr int kYR = 4899, kYG = 9617, kYB = 1868;
constexpr int kBR = -2763, kBG = -5425, kBB = 8192;
constexpr int kRR = 8192, kRG = -6855, kRB = -1327;
constexpr int kIR = 22970, kIGB = -5638, kIGR = -11696, kIB = 29032;
}  // namespace

tc_error_t tc_rgb_to_ycbcr(const uint8_t *rgb, int rgb_stride, tc_pixel_t *y, int stride_y, tc_pixel_t *cb,
                           int stride_cb, tc_pixel_t *cr, int stride_cr, int width, int height) {
    if (!rgb || !y || !cb || !cr || width <= 0 || height <= 0) return TC_ERR_PARAM;
    const int cw = width / 2, ch = height / 2;
    for (int r = 0; r < height; ++r) {
        const uint8_t *p = rgb + (size_t)r * rgb_stride;
        for (int c = 0; c < width; ++c, p += 3)
            y[(size_t)r * stride_y + c] = clip8((kYR * p[0] + kYG * p[1] + kYB * p[2] + 8192) >> 14);
    }
    // chroma: each 2x2 block's four (value + 128) summed, then / 4
    for (int r = 0; r < ch; ++r)
        for (int c = 0; c < cw; ++c) {
            int sb = 0, sr = 0;
            for (int dy = 0; dy < 2; ++dy)
                for (int dx = 0; dx < 2; ++dx) {
                    const uint8_t *p = rgb + (size_t)(2 * r + dy) * rgb_stride + (size_t)(2 * c + dx) * 3;
                    sb += ((kBR * p[0] + kBG * p[1] + kBB * p[2] + 8192) >> 14) + 128;
                    sr += ((kRR * p[0] + kRG * p[1] + kRB * p[2] + 8192) >> 14) + 128;
                }
            cb[(size_t)r * stride_cb + c] = clip8(sb / 4);
            cr[(size_t)r * stride_cr + c] = clip8(sr / 4);
        }
    return TC_OK;
}

tc_error_t tc_ycbcr_to_rgb(const tc_pixel_t *y, int stride_y, const tc_pixel_t *cb, int stride_cb,
                           const tc_pixel_t *cr, int stride_cr, uint8_t *rgb, int rgb_stride, int width,
                           int height) {
    if (!y || !cb || !cr || !rgb || width <= 0 || height <= 0) return TC_ERR_PARAM;
    for (int r = 0; r < height; ++r) {
        uint8_t *p = rgb + (size_t)r * rgb_stride;
        for (int c = 0; c < width; ++c, p += 3) {
            const int Y = y[(size_t)r * stride_y + c];
            const int U = cb[(size_t)(r / 2) * stride_cb + c / 2] - 128, V = cr[(size_t)(r / 2) * stride_cr + c / 2] - 128;
            p[0] = clip8(Y + ((kIR * V + 8192) >> 14));
            p[1] = clip8(Y + ((kIGB * U + kIGR * V + 8192) >> 14));
            p[2] = clip8(Y + ((kIB * U + 8192) >> 14));
        }
    }
    return TC_OK;
}

}  // extern "C"
