// tcb_common_abi.cpp — host implementations of the entry points declared in
// include/tcodec_b200_common.h (the internal API the reference's C
// regression suite calls directly).  Same names, argument meanings and
// struct layouts as the reference; the arithmetic is the format's own
// (bit order, Exp-Golomb mapping, range-coder state machine and context
// assignment, transform matrices and rounding, filter formulas), written
// here for host memory.
#include <string.h>

#include "../../include/tcodec_b200_common.h"
#include "tcb_entropy.h"
#include "tcb_resid.cuh"

namespace {

inline int clip3(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ---------------------------------------------------------------- contexts
// Context layout of the v2 syntax (reference include/tcodec_common.h:
// 377-405 and src/range_coder.c): a context index past the table maps to
// the spare context 75, the chroma coefficient bank starts 65 above luma.
constexpr int CTX_COUNT = 119, CTX_SPARE = 75;
constexpr int C_SIG = 21, C_SIG_DC = 29, C_LAST = 30, C_GT1 = 35, C_GT1_DC = 41, C_GT2 = 42, C_GT2_DC = 44,
              C_SIGN = 45, C_SIGN_DC = 46, C_LEVEL = 47, C_LEVEL_DC = 53, C_CHROMA = 86;

inline int ctx_index(int c) { return c >= CTX_COUNT ? CTX_SPARE : c; }

// ---------------------------------------------------------------- transforms
struct DctTables {
    int m4[16], m8[64];
    DctTables() {
        tcb::dct_matrix(4, m4);
        tcb::dct_matrix(8, m8);
    }
};
const DctTables &dct() {
    static const DctTables t;
    return t;
}

// One separable pass over n points: out[k] = round(sum_j M[k][j] in[j]) with
// M = the matrix (forward) or its transpose (inverse), 14-bit constants.
inline void dct_points(const int *m, int n, const int *in, int *out, bool transpose) {
    for (int k = 0; k < n; ++k) {
        long long acc = 0;
        for (int j = 0; j < n; ++j) acc += (long long)(transpose ? m[j * n + k] : m[k * n + j]) * in[j];
        out[k] = (int)((acc + 8192) >> 14);
    }
}

// Forward: rows of the strided input, then columns; coefficient (v, h) at
// out[v * n + h].  Inverse: the transposed passes, sample (r, c) at
// out[r * stride + c].
void fdct(int n, const tc_coeff_t *in, int stride, tc_coeff_t *out) {
    const int *m = n == 4 ? dct().m4 : dct().m8;
    int rows[64], t[8], r[8];
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) t[j] = in[i * stride + j];
        dct_points(m, n, t, rows + i * n, false);
    }
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < n; ++i) t[i] = rows[i * n + j];
        dct_points(m, n, t, r, false);
        for (int i = 0; i < n; ++i) out[i * n + j] = (tc_coeff_t)r[i];
    }
}
void idct(int n, const tc_coeff_t *in, tc_coeff_t *out, int stride) {
    const int *m = n == 4 ? dct().m4 : dct().m8;
    int rows[64], t[8], r[8];
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) t[j] = in[i * n + j];
        dct_points(m, n, t, rows + i * n, true);
    }
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < n; ++i) t[i] = rows[i * n + j];
        dct_points(m, n, t, r, true);
        for (int i = 0; i < n; ++i) out[i * stride + j] = (tc_coeff_t)r[i];
    }
}

// Walsh-Hadamard butterflies in the reference's output order: 4 points
// [s+t, s-t, u+v, u-v] with s = x0+x2, t = x1+x3, u = x0-x2, v = x1-x3;
// 8 points apply that to the sums and the differences of x[i], x[i+4].
inline void had4(const int *x, int *y) {
    const int s = x[0] + x[2], t = x[1] + x[3], u = x[0] - x[2], v = x[1] - x[3];
    y[0] = s + t; y[1] = s - t; y[2] = u + v; y[3] = u - v;
}
inline void had(int n, const int *x, int *y) {
    if (n == 4) { had4(x, y); return; }
    int a[4], b[4];
    for (int i = 0; i < 4; ++i) { a[i] = x[i] + x[i + 4]; b[i] = x[i] - x[i + 4]; }
    had4(a, y);
    had4(b, y + 4);
}
// Rows, then columns with a rounded division by n.  in/out strides as the
// forward (in strided, out raster) or inverse (in raster, out strided).
void wht(int n, const tc_coeff_t *in, int is, tc_coeff_t *out, int os) {
    const int sh = n == 4 ? 2 : 3, rnd = 1 << (sh - 1);
    int rows[64], t[8], r[8];
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) t[j] = in[i * is + j];
        had(n, t, rows + i * n);
    }
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < n; ++i) t[i] = rows[i * n + j];
        had(n, t, r);
        for (int i = 0; i < n; ++i) out[i * os + j] = (tc_coeff_t)((r[i] + rnd) >> sh);
    }
}

// ---------------------------------------------------------------- range coder
void enc_put(tc_rc_enc_t *rc, uint32_t byte) { tc_bs_writer_write_bits(rc->bs, byte & 0xFF, 8); }

void enc_shift(tc_rc_enc_t *rc) {
    const uint32_t top = rc->low >> 24;
    if (top == 0xFF) {
        ++rc->outstanding;
    } else {
        if (rc->cache_byte >= 0) enc_put(rc, (uint32_t)rc->cache_byte);
        for (; rc->outstanding > 0; --rc->outstanding) enc_put(rc, 0xFF);
        rc->cache_byte = (int)top;
    }
    rc->low <<= 8;
    rc->range <<= 8;
}

// One byte for the decoder's window: a direct load when the reader is
// byte aligned, zero past the end.
uint32_t dec_byte(tc_bs_reader_t *bs) {
    if (bs->byte_pos >= bs->size) return 0;
    if (bs->bit_pos == 0) return bs->buf[bs->byte_pos++];
    return tc_bs_reader_read_bits(bs, 8);
}

// Band of coefficient i of an n-coefficient TU for the significance
// contexts: i * 8 / n.
inline int coef_band(int i, int n) { return n == 64 ? (i >> 3) : (n == 16 ? (i >> 1) : i * 8 / n); }

// ---------------------------------------------------------------- filters
inline bool edge_on(int p0, int q0, int qp) { return (p0 > q0 ? p0 - q0 : q0 - p0) < clip3(qp, 8, 48); }
inline int weak(int p1, int p0, int q0, int q1, int tc) {
    return clip3(p0 + clip3((9 * (q0 - p0) - 3 * (q1 - p1) + 8) >> 4, -tc, tc), 0, 255);
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------- bitstream
void tc_bs_writer_init(tc_bs_writer_t *w, uint8_t *buf, size_t capacity) {
    w->buf = buf;
    w->capacity = capacity;
    w->byte_pos = 0;
    w->bit_pos = 0;
    if (capacity > 0) buf[0] = 0;
}

void tc_bs_writer_write_bits(tc_bs_writer_t *w, uint32_t val, int nbits) {
    if (nbits <= 0) return;
    if (nbits > 32) nbits = 32;
    if (nbits < 32) val &= (1u << nbits) - 1;
    while (nbits > 0) {
        const int avail = 8 - w->bit_pos, n = nbits < avail ? nbits : avail;
        if (w->byte_pos < w->capacity)
            w->buf[w->byte_pos] |= (uint8_t)((val >> (nbits - n)) << (avail - n));
        w->bit_pos += n;
        nbits -= n;
        if (w->bit_pos == 8) {
            w->bit_pos = 0;
            ++w->byte_pos;
            if (w->byte_pos < w->capacity) w->buf[w->byte_pos] = 0;
        }
    }
}

void tc_bs_writer_write_ue(tc_bs_writer_t *w, uint32_t val) {
    const uint64_t code = (uint64_t)val + 1;
    int nb = 0;
    for (uint64_t t = code; t; t >>= 1) ++nb;
    tc_bs_writer_write_bits(w, 0, nb - 1);
    tc_bs_writer_write_bits(w, (uint32_t)code, nb > 32 ? 32 : nb);
}

static uint32_t se_map(int32_t v) {
    return v > 0 ? (uint32_t)(2 * (int64_t)v - 1) : (v < 0 ? (uint32_t)(-2 * (int64_t)v) : 0u);
}

void tc_bs_writer_write_se(tc_bs_writer_t *w, int32_t val) { tc_bs_writer_write_ue(w, se_map(val)); }

int tc_bs_se_bits(int32_t val) {
    uint32_t code = se_map(val) + 1;
    int nb = 0;
    for (; code; code >>= 1) ++nb;
    return 2 * nb - 1;
}

void tc_bs_writer_byte_align(tc_bs_writer_t *w) {
    if (w->bit_pos > 0) {
        w->bit_pos = 0;
        ++w->byte_pos;
        if (w->byte_pos < w->capacity) w->buf[w->byte_pos] = 0;
    }
}

size_t tc_bs_writer_bytes(tc_bs_writer_t *w) { return w->byte_pos + (w->bit_pos > 0 ? 1 : 0); }

void tc_bs_reader_init(tc_bs_reader_t *r, const uint8_t *buf, size_t size) {
    r->buf = buf;
    r->size = size;
    r->byte_pos = 0;
    r->bit_pos = 0;
    r->error = 0;
}

uint32_t tc_bs_reader_read_bits(tc_bs_reader_t *r, int nbits) {
    uint32_t v = 0;
    if (nbits > 32) nbits = 32;
    while (nbits > 0) {
        if (r->byte_pos >= r->size) { r->error = 1; return v; }
        const int avail = 8 - r->bit_pos, n = nbits < avail ? nbits : avail;
        const uint32_t bits = ((uint32_t)r->buf[r->byte_pos] >> (avail - n)) & ((1u << n) - 1);
        v = (n == 32 ? 0 : (v << n)) | bits;
        r->bit_pos += n;
        nbits -= n;
        if (r->bit_pos == 8) { r->bit_pos = 0; ++r->byte_pos; }
    }
    return v;
}

uint32_t tc_bs_reader_read_ue(tc_bs_reader_t *r) {
    int zeros = 0;
    bool one = false;
    while (r->byte_pos < r->size) {
        if (tc_bs_reader_read_bits(r, 1)) { one = true; break; }
        if (++zeros > 31) { r->error = 1; return 0; }
    }
    if (!one) { r->error = 1; return 0; }
    const uint32_t suffix = zeros ? tc_bs_reader_read_bits(r, zeros) : 0;
    return (uint32_t)((1ull << zeros) - 1) + suffix;
}

int32_t tc_bs_reader_read_se(tc_bs_reader_t *r) {
    const uint32_t m = tc_bs_reader_read_ue(r);
    if (m == 0) return 0;
    return (m & 1) ? (int32_t)((m + 1) / 2) : -(int32_t)(m / 2);
}

int tc_bs_reader_eof(tc_bs_reader_t *r) { return r->byte_pos >= r->size; }

uint16_t tc_crc16(const uint8_t *data, size_t len) { return tcb::crc16_ccitt(data, len); }

// ---------------------------------------------------------------- range coder
void tc_rc_enc_init(tc_rc_enc_t *rc, tc_bs_writer_t *bs) {
    rc->bs = bs;
    rc->low = 0;
    rc->range = 0xFFFFFFFFu;
    rc->cache_byte = -1;
    rc->outstanding = 0;
}

void tc_rc_enc_bit(tc_rc_enc_t *rc, tc_rc_ctx_t *ctx, int bit) {
    const int state = *ctx & 0x3F, mps = (*ctx >> 7) & 1;
    const uint32_t rlps = (rc->range >> 8) * tcb::kLpsProb[state];
    if (bit == mps) {
        rc->range -= rlps;
        if (state < 63) *ctx = (tc_rc_ctx_t)((mps << 7) | (state + 1));
    } else {
        const uint32_t before = rc->low;
        rc->low += rc->range - rlps;
        rc->range = rlps;
        *ctx = (tc_rc_ctx_t)(((state == 0 ? (mps ^ 1) : mps) << 7) | tcb::kNextLps[state]);
        if (rc->low < before) {   // the addition carried into the pending bytes
            if (rc->cache_byte >= 0) {
                enc_put(rc, (uint32_t)rc->cache_byte + 1);
                for (; rc->outstanding > 0; --rc->outstanding) enc_put(rc, 0x00);
            }
            rc->cache_byte = -1;
            rc->outstanding = 0;
        }
    }
    while (rc->range < (1u << 24)) enc_shift(rc);
}

void tc_rc_enc_flush(tc_rc_enc_t *rc) {
    if (rc->cache_byte >= 0) enc_put(rc, (uint32_t)rc->cache_byte);
    for (; rc->outstanding > 0; --rc->outstanding) enc_put(rc, 0xFF);
    rc->cache_byte = -1;
    for (int i = 0; i < 5; ++i) {
        enc_put(rc, rc->low >> 24);
        rc->low <<= 8;
    }
}

void tc_rc_dec_init(tc_rc_dec_t *rc, tc_bs_reader_t *bs) {
    rc->bs = bs;
    rc->low = 0;
    rc->range = 0xFFFFFFFFu;
    for (int i = 0; i < 4; ++i) rc->low = (rc->low << 8) | dec_byte(bs);
}

int tc_rc_dec_bit(tc_rc_dec_t *rc, tc_rc_ctx_t *ctx) {
    const int state = *ctx & 0x3F, mps = (*ctx >> 7) & 1;
    const uint32_t rlps = (rc->range >> 8) * tcb::kLpsProb[state];
    int bit;
    if (rc->low < rc->range - rlps) {
        rc->range -= rlps;
        bit = mps;
        if (state < 63) *ctx = (tc_rc_ctx_t)((mps << 7) | (state + 1));
    } else {
        rc->low -= rc->range - rlps;
        rc->range = rlps;
        bit = mps ^ 1;
        *ctx = (tc_rc_ctx_t)(((state == 0 ? (mps ^ 1) : mps) << 7) | tcb::kNextLps[state]);
    }
    while (rc->range < (1u << 24)) {
        rc->low <<= 8;
        rc->range = rc->range == 0 ? 0xFFu : (rc->range << 8);
        rc->low |= dec_byte(rc->bs);
    }
    return bit;
}

void tc_rc_ctx_init(tc_rc_ctx_t *ctx, int num_ctx) {
    if (num_ctx > 0) memset(ctx, 0, (size_t)num_ctx);
}

void tc_rc_ctx_copy(tc_rc_ctx_t *dst, const tc_rc_ctx_t *src, int num_ctx) {
    if (num_ctx > 0) memcpy(dst, src, (size_t)num_ctx);
}

void tc_rc_enc_bits(tc_rc_enc_t *rc, tc_rc_ctx_t *ctx, int base, uint32_t val, int nbits) {
    for (int i = 0; i < nbits; ++i) tc_rc_enc_bit(rc, &ctx[ctx_index(base + i)], (int)((val >> (nbits - 1 - i)) & 1));
}

uint32_t tc_rc_dec_bits(tc_rc_dec_t *rc, tc_rc_ctx_t *ctx, int base, int nbits) {
    uint32_t v = 0;
    for (int i = 0; i < nbits; ++i) v = (v << 1) | (uint32_t)tc_rc_dec_bit(rc, &ctx[ctx_index(base + i)]);
    return v;
}

// Context-coded Exp-Golomb: prefix zeros on contexts base.., the marker 1
// on base + zeros, suffix bits on the contexts after it.  Returns the
// number of coded bits.
uint32_t tc_rc_enc_ue(tc_rc_enc_t *rc, tc_rc_ctx_t *ctx, int base, uint32_t val) {
    const uint64_t code = (uint64_t)val + 1;
    int nb = 0;
    for (uint64_t t = code; t; t >>= 1) ++nb;
    const int z = nb - 1;
    for (int i = 0; i < z; ++i) tc_rc_enc_bit(rc, &ctx[ctx_index(base + i)], 0);
    tc_rc_enc_bit(rc, &ctx[ctx_index(base + z)], 1);
    for (int i = 0; i < z; ++i)
        tc_rc_enc_bit(rc, &ctx[ctx_index(base + z + 1 + i)], (int)((code >> (z - 1 - i)) & 1));
    return (uint32_t)(2 * z + 1);
}

uint32_t tc_rc_dec_ue(tc_rc_dec_t *rc, tc_rc_ctx_t *ctx, int base) {
    int z = 0;
    while (!tc_rc_dec_bit(rc, &ctx[ctx_index(base + z)]))
        if (++z > 31) return 0;
    uint32_t suffix = 0;
    for (int i = 0; i < z; ++i) suffix = (suffix << 1) | (uint32_t)tc_rc_dec_bit(rc, &ctx[ctx_index(base + z + 1 + i)]);
    return (uint32_t)((1ull << z) - 1) + suffix;
}

void tc_rc_enc_coeffs(tc_rc_enc_t *rc, tc_rc_ctx_t *ctx, const tc_coeff_t *c, int n, tc_block_size_t dct_size,
                      int is_chroma) {
    (void)dct_size;
    const int o = is_chroma ? C_CHROMA - C_SIG : 0;
    int last = -1;
    for (int i = n - 1; i >= 0; --i)
        if (c[i]) { last = i; break; }
    tc_rc_enc_bit(rc, &ctx[C_LAST + o], last >= 0);
    if (last < 0) return;
    // last position: unary up to 4 (contexts LAST..LAST+3), else escape + EG
    const int pre = last < 4 ? last : 4;
    for (int i = 0; i < pre; ++i) tc_rc_enc_bit(rc, &ctx[C_LAST + o + (i & 3)], 0);
    if (last < 4) tc_rc_enc_bit(rc, &ctx[C_LAST + o + (pre & 3)], 1);
    else tc_rc_enc_ue(rc, ctx, C_LAST + o, (uint32_t)(last - 4));
    int g1 = 0;
    for (int i = last; i >= 0; --i) {
        const bool dc = i == 0;
        int sig = dc ? C_SIG_DC + o : C_SIG + o + coef_band(i, n);
        if (sig >= CTX_COUNT) sig = CTX_COUNT - 1;
        if (!c[i]) { tc_rc_enc_bit(rc, &ctx[sig], 0); continue; }
        tc_rc_enc_bit(rc, &ctx[sig], 1);
        const int mag = c[i] < 0 ? -c[i] : c[i];
        tc_rc_enc_bit(rc, &ctx[dc ? C_GT1_DC + o : C_GT1 + o + (g1 < 5 ? g1 : 5)], mag > 1);
        if (mag > 1) {
            tc_rc_enc_bit(rc, &ctx[dc ? C_GT2_DC + o : C_GT2 + o + (g1 < 1 ? g1 : 1)], mag > 2);
            if (mag > 2) tc_rc_enc_ue(rc, ctx, dc ? C_LEVEL_DC + o : C_LEVEL + o, (uint32_t)(mag - 3));
            if (++g1 > 5) g1 = 5;
        }
        tc_rc_enc_bit(rc, &ctx[dc ? C_SIGN_DC + o : C_SIGN + o], c[i] < 0);
    }
}

void tc_rc_dec_coeffs(tc_rc_dec_t *rc, tc_rc_ctx_t *ctx, tc_coeff_t *c, int n, tc_block_size_t dct_size,
                      int is_chroma) {
    (void)dct_size;
    const int o = is_chroma ? C_CHROMA - C_SIG : 0;
    if (!tc_rc_dec_bit(rc, &ctx[C_LAST + o])) {
        memset(c, 0, sizeof(tc_coeff_t) * (size_t)n);
        return;
    }
    int last = -1;
    for (int i = 0; i < 4 && last < 0; ++i)
        if (tc_rc_dec_bit(rc, &ctx[C_LAST + o + i])) last = i;
    if (last < 0) {
        const uint32_t extra = tc_rc_dec_ue(rc, ctx, C_LAST + o);
        if (extra > (uint32_t)n) { rc->bs->error = 1; return; }
        last = 4 + (int)extra;
    }
    if (last >= n) { rc->bs->error = 1; return; }
    if (last + 1 < n) memset(c + last + 1, 0, sizeof(tc_coeff_t) * (size_t)(n - last - 1));
    int g1 = 0;
    for (int i = last; i >= 0; --i) {
        const bool dc = i == 0;
        int sig = dc ? C_SIG_DC + o : C_SIG + o + coef_band(i, n);
        if (sig >= CTX_COUNT) sig = CTX_COUNT - 1;
        if (!tc_rc_dec_bit(rc, &ctx[sig])) { c[i] = 0; continue; }
        int mag = 1;
        if (tc_rc_dec_bit(rc, &ctx[dc ? C_GT1_DC + o : C_GT1 + o + (g1 < 5 ? g1 : 5)])) {
            mag = 2;
            if (tc_rc_dec_bit(rc, &ctx[dc ? C_GT2_DC + o : C_GT2 + o + (g1 < 1 ? g1 : 1)]))
                mag = 3 + (int)tc_rc_dec_ue(rc, ctx, dc ? C_LEVEL_DC + o : C_LEVEL + o);
            if (++g1 > 5) g1 = 5;
        }
        if (mag > 32767) { rc->bs->error = 1; return; }
        c[i] = (tc_coeff_t)(tc_rc_dec_bit(rc, &ctx[dc ? C_SIGN_DC + o : C_SIGN + o]) ? -mag : mag);
    }
}

// ---------------------------------------------------------------- transforms
void tc_fdct4x4_res(const tc_coeff_t *in, int stride, tc_coeff_t *out) { fdct(4, in, stride, out); }
void tc_idct4x4_res(const tc_coeff_t *in, tc_coeff_t *out, int stride) { idct(4, in, out, stride); }
void tc_fdct8x8_res(const tc_coeff_t *in, int stride, tc_coeff_t *out) { fdct(8, in, stride, out); }
void tc_idct8x8_res(const tc_coeff_t *in, tc_coeff_t *out, int stride) { idct(8, in, out, stride); }
void tc_fwht4x4(const tc_coeff_t *in, int stride, tc_coeff_t *out) { wht(4, in, stride, out, 4); }
void tc_iwht4x4(const tc_coeff_t *in, tc_coeff_t *out, int stride) { wht(4, in, 4, out, stride); }
void tc_fwht8x8(const tc_coeff_t *in, int stride, tc_coeff_t *out) { wht(8, in, stride, out, 8); }
void tc_iwht8x8(const tc_coeff_t *in, tc_coeff_t *out, int stride) { wht(8, in, 8, out, stride); }

// ---------------------------------------------------------------- filters
void tc_deblock_ctu(tc_pixel_t *Y, int sy, tc_pixel_t *cb, int scb, tc_pixel_t *cr, int scr, int x0, int y0,
                    int qp) {
    const int tc = clip3(qp / 3, 1, 10), cq = clip3(qp - 1, 0, 63), ctc = clip3(cq / 4, 1, 6);
    // luma: vertical edges x = 4..60, then horizontal edges y = 4..60
    for (int e = 4; e < 64; e += 4)
        for (int r = 0; r < 64; ++r) {
            tc_pixel_t *p = Y + (size_t)(y0 + r) * sy + x0 + e;
            const int p1 = p[-2], p0 = p[-1], q0 = p[0], q1 = p[1];
            if (edge_on(p0, q0, qp)) { p[-1] = (tc_pixel_t)weak(p1, p0, q0, q1, tc); p[0] = (tc_pixel_t)weak(q1, q0, p0, p1, tc); }
        }
    for (int e = 4; e < 64; e += 4)
        for (int c = 0; c < 64; ++c) {
            tc_pixel_t *p = Y + (size_t)(y0 + e) * sy + x0 + c;
            const int p1 = p[-2 * sy], p0 = p[-sy], q0 = p[0], q1 = p[sy];
            if (edge_on(p0, q0, qp)) { p[-sy] = (tc_pixel_t)weak(p1, p0, q0, q1, tc); p[0] = (tc_pixel_t)weak(q1, q0, p0, p1, tc); }
        }
    // chroma: Cb vertical edges x = 4..28; horizontal edges filter rows
    // (4e, 4e+1) of both planes with the Cr edge deciding
    for (int e = 4; e < 32; e += 4)
        for (int r = 0; r < 32; ++r) {
            tc_pixel_t *p = cb + (size_t)(y0 / 2 + r) * scb + x0 / 2 + e;
            const int p0 = p[-1], q0 = p[0];
            if (edge_on(p0, q0, cq)) {
                const int d = clip3((q0 - p0 + 1) >> 1, -ctc, ctc);
                p[-1] = (tc_pixel_t)clip3(p0 + d, 0, 255);
                p[0] = (tc_pixel_t)clip3(q0 - d, 0, 255);
            }
        }
    for (int e = 4; e < 32; e += 4)
        for (int c = 0; c < 32; ++c) {
            tc_pixel_t *pr = cr + (size_t)(y0 / 2 + e) * scr + x0 / 2 + c;
            tc_pixel_t *pb = cb + (size_t)(y0 / 2 + e) * scb + x0 / 2 + c;
            const int p0 = pr[0], q0 = pr[scr], b0 = pb[0], b1 = pb[scb];
            if (edge_on(p0, q0, cq)) {
                int d = clip3((q0 - p0 + 1) >> 1, -ctc, ctc);
                pr[0] = (tc_pixel_t)clip3(p0 + d, 0, 255);
                pr[scr] = (tc_pixel_t)clip3(q0 - d, 0, 255);
                d = clip3((b1 - b0 + 1) >> 1, -ctc, ctc);
                pb[0] = (tc_pixel_t)clip3(b0 + d, 0, 255);
                pb[scb] = (tc_pixel_t)clip3(b1 - d, 0, 255);
            }
        }
}

void tc_sao_ctu_luma(tc_pixel_t *Y, int s, int x, int y0, int width, int height, int band, int offset) {
    band = clip3(band, 0, 31);
    offset = clip3(offset, -7, 7);
    const int x1 = x + 64 < width ? x + 64 : width, y1 = y0 + 64 < height ? y0 + 64 : height;
    for (int r = y0; r < y1; ++r)
        for (int c = x; c < x1; ++c) {
            tc_pixel_t *p = Y + (size_t)r * s + c;
            if ((*p >> 3) == band) *p = (tc_pixel_t)clip3(*p + offset, 0, 255);
        }
}

// Exact band-offset choice from per-value statistics: for every
// reconstructed value v, its count and the sum and sum of squares of the
// co-located originals give the SSE of any substitution v -> v' in closed
// form, so each band's candidate is scored without another pass.
int tc_sao_choose_bo(const tc_pixel_t *org, int os, const tc_pixel_t *rec, int rs, int x, int y, int width,
                     int height, int *band, int *offset) {
    long long n[256] = {0}, so[256] = {0}, sq[256] = {0};
    const int x1 = x + 64 < width ? x + 64 : width, y1 = y + 64 < height ? y + 64 : height;
    for (int r = y; r < y1; ++r)
        for (int c = x; c < x1; ++c) {
            const int v = rec[(size_t)r * rs + c], o = org[(size_t)r * os + c];
            ++n[v]; so[v] += o; sq[v] += (long long)o * o;
        }
    auto sse_as = [&](int v, int w) { return sq[v] - 2LL * w * so[v] + (long long)w * w * n[v]; };
    long long base = 0;
    for (int v = 0; v < 256; ++v) base += sse_as(v, v);
    long long best = base;
    int bb = 0, bo = 0;
    for (int b = 0; b < 32; ++b) {
        long long cnt = 0, sum = 0;
        for (int v = 8 * b; v < 8 * b + 8; ++v) { cnt += n[v]; sum += so[v] - (long long)v * n[v]; }
        if (!cnt) continue;
        const int cand = clip3((int)((sum + (sum >= 0 ? cnt / 2 : -(cnt / 2))) / cnt), -7, 7);
        if (!cand) continue;
        long long sse = base;
        for (int v = 8 * b; v < 8 * b + 8; ++v) sse += sse_as(v, clip3(v + cand, 0, 255)) - sse_as(v, v);
        if (sse < best) { best = sse; bb = b; bo = cand; }
    }
    if (best >= base) return 0;
    *band = bb;
    *offset = bo;
    return 1;
}

}  // extern "C"
