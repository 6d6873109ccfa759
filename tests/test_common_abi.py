"""The internal entry points the reference's C regression suite links
against (include/tcodec_b200_common.h) against the reference library
itself (oracle/_ref/libtcref.so, the same names built from the reference
sources): identical bytes from the bitstream writer and the range coder,
identical values read back, identical transform outputs and filtered
planes, on seeded random inputs.  CPU only."""
import ctypes

import numpy as np
import pytest

from oracle import tcref

pytestmark = pytest.mark.skipif(not tcref.available(), reason="oracle/_ref not built")

c_int, u32, i16p, u8p = ctypes.c_int, ctypes.c_uint32, ctypes.POINTER(ctypes.c_int16), ctypes.POINTER(ctypes.c_uint8)


class BsWriter(ctypes.Structure):
    _fields_ = [("buf", ctypes.c_void_p), ("capacity", ctypes.c_size_t), ("byte_pos", ctypes.c_size_t),
                ("bit_pos", c_int)]


class BsReader(ctypes.Structure):
    _fields_ = [("buf", ctypes.c_void_p), ("size", ctypes.c_size_t), ("byte_pos", ctypes.c_size_t),
                ("bit_pos", c_int), ("error", c_int)]


class RcEnc(ctypes.Structure):
    _fields_ = [("bs", ctypes.POINTER(BsWriter)), ("low", u32), ("range", u32), ("cache_byte", c_int),
                ("outstanding", c_int)]


class RcDec(ctypes.Structure):
    _fields_ = [("bs", ctypes.POINTER(BsReader)), ("low", u32), ("range", u32)]


def libs():
    from tcodec_b200 import api
    ours = api.load_library()
    ref = ctypes.CDLL(tcref.REF_LIB, mode=ctypes.RTLD_LOCAL)
    for L in (ours, ref):
        L.tc_bs_reader_read_bits.restype = u32
        L.tc_bs_reader_read_ue.restype = u32
        L.tc_bs_reader_read_se.restype = ctypes.c_int32
        L.tc_bs_writer_bytes.restype = ctypes.c_size_t
        L.tc_rc_dec_bits.restype = u32
        L.tc_rc_dec_ue.restype = u32
        L.tc_rc_enc_ue.restype = u32
        L.tc_bs_writer_write_bits.argtypes = [ctypes.POINTER(BsWriter), u32, c_int]
        L.tc_bs_writer_write_ue.argtypes = [ctypes.POINTER(BsWriter), u32]
        L.tc_bs_writer_write_se.argtypes = [ctypes.POINTER(BsWriter), ctypes.c_int32]
        L.tc_rc_enc_bits.argtypes = [ctypes.POINTER(RcEnc), u8p, c_int, u32, c_int]
        L.tc_rc_enc_ue.argtypes = [ctypes.POINTER(RcEnc), u8p, c_int, u32]
    return ours, ref


def ops_sequence(rng, n):
    ops = []
    for _ in range(n):
        k = int(rng.integers(0, 4))
        if k == 0:
            nb = int(rng.integers(1, 33))
            ops.append(("bits", int(rng.integers(0, 1 << nb, dtype=np.uint64)), nb))
        elif k == 1:
            ops.append(("ue", int(rng.integers(0, 1 << int(rng.integers(1, 20)))), 0))
        elif k == 2:
            ops.append(("se", int(rng.integers(-70000, 70001)), 0))
        else:
            ops.append(("align", 0, 0))
    return ops


def write_ops(L, ops):
    buf = (ctypes.c_uint8 * 65536)()
    w = BsWriter()
    L.tc_bs_writer_init(ctypes.byref(w), buf, len(buf))
    for op, v, nb in ops:
        if op == "bits":
            L.tc_bs_writer_write_bits(ctypes.byref(w), v, nb)
        elif op == "ue":
            L.tc_bs_writer_write_ue(ctypes.byref(w), v)
        elif op == "se":
            L.tc_bs_writer_write_se(ctypes.byref(w), v)
        else:
            L.tc_bs_writer_byte_align(ctypes.byref(w))
    n = L.tc_bs_writer_bytes(ctypes.byref(w))
    return bytes(buf[:n])


def read_ops(L, data, ops):
    buf = (ctypes.c_uint8 * len(data)).from_buffer_copy(data)
    r = BsReader()
    L.tc_bs_reader_init(ctypes.byref(r), buf, len(data))
    out = []
    for op, v, nb in ops:
        if op == "bits":
            out.append(L.tc_bs_reader_read_bits(ctypes.byref(r), nb))
        elif op == "ue":
            out.append(L.tc_bs_reader_read_ue(ctypes.byref(r)))
        elif op == "se":
            out.append(L.tc_bs_reader_read_se(ctypes.byref(r)))
        else:
            if r.bit_pos:
                r.bit_pos = 0
                r.byte_pos += 1
            out.append(None)
    return out, r.error


def test_bitstream_writer_reader_match_reference():
    ours, ref = libs()
    rng = np.random.default_rng(1)
    for _ in range(20):
        ops = ops_sequence(rng, 200)
        a, b = write_ops(ours, ops), write_ops(ref, ops)
        assert a == b
        want = [v if op in ("bits", "ue", "se") else None for op, v, nb in ops]
        got, err = read_ops(ours, a, ops)
        assert err == 0 and got == want
        assert read_ops(ref, a, ops)[0] == got
        # reading past the end sets the error flag in both
        assert read_ops(ours, a[:len(a) // 2], ops)[1] == read_ops(ref, a[:len(a) // 2], ops)[1] == 1


def sparse_coeffs(rng, n):
    c = np.zeros(n, np.int16)
    k = int(rng.integers(0, n + 1))
    if k:
        idx = rng.choice(n, size=min(n, int(rng.integers(1, 12))), replace=False)
        idx = idx[idx < k] if (idx < k).any() else idx[:1]
        mags = rng.geometric(0.35, size=len(idx)) * np.where(rng.random(len(idx)) < 0.5, -1, 1)
        mags[rng.random(len(idx)) < 0.05] *= 300
        c[idx] = np.clip(mags, -32767, 32767)
    return c


def rc_symbols(rng, n):
    syms = []
    for _ in range(n):
        k = int(rng.integers(0, 4))
        if k == 0:
            syms.append(("bit", int(rng.integers(0, 119)), int(rng.random() < 0.2)))
        elif k == 1:
            syms.append(("bits", int(rng.integers(0, 125)), (int(rng.integers(0, 32)), 5)))
        elif k == 2:
            syms.append(("ue", int(rng.integers(0, 125)), int(rng.integers(0, 5000))))
        else:
            n_ = 16 if rng.random() < 0.5 else 64
            syms.append(("coeffs", int(rng.random() < 0.3), sparse_coeffs(rng, n_)))
    return syms


def rc_encode(L, syms):
    buf = (ctypes.c_uint8 * (1 << 20))()
    w = BsWriter()
    L.tc_bs_writer_init(ctypes.byref(w), buf, len(buf))
    rc = RcEnc()
    L.tc_rc_enc_init(ctypes.byref(rc), ctypes.byref(w))
    ctx = (ctypes.c_uint8 * 119)()
    L.tc_rc_ctx_init(ctx, 119)
    for s, a, b in syms:
        if s == "bit":
            L.tc_rc_enc_bit(ctypes.byref(rc), ctypes.byref(ctx, a), b)
        elif s == "bits":
            L.tc_rc_enc_bits(ctypes.byref(rc), ctx, a, b[0], b[1])
        elif s == "ue":
            L.tc_rc_enc_ue(ctypes.byref(rc), ctx, a, b)
        else:
            cb = np.ascontiguousarray(b)
            L.tc_rc_enc_coeffs(ctypes.byref(rc), ctx, cb.ctypes.data_as(i16p), len(cb), 1 if len(cb) == 64 else 0, a)
    L.tc_rc_enc_flush(ctypes.byref(rc))
    return bytes(buf[:L.tc_bs_writer_bytes(ctypes.byref(w))]), bytes(ctx)


def rc_decode(L, data, syms):
    buf = (ctypes.c_uint8 * len(data)).from_buffer_copy(data)
    r = BsReader()
    L.tc_bs_reader_init(ctypes.byref(r), buf, len(data))
    rc = RcDec()
    L.tc_rc_dec_init(ctypes.byref(rc), ctypes.byref(r))
    ctx = (ctypes.c_uint8 * 119)()
    L.tc_rc_ctx_init(ctx, 119)
    out = []
    for s, a, b in syms:
        if s == "bit":
            out.append(L.tc_rc_dec_bit(ctypes.byref(rc), ctypes.byref(ctx, a)))
        elif s == "bits":
            out.append(L.tc_rc_dec_bits(ctypes.byref(rc), ctx, a, b[1]))
        elif s == "ue":
            out.append(L.tc_rc_dec_ue(ctypes.byref(rc), ctx, a))
        else:
            cb = np.zeros(len(b), np.int16)
            L.tc_rc_dec_coeffs(ctypes.byref(rc), ctx, cb.ctypes.data_as(i16p), len(cb), 1 if len(cb) == 64 else 0, a)
            out.append(cb.tolist())
    return out, bytes(ctx)


def test_range_coder_matches_reference():
    ours, ref = libs()
    rng = np.random.default_rng(2)
    for _ in range(8):
        syms = rc_symbols(rng, 400)
        a, ctx_a = rc_encode(ours, syms)
        b, ctx_b = rc_encode(ref, syms)
        assert a == b and ctx_a == ctx_b
        want = [b_ if s == "bit" else (b_[0] if s == "bits" else (b_ if s == "ue" else b_.tolist()))
                for s, _, b_ in syms]
        got, dctx = rc_decode(ours, a, syms)
        assert got == want
        assert rc_decode(ref, a, syms) == (got, dctx)


def test_transforms_match_reference():
    ours, ref = libs()
    rng = np.random.default_rng(3)
    for name, n, fwd in (("tc_fdct4x4_res", 4, True), ("tc_idct4x4_res", 4, False), ("tc_fdct8x8_res", 8, True),
                         ("tc_idct8x8_res", 8, False), ("tc_fwht4x4", 4, True), ("tc_iwht4x4", 4, False),
                         ("tc_fwht8x8", 8, True), ("tc_iwht8x8", 8, False)):
        for it in range(200):
            stride = n + int(rng.integers(0, 5))
            lim = 512 if fwd else 4096
            x = rng.integers(-lim, lim, size=(n, stride)).astype(np.int16)
            res = []
            for L in (ours, ref):
                if fwd:
                    out = np.zeros(n * n, np.int16)
                    getattr(L, name)(x.ctypes.data_as(i16p), stride, out.ctypes.data_as(i16p))
                else:
                    raw = np.ascontiguousarray(x[:, :n]).reshape(-1)
                    out = np.zeros((n, stride), np.int16)
                    getattr(L, name)(raw.ctypes.data_as(i16p), out.ctypes.data_as(i16p), stride)
                    out = out[:, :n]
                res.append(out)
            assert np.array_equal(res[0], res[1]), (name, it)


def test_filters_match_reference():
    ours, ref = libs()
    rng = np.random.default_rng(4)
    for it in range(6):
        w, h = 192, 128
        base = np.clip(128 + 40 * np.sin(np.arange(w)[None, :] / 9.0 + it) + rng.normal(0, 6, (h, w)), 0, 255)
        y = (np.round(base / 6) * 6).clip(0, 255).astype(np.uint8)
        cb = y[::2, ::2].copy()
        cr = (255 - y[::2, ::2]).copy()
        org = np.clip(y.astype(int) + rng.integers(-3, 6, (h, w)), 0, 255).astype(np.uint8)
        qp = int(rng.integers(10, 52))
        planes = []
        for L in (ours, ref):
            yy, bb, rr = y.copy(), cb.copy(), cr.copy()
            for ty in range(0, h, 64):
                for tx in range(0, w, 64):
                    L.tc_deblock_ctu(yy.ctypes.data_as(u8p), w, bb.ctypes.data_as(u8p), w // 2,
                                     rr.ctypes.data_as(u8p), w // 2, tx, ty, qp)
            params = []
            for ty in range(0, h, 64):
                for tx in range(0, w, 64):
                    band, off = c_int(-1), c_int(-9)
                    has = L.tc_sao_choose_bo(org.ctypes.data_as(u8p), w, yy.ctypes.data_as(u8p), w, tx, ty, w, h,
                                             ctypes.byref(band), ctypes.byref(off))
                    params.append((has, band.value, off.value) if has else (0,))
                    if has:
                        L.tc_sao_ctu_luma(yy.ctypes.data_as(u8p), w, tx, ty, w, h, band.value, off.value)
            planes.append((yy, bb, rr, params))
        for k in range(3):
            assert np.array_equal(planes[0][k], planes[1][k]), (it, k)
        assert planes[0][3] == planes[1][3], it


def test_colour_conversion_matches_reference():
    ours, ref = libs()
    rng = np.random.default_rng(5)
    for w, h in ((64, 48), (38, 22), (130, 66)):
        rgb = rng.integers(0, 256, (h, w * 3 + 5), dtype=np.uint8)
        out = []
        for L in (ours, ref):
            y = np.zeros((h, w + 3), np.uint8)
            cb = np.zeros((h // 2, w // 2 + 1), np.uint8)
            cr = np.zeros_like(cb)
            assert L.tc_rgb_to_ycbcr(rgb.ctypes.data_as(u8p), rgb.shape[1], y.ctypes.data_as(u8p), y.shape[1],
                                     cb.ctypes.data_as(u8p), cb.shape[1], cr.ctypes.data_as(u8p), cr.shape[1],
                                     w, h) == 0
            back = np.zeros((h, w * 3), np.uint8)
            assert L.tc_ycbcr_to_rgb(y.ctypes.data_as(u8p), y.shape[1], cb.ctypes.data_as(u8p), cb.shape[1],
                                     cr.ctypes.data_as(u8p), cr.shape[1], back.ctypes.data_as(u8p), back.shape[1],
                                     w, h) == 0
            out.append((y[:, :w], cb[:, :w // 2], cr[:, :w // 2], back))
        for a, b in zip(out[0], out[1]):
            assert np.array_equal(a, b), (w, h)
    assert ours.tc_rgb_to_ycbcr(None, 0, None, 0, None, 0, None, 0, 4, 4) == ref.tc_rgb_to_ycbcr(None, 0, None, 0, None, 0, None, 0, 4, 4) == -2
