"""CPU pins of the oracle (oracle/tcoracle.c) against the reference C
library built from the reference sources, and of the reference build
against the reference's committed golden hashes.  No GPU needed."""
import ctypes
import hashlib
import struct

import numpy as np
import pytest

from tests import orabind as ob
from tests.golden import make_golden as golden

PORT = ob.port()
REF = ob.ref()
needs_ref = pytest.mark.skipif(REF is None, reason="oracle/_ref not built (no reference tree here)")

RNG = np.random.default_rng(12345)


def textured(h, w, seed):
    r = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    base = 128 + 50 * np.sin(xx / 7.0 + r.uniform(0, 6)) * np.cos(yy / 9.0 + r.uniform(0, 6))
    return np.clip(base + r.normal(0, 12, (h, w)), 0, 255).astype(np.uint8)


# ---------------------------------------------------------------- tables
@needs_ref
def test_quant_tables_match_reference():
    for qp in range(64):
        assert PORT.or_qscale(qp) == REF.tc_qscale(qp)
        assert PORT.or_lambda(qp) == REF.tc_lambda(qp)
        tab = (ctypes.c_int * 256)()
        REF.tc_build_eff_scale_table(qp, tab)
        for band in range(4):
            assert PORT.or_eff_scale(qp, band) == tab[band * 64]
    for n in (16, 64):
        for pos in range(n):
            assert PORT.or_freq_band(pos, n) == REF.tc_freq_band(pos, int(np.sqrt(n)))


def test_quant_reciprocal_is_exact():
    """The kernels divide by eff with umulhi(n, floor(2^32/eff)+1); check it
    equals C division for every quantiser step and every numerator < 2^16."""
    effs = sorted({PORT.or_eff_scale(qp, b) for qp in range(64) for b in range(4)})
    n = np.arange(1 << 16, dtype=np.uint64)
    for e in effs:
        if e <= 1:
            continue
        rcp = np.uint64((1 << 32) // e + 1)
        got = (n * rcp) >> np.uint64(32)
        assert np.array_equal(got, n // np.uint64(e)), e


def test_dct_matrix_closed_form():
    m8 = (ctypes.c_int * 64)()
    PORT.or_dct_matrix(8, m8)
    assert list(m8)[:16] == [5793] * 8 + [8035, 6811, 4551, 1598, -1598, -4551, -6811, -8035]
    m4 = (ctypes.c_int * 16)()
    PORT.or_dct_matrix(4, m4)
    assert list(m4) == [8192] * 4 + [10703, 4433, -4433, -10703, 8192, -8192, -8192, 8192,
                                      4433, -10703, 10703, -4433]


# ---------------------------------------------------------------- transforms
@needs_ref
@pytest.mark.parametrize("n", [4, 8])
def test_dct_wht_match_reference(n):
    f_ref = {4: (REF.tc_fdct4x4_res, REF.tc_idct4x4_res, REF.tc_fwht4x4, REF.tc_iwht4x4),
             8: (REF.tc_fdct8x8_res, REF.tc_idct8x8_res, REF.tc_fwht8x8, REF.tc_iwht8x8)}[n]
    for trial in range(300):
        lim = 512 if trial % 2 else 32767
        x = RNG.integers(-lim, lim, size=(n, n)).astype(np.int16)
        if trial == 0:
            x[:] = 511
        a, b = np.zeros((n, n), np.int16), np.zeros((n, n), np.int16)
        f_ref[0](ob.P(x), n, ob.P(a))
        PORT.or_fdct(n, ob.P(x), n, ob.P(b))
        assert np.array_equal(a, b)
        f_ref[1](ob.P(x), ob.P(a), n)
        PORT.or_idct(n, ob.P(x), ob.P(b), n)
        assert np.array_equal(a, b)
        small = (x // 8).astype(np.int16)
        f_ref[2](ob.P(small), n, ob.P(a))
        PORT.or_fwht(n, ob.P(small), n, ob.P(b))
        assert np.array_equal(a, b)
        f_ref[3](ob.P(small), ob.P(a), n)
        PORT.or_iwht(n, ob.P(small), ob.P(b), n)
        assert np.array_equal(a, b)


@needs_ref
def test_dc_shortcut_identity():
    """Reference test_transform_roundtrip: DC-only inverse equals the
    two-pass DC product for dc in [-2000, 2000]."""
    for n, k in ((4, 8192), (8, 5793)):
        for dc in range(-2000, 2001, 7):
            x = np.zeros((n, n), np.int16)
            x[0, 0] = dc
            out = np.zeros((n, n), np.int16)
            PORT.or_idct(n, ob.P(x), ob.P(out), n)
            v = (dc * k + 8192) >> 14
            v = (v * k + 8192) >> 14
            assert np.all(out == v)


# ---------------------------------------------------------------- motion
@needs_ref
def test_sad_and_motion_search_match_reference():
    W, H = 160, 96
    ref = textured(H, W, 1)
    cur = np.roll(ref, (3, -5), axis=(0, 1)).copy()
    cur = np.clip(cur.astype(int) + RNG.integers(-3, 4, cur.shape), 0, 255).astype(np.uint8)
    for trial in range(120):
        blk = [8, 16, 32, 64][trial % 4]
        x = int(RNG.integers(0, W - blk + 1)) // 8 * 8
        y = int(RNG.integers(0, H - blk + 1)) // 8 * 8
        cx = x + int(RNG.integers(-20, 21))
        cy = y + int(RNG.integers(-20, 21))
        sr = [16, 24, 32][trial % 3]
        org = np.ascontiguousarray(cur[y:y + blk, x:x + blk])
        s_ref = ctypes.c_int()
        mv = REF.tc_motion_est(ob.P(ref), W, W, H, ob.P(org), blk, cx, cy, blk, sr, ctypes.byref(s_ref))
        mx, my, s_port = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        PORT.or_motion_est(ob.P(ref), W, W, H, ob.P(org), blk, cx, cy, blk, sr,
                           ctypes.byref(mx), ctypes.byref(my), ctypes.byref(s_port))
        assert (mv.x, mv.y, s_ref.value) == (mx.value, my.value, s_port.value)
        assert REF.tc_sad(ob.P(org), blk, ob.P(org), blk, blk) == 0
        blk2 = np.ascontiguousarray(ref[y:y + blk, x:x + blk])
        assert REF.tc_sad(ob.P(org), blk, ob.P(blk2), blk, blk) == PORT.or_sad(ob.P(org), blk, ob.P(blk2), blk, blk)


@needs_ref
def test_luma_chroma_mc_match_reference():
    W, H = 96, 64
    ref = textured(H, W, 2)
    refc = textured(H // 2, W // 2, 3)
    for trial in range(600):
        blk = [8, 16, 32][trial % 3]
        mvx = int(RNG.integers(-16 * 4, (W + 8) * 4))
        mvy = int(RNG.integers(-16 * 4, (H + 8) * 4))
        a = np.zeros((blk, blk), np.uint8)
        b = np.zeros((blk, blk), np.uint8)
        REF.tc_inter_predict(ob.P(ref), W, W, H, ob.MV(mvx, mvy), ob.P(a), blk, blk)
        PORT.or_pred_luma(ob.P(ref), W, W, H, mvx, mvy, ob.P(b), blk, blk)
        assert np.array_equal(a, b), (mvx, mvy, blk)
        cb = blk // 2
        a, b = np.zeros((cb, cb), np.uint8), np.zeros((cb, cb), np.uint8)
        REF.tc_inter_predict_chroma(ob.P(refc), W // 2, W // 2, H // 2, ob.MV(mvx, mvy), ob.P(a), cb, cb)
        PORT.or_pred_chroma(ob.P(refc), W // 2, W // 2, H // 2, mvx, mvy, ob.P(b), cb, cb)
        assert np.array_equal(a, b)


# ---------------------------------------------------------------- intra
@needs_ref
def test_intra_refs_and_modes_match_reference():
    W, H = 128, 96
    rec = textured(H, W, 4)
    for (x, y) in [(0, 0), (64, 0), (0, 32), (40, 24), (120, 88), (64, 64)]:
        for n in (8, 16, 32, 64):
            if x + n > W or y + n > H:
                continue
            ra_r = np.zeros(2 * n + 2, np.uint8)
            rl_r = np.zeros(2 * n + 2, np.uint8)
            REF.tc_intra_get_ref_v2(ob.P(rec), W, x, y, n, W, H, ob.PO(ra_r, 1), ob.PO(rl_r, 1))
            ra_p = np.zeros(2 * n + 2, np.uint8)
            rl_p = np.zeros(2 * n + 2, np.uint8)
            PORT.or_intra_refs(ob.P(rec), W, x, y, n, W, H, ob.P(ra_p), ob.P(rl_p))
            assert np.array_equal(ra_r, ra_p) and np.array_equal(rl_r, rl_p)
            for mode in range(18):
                a = np.zeros((n, n), np.uint8)
                b = np.zeros((n, n), np.uint8)
                REF.tc_intra_predict(ob.P(a), n, ob.PO(ra_r, 1), ob.PO(rl_r, 1), n, mode)
                PORT.or_intra_pred(ob.P(b), n, ob.P(ra_p), ob.P(rl_p), n, mode)
                assert np.array_equal(a, b), (x, y, n, mode)


@needs_ref
def test_chroma_dc_and_cfl_match_reference():
    W, H = 128, 128
    for seed in range(30):
        ry = textured(H, W, 10 + seed)
        rc = textured(H // 2, W // 2, 50 + seed)
        for (lx, ly, n) in [(0, 0, 16), (64, 0, 32), (0, 64, 8), (32, 32, 64), (16, 48, 16)]:
            if lx + n > W or ly + n > H:
                continue
            cs = n // 2
            a = np.zeros((cs, cs), np.uint8)
            b = np.zeros((cs, cs), np.uint8)
            REF.tc_intra_chroma_dc(ob.P(rc), W // 2, lx // 2, ly // 2, cs, ob.P(a), cs)
            PORT.or_chroma_dc(ob.P(rc), W // 2, lx // 2, ly // 2, cs, ob.P(b), cs)
            assert np.array_equal(a, b)
            REF.tc_cfl_blend(ob.P(a), cs, ob.P(ry), W, ob.P(rc), W // 2, lx, ly, lx // 2, ly // 2, cs, cs)
            PORT.or_cfl_blend(ob.P(b), cs, ob.P(ry), W, ob.P(rc), W // 2, lx, ly, lx // 2, ly // 2, cs, cs)
            assert np.array_equal(a, b)


# ---------------------------------------------------------------- filters
@needs_ref
def test_deblock_and_sao_match_reference():
    W, H = 192, 136
    for seed in range(8):
        y = textured(H, W, 100 + seed)
        y[::8] = np.clip(y[::8].astype(int) + 9, 0, 255)
        cb = textured(H // 2, W // 2, 200 + seed)
        cr = textured(H // 2, W // 2, 300 + seed)
        org = textured(H, W, 400 + seed)
        ya, cba, cra = y.copy(), cb.copy(), cr.copy()
        yb, cbb, crb = y.copy(), cb.copy(), cr.copy()
        for (cx, cy) in [(0, 0), (64, 0), (128, 64)]:
            qp = [12, 27, 32, 42, 63][(cx + cy + seed) % 5]
            REF.tc_deblock_ctu(ob.P(ya), W, ob.P(cba), W // 2, ob.P(cra), W // 2, cx, cy, qp)
            PORT.or_deblock_ctu(ob.P(yb), W, ob.P(cbb), W // 2, ob.P(crb), W // 2, cx, cy, qp)
        assert np.array_equal(ya, yb) and np.array_equal(cba, cbb) and np.array_equal(cra, crb)
        for (cx, cy) in [(0, 0), (128, 128), (64, 64)]:
            b1, o1, b2, o2 = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
            h1 = REF.tc_sao_choose_bo(ob.P(org), W, ob.P(ya), W, cx, cy, W, H, ctypes.byref(b1), ctypes.byref(o1))
            h2 = PORT.or_sao_choose(ob.P(org), W, ob.P(yb), W, cx, cy, W, H, ctypes.byref(b2), ctypes.byref(o2))
            assert h1 == h2 and (not h1 or (b1.value, o1.value) == (b2.value, o2.value))
            if h1:
                REF.tc_sao_ctu_luma(ob.P(ya), W, cx, cy, W, H, b1, o1)
                PORT.or_sao_apply(ob.P(yb), W, cx, cy, W, H, b2, o2)
                assert np.array_equal(ya, yb)


# ---------------------------------------------------------------- golden pins
@needs_ref
def test_reference_build_reproduces_committed_golden_hashes(ref_lib):
    """The oracle library itself is pinned to the reference's committed
    conformance hashes (keyframe streams at QP 22/32/42)."""
    from tcodec_b200 import api
    entries = golden.load()
    assert len(entries) == 96
    for (digest, name, pat, w, h, qp, var) in entries[::3]:
        y, cb, cr = golden.clip(pat, w, h)
        Y = np.frombuffer(y, np.uint8).reshape(h, w)
        C = np.frombuffer(cb, np.uint8).reshape(h // 2, w // 2)
        cfg = api.make_config(ref_lib, w, h, qp=qp, preset=2, keyframe_interval=250, **golden.VARIANTS[var])
        pk = api.encode_sequence(ref_lib, cfg, [(Y, C, C)])
        blob = b"".join(struct.pack("<I", len(p)) + p for p in pk)
        assert hashlib.sha256(blob).hexdigest() == digest, name
