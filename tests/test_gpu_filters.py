"""Standalone in-loop filter kernels (tcb_deblock_frames, tcb_sao_frames)
against the oracle restatement, bit-exact: several frames per launch,
frame sizes with partial CTUs, aligned (16-byte vector) and unaligned
(byte path) strides, QPs across the range."""
import ctypes

import numpy as np
import pytest

from tcodec_b200.api import FilterFrame
from tests import orabind

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from tcodec_b200 import api
    return api.bind_b200(api.load_library())


def blocky(rng, h, w, step):
    """Smooth content quantised in step x step blocks plus mild noise: block
    edges with small steps, the case deblocking filters."""
    hp, wp = -(-h // step) * step, -(-w // step) * step
    yy, xx = np.mgrid[0:hp, 0:wp]
    base = 128 + 60 * np.sin(xx / 23.0 + rng.uniform(0, 6)) * np.cos(yy / 17.0 + rng.uniform(0, 6))
    q = base.reshape(hp // step, step, wp // step, step).mean(axis=(1, 3))
    q = np.repeat(np.repeat(q, step, 0), step, 1)[:h, :w]
    return np.clip(q + rng.normal(0, 1.5, (h, w)), 0, 255).astype(np.uint8)


def make_case(rng, w, h, qp, pad):
    y = blocky(rng, h, w, 4)
    cb = blocky(rng, h // 2, w // 2, 4)
    cr = blocky(rng, h // 2, w // 2, 4)
    # source = recon + a bias (different per half of the frame) + noise, so
    # that band offsets pay off in many CTUs and not in others
    bias = np.where(np.arange(w)[None, :] < w // 2, 5, 0)
    src = np.clip(y.astype(int) + bias + rng.integers(-2, 3, (h, w)), 0, 255).astype(np.uint8)
    return dict(w=w, h=h, qp=qp, pad=pad, y=y, cb=cb, cr=cr, src=src)


CASES = [(1920, 1080, 32, 0), (200, 136, 22, 0), (256, 192, 42, 3), (130, 70, 51, 0), (320, 240, 12, 5)]


def to_dev(a, pad):
    import torch
    h, w = a.shape
    buf = np.zeros((h, w + pad), np.uint8)
    buf[:, :w] = a
    return torch.from_numpy(buf).cuda()


def run(lib, fn, cases, kernel=None, threads=0):
    """One call of fn over the cases; with threads != 0 the call runs the
    CTA-size variant `threads` (recorded for the first frame's size, the
    size a launch is tuned by, and removed afterwards)."""
    if threads:
        assert lib.tcb_autotune_set_threads(kernel, cases[0]["w"], cases[0]["h"], threads) == 0
    try:
        return _run(lib, fn, cases)
    finally:
        if threads:
            lib.tcb_autotune_set_threads(kernel, cases[0]["w"], cases[0]["h"], 0)


def _run(lib, fn, cases):
    import torch
    frames = (FilterFrame * len(cases))()
    keep = []
    for f, c in zip(frames, cases):
        ty, tcb, tcr, ts = (to_dev(c[k], c["pad"]) for k in ("y", "cb", "cr", "src"))
        nctu = ((c["w"] + 63) // 64) * ((c["h"] + 63) // 64)
        tp = torch.full((nctu * 3,), -1, dtype=torch.int16, device="cuda")
        keep.append((ty, tcb, tcr, ts, tp))
        f.width, f.height, f.qp = c["w"], c["h"], c["qp"]
        f.stride_y, f.stride_c, f.stride_src = ty.shape[1], tcb.shape[1], ts.shape[1]
        f.y, f.cb, f.cr, f.src_y, f.sao_params = ty.data_ptr(), tcb.data_ptr(), tcr.data_ptr(), ts.data_ptr(), tp.data_ptr()
    torch.cuda.synchronize()
    assert fn(frames, len(cases), torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    out = []
    for c, (ty, tcb, tcr, ts, tp) in zip(cases, keep):
        w, h = c["w"], c["h"]
        out.append(dict(y=ty.cpu().numpy()[:, :w], cb=tcb.cpu().numpy()[:, :w // 2], cr=tcr.cpu().numpy()[:, :w // 2],
                        params=tp.cpu().numpy().reshape(-1, 3)))
    return out


def oracle_deblock(c):
    L = orabind.port()
    y, cb, cr = c["y"].copy(), c["cb"].copy(), c["cr"].copy()
    for r in range(c["h"] // 64):
        for col in range(c["w"] // 64):
            L.or_deblock_ctu(orabind.P(y), c["w"], orabind.P(cb), c["w"] // 2, orabind.P(cr), c["w"] // 2,
                             col * 64, r * 64, c["qp"])
    return y, cb, cr


def oracle_sao(c):
    L = orabind.port()
    y = c["y"].copy()
    params = []
    for r in range(0, c["h"], 64):
        for col in range(0, c["w"], 64):
            b, o = ctypes.c_int(), ctypes.c_int()
            has = L.or_sao_decide(orabind.P(c["src"]), c["w"], orabind.P(y), c["w"], col, r, c["w"], c["h"],
                                  c["qp"], ctypes.byref(b), ctypes.byref(o))
            if has:
                L.or_sao_apply(orabind.P(y), c["w"], col, r, c["w"], c["h"], b.value, o.value)
            params.append((has, b.value, o.value))
    return y, np.array(params, np.int16)


@pytest.mark.parametrize("threads", [0, 64, 128, 256])
def test_deblock_frames_match_oracle(lib, threads):
    from tcodec_b200 import api
    rng = np.random.default_rng(5)
    cases = [make_case(rng, *c) for c in CASES]
    got = run(lib, lib.tcb_deblock_frames, cases, api.KERNEL_DEBLOCK, threads)
    for c, g in zip(cases, got):
        y, cb, cr = oracle_deblock(c)
        assert np.array_equal(g["y"], y), (c["w"], c["h"], c["qp"])
        assert np.array_equal(g["cb"], cb) and np.array_equal(g["cr"], cr), (c["w"], c["h"], c["qp"])


@pytest.mark.parametrize("threads", [0, 64, 128])
def test_sao_frames_match_oracle(lib, threads):
    from tcodec_b200 import api
    rng = np.random.default_rng(6)
    cases = [make_case(rng, *c) for c in CASES]
    # extreme values so bands 0 and 31 (where the offset clips) occur
    cases[1]["y"][:40, :40] = rng.integers(0, 6, (40, 40))
    cases[1]["src"][:40, :40] = 0
    cases[4]["y"][64:100, 64:128] = rng.integers(249, 256, (36, 64))
    cases[4]["src"][64:100, 64:128] = 255
    got = run(lib, lib.tcb_sao_frames, cases, api.KERNEL_SAO, threads)
    n_sao = 0
    for c, g in zip(cases, got):
        y, params = oracle_sao(c)
        assert np.array_equal(g["params"], params), (c["w"], c["h"], c["qp"])
        assert np.array_equal(g["y"], y), (c["w"], c["h"], c["qp"])
        n_sao += int(params[:, 0].sum())
    assert n_sao > 0   # the cases exercise the apply path


def test_filters_random_content(lib):
    """Uniformly random samples (the standalone bench's content): every CTU
    has samples in bands 0 and 31 and edges of every strength."""
    rng = np.random.default_rng(8)
    cases = []
    for w, h, qp, pad in ((256, 128, 30, 0), (136, 100, 45, 4)):
        c = dict(w=w, h=h, qp=qp, pad=pad)
        for k, (hh, ww) in (("y", (h, w)), ("cb", (h // 2, w // 2)), ("cr", (h // 2, w // 2)), ("src", (h, w))):
            c[k] = rng.integers(0, 256, (hh, ww)).astype(np.uint8)
        cases.append(c)
    got = run(lib, lib.tcb_deblock_frames, cases)
    for c, g in zip(cases, got):
        y, cb, cr = oracle_deblock(c)
        assert np.array_equal(g["y"], y) and np.array_equal(g["cb"], cb) and np.array_equal(g["cr"], cr)
    got = run(lib, lib.tcb_sao_frames, cases)
    for c, g in zip(cases, got):
        y, params = oracle_sao(c)
        assert np.array_equal(g["params"], params) and np.array_equal(g["y"], y)


def test_autotuner_picks_a_variant_per_kernel(lib):
    from tcodec_b200 import api
    w, h = 320, 192
    assert lib.tcb_autotune_frame_kernels(w, h, 2) == 0
    assert lib.tcb_autotune_threads(api.KERNEL_DEBLOCK, w, h) in (64, 128, 256)
    assert lib.tcb_autotune_threads(api.KERNEL_SAO, w, h) in (64, 128)
    assert lib.tcb_autotune_threads(api.KERNEL_MC, w, h) in (64, 128, 256)
    assert lib.tcb_autotune_threads(api.KERNEL_MC, w + 2, h) == 0        # other sizes untouched
    assert lib.tcb_autotune_set_threads(api.KERNEL_SAO, w, h, 256) != 0  # not a SAO variant
    for k in (api.KERNEL_DEBLOCK, api.KERNEL_SAO, api.KERNEL_MC):
        assert lib.tcb_autotune_set_threads(k, w, h, 0) == 0
        assert lib.tcb_autotune_threads(k, w, h) == 0


@pytest.mark.parametrize("threads", [64, 128, 256])
def test_deblock_tma_staging_matches_oracle(lib, threads):
    """The TMA-staged deblocking kernel (TCB_STAGING_TMA: 2D tile copies in
    and out of shared memory) on frames whose planes meet the tensor-map
    alignment (16-byte bases and strides), against the oracle; no bounded
    wait may have given up."""
    from tcodec_b200 import api
    rng = np.random.default_rng(12)
    cases = [make_case(rng, w, h, qp, 0) for w, h, qp in ((1920, 1080, 32), (256, 192, 42), (320, 240, 27),
                                                          (640, 384, 37))]
    assert lib.tcb_frame_kernels_errors() == 0
    got = run(lib, lib.tcb_deblock_frames, cases, api.KERNEL_DEBLOCK, threads | api.STAGING_TMA)
    assert lib.tcb_frame_kernels_errors() == 0
    for c, g in zip(cases, got):
        y, cb, cr = oracle_deblock(c)
        assert np.array_equal(g["y"], y), (c["w"], c["h"], c["qp"])
        assert np.array_equal(g["cb"], cb) and np.array_equal(g["cr"], cr), (c["w"], c["h"], c["qp"])
