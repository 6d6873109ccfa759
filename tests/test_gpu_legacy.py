"""Legacy (v0 / v1) 8x8 block path on the GPU against the reference.

The encoder runs tcb_legacy.cu's CTU wavefront (decisions and
reconstruction on the device, syntax on the host); the decoder parses on
the host and reconstructs on the device.  Parity is byte-exact packets and
sample-exact reconstructions:
  * the reference's committed conformance hashes of every v0, v1 and v1e
    stream of its golden corpus (reference golden/MANIFEST.sha256);
  * live sequences against the reference library (oracle/_ref/libtcref.so):
    P frames, key frames at the interval, multi-reference search, B-frame
    GOPs, raw / range-coded syntax, one run or per-row runs, CRC;
  * the decoder on reference-encoded streams against the reference decoder.
"""
import hashlib
import struct

import numpy as np
import pytest

from tests.golden import make_golden as golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from tcodec_b200 import api
    return api.load_library()


def _enc_file(lib, frames, **kw):
    from tcodec_b200 import api
    cfg = api.make_config(lib, frames[0][0].shape[1], frames[0][0].shape[0], **kw)
    pk = api.encode_sequence(lib, cfg, frames)
    return b"".join(struct.pack("<I", len(p)) + p for p in pk)


def test_golden_legacy_streams(lib):
    """All 72 v0 / v1 / v1e streams of the reference's golden corpus."""
    bad = []
    rows = golden.load(golden.OUT_LEGACY)
    assert len(rows) == 72
    for (digest, name, pat, w, h, qp, var) in rows:
        y, cb, cr = golden.clip(pat, w, h)
        Y = np.frombuffer(y, np.uint8).reshape(h, w)
        C = np.frombuffer(cb, np.uint8).reshape(h // 2, w // 2)
        blob = _enc_file(lib, [(Y, C, C)], qp=qp, preset=2, keyframe_interval=250, **golden.LEGACY_VARIANTS[var])
        if hashlib.sha256(blob).hexdigest() != digest:
            bad.append(name)
    assert not bad, bad


CASES = [
    # (id, w, h, frames, config)
    ("v1_wpp_p", 192, 136, 6, dict(version=1, qp=30, preset=2, entropy=False)),
    ("v1_rows_serial", 192, 136, 5, dict(version=1, qp=26, preset=1, entropy=False, threads=1)),
    ("v0_p", 128, 128, 5, dict(version=0, qp=34, preset=2, entropy=False)),
    ("v1e_crc", 192, 136, 6, dict(version=1, qp=28, preset=2, entropy=True, crc=True)),
    ("v1_slow_multiref", 192, 136, 6, dict(version=1, qp=30, preset=3, profile=1, entropy=False)),
    ("v1e_ultrafast", 320, 240, 4, dict(version=1, qp=38, preset=0, entropy=True)),
    ("v1_keyint3", 136, 88, 7, dict(version=1, qp=22, preset=2, entropy=False, keyframe_interval=3)),
    ("v1e_gop4_b", 192, 136, 9, dict(version=1, qp=30, preset=2, profile=1, entropy=True, b_frames=True)),
    ("v1_gop4_b_wpp", 192, 136, 9, dict(version=1, qp=32, preset=2, entropy=False, b_frames=True)),
]


def _clip(w, h, n, seed):
    from tcodec_b200 import synth
    return synth.moving_rects_clip(w, h, n, seed_rects=seed, seed_noise=seed + 1)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_live_parity_with_reference(lib, ref_lib, case):
    from tcodec_b200 import api
    _, w, h, n, kw = case
    frames = _clip(w, h, n, 11)
    kw = dict(kw)
    kw.setdefault("keyframe_interval", 1000)
    outs = []
    for L in (ref_lib, lib):
        cfg = api.make_config(L, w, h, **kw)
        outs.append(api.encode_sequence(L, cfg, frames, with_recon=True))
    (pr, rr), (pg, rg) = outs
    assert len(pr) == len(pg)
    for i, (a, b) in enumerate(zip(pr, pg)):
        assert a == b, f"packet {i} differs"
    for a, b in zip(rr, rg):
        for pa, pb in zip(a, b):
            assert np.array_equal(pa, pb)


@pytest.mark.parametrize("case", [c for c in CASES if c[0] in ("v1_wpp_p", "v1e_crc", "v1_slow_multiref",
                                                                 "v0_p", "v1e_gop4_b", "v1_gop4_b_wpp")],
                         ids=lambda c: c[0])
def test_decoder_matches_reference_decoder(lib, ref_lib, case):
    from tcodec_b200 import api
    _, w, h, n, kw = case
    frames = _clip(w, h, n, 5)
    kw = dict(kw)
    kw.setdefault("keyframe_interval", 1000)
    cfg = api.make_config(ref_lib, w, h, **kw)
    pkts = api.encode_sequence(ref_lib, cfg, frames)
    want = api.decode_sequence(ref_lib, pkts, w, h)
    got = api.decode_sequence(lib, pkts, w, h)
    assert len(want) == len(got) == n
    for i, (a, b) in enumerate(zip(want, got)):
        for pa, pb in zip(a, b):
            assert np.array_equal(pa, pb), f"frame {i}"


def test_encoder_decoder_round_trip(lib):
    """The library's own legacy stream decodes to its own reconstruction."""
    from tcodec_b200 import api
    w, h, n = 200, 120, 6
    frames = _clip(w, h, n, 3)
    cfg = api.make_config(lib, w, h, version=1, qp=27, preset=2, entropy=True, keyframe_interval=1000)
    pkts, recons = api.encode_sequence(lib, cfg, frames, with_recon=True)
    dec = api.decode_sequence(lib, pkts, w, h)
    for r, d in zip(recons, dec):
        for pa, pb in zip(r, d):
            assert np.array_equal(pa, pb)
