"""GPU decoder: host parse + device reconstruction of v2 streams.

The decoded pictures must equal (a) the encoder's own reconstruction and
(b) the reference decoder's output on the same stream — for P-only,
multiref, raw Exp-Golomb, CRC, entry-point and B-frame (display reorder)
streams produced by either encoder.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from tcodec_b200 import api
    return api.load_library()


CASES = [
    dict(src="rect", w=320, h=240, n=5, qp=27, preset=2, profile=1),
    dict(src="sin", w=96, h=80, n=4, qp=32, preset=2, profile=0, entropy=False, crc=True),
    dict(src="rect", w=192, h=128, n=9, qp=32, preset=2, profile=1, b_frames=True),
    dict(src="sin", w=128, h=128, n=5, qp=37, preset=1, profile=0),
    dict(src="rect", w=256, h=136, n=4, qp=22, preset=0, profile=0, keyframe_interval=2),
]


def _frames(c):
    from tcodec_b200 import synth
    return (synth.sinusoid_clip if c["src"] == "sin" else synth.moving_rects_clip)(c["w"], c["h"], c["n"])


@pytest.mark.parametrize("ci", range(len(CASES)))
def test_decoder_matches_encoder_recon_and_reference_decoder(lib, ref_lib, ci):
    from tcodec_b200 import api
    c = dict(CASES[ci])
    frames = _frames(c)
    kw = {k: v for k, v in c.items() if k not in ("src", "w", "h", "n")}
    kw.setdefault("keyframe_interval", 1000)
    cfg = api.make_config(lib, c["w"], c["h"], **kw)
    pk, recons = api.encode_sequence(lib, cfg, frames, with_recon=True)
    mine = api.decode_sequence(lib, pk)
    ref = api.decode_sequence(ref_lib, pk)
    assert len(mine) == len(ref) == c["n"]
    for a, b in zip(mine, ref):
        for pa, pb in zip(a, b):
            assert np.array_equal(pa, pb)
    if not kw.get("b_frames"):
        for a, b in zip(mine, recons):
            for pa, pb in zip(a, b):
                assert np.array_equal(pa, pb)


@pytest.mark.parametrize("threads", [1, 3, 16])
def test_decoder_entry_point_rows_any_thread_count(lib, ref_lib, threads):
    """A 1280x720 GOP4-B stream (12 CTU rows, each an entry-point
    substream) decodes to the reference decoder's pictures whatever the
    number of host threads parsing the rows (tc_decoder_set_threads)."""
    from tcodec_b200 import api, synth
    frames = synth.workload("rects", frames=6, width=1280, height=720)
    cfg = api.make_config(lib, 1280, 720, qp=27, preset=2, profile=1, keyframe_interval=1000, b_frames=True)
    pk = api.encode_sequence(lib, cfg, frames)
    mine = api.decode_sequence(lib, pk, threads=threads)
    ref = api.decode_sequence(ref_lib, pk)
    assert len(mine) == len(ref) == len(frames)
    for a, b in zip(mine, ref):
        for pa, pb in zip(a, b):
            assert np.array_equal(pa, pb)


def test_decoder_on_reference_streams(lib, ref_lib):
    from tcodec_b200 import api, synth
    frames = synth.moving_rects_clip(160, 96, 5, seed_rects=5)
    cfg = api.make_config(ref_lib, 160, 96, qp=30, preset=2, profile=1, keyframe_interval=1000)
    pk = api.encode_sequence(ref_lib, cfg, frames)
    a = api.decode_sequence(lib, pk)
    b = api.decode_sequence(ref_lib, pk)
    for fa, fb in zip(a, b):
        for pa, pb in zip(fa, fb):
            assert np.array_equal(pa, pb)


def test_truncated_and_corrupt_packets_rejected(lib):
    """Truncated packets must be rejected (reference test_v2_roundtrip
    1125-1134); a corrupted CRC is reported, not fatal."""
    from tcodec_b200 import api, synth
    frames = synth.sinusoid_clip(64, 64, 2)
    cfg = api.make_config(lib, 64, 64, qp=32, crc=True, keyframe_interval=1000)
    pk = api.encode_sequence(lib, cfg, frames)
    dec = api.Decoder(lib)
    with pytest.raises(RuntimeError):
        dec.decode(pk[0][:5])
    with pytest.raises(RuntimeError):
        dec.decode(b"XYZ" + pk[0][3:])
    dec.close()
    dec = api.Decoder(lib)
    bad = bytearray(pk[0])
    bad[-1] ^= 0xFF
    dec.decode(bytes(bad))
    assert dec.crc_valid() == 0
    dec.decode(pk[1])
    assert dec.crc_valid() == 1
    dec.close()
