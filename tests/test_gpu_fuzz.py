"""Corrupted v2 streams through the decoder, after the reference's fuzz
tests (test/test_tcodec.c:1282-1726 bit flips and malformed packets,
2381-2468 systematic edge cases), which require that decoding never
crashes.  Here the outcome of every packet (error code, a picture held for
display reorder, or the decoded picture) must also equal the reference
decoder's, packet by packet, for every mutation that leaves the version
and frame-size bytes of the header alone.

Those bytes are the exception.  A version flipped to v0 / v1 sends the
reference to its legacy block decoder, which this library does not have
(v2 only: such frames are rejected).  A frame size changed in mid-stream
makes the reference reallocate its current frame while it keeps decoding
with the first frame's size and its old reference frames, a state its
debug build asserts against; this decoder starts over at the new size
(reference frames dropped).  For those mutations the test requires only
that every call returns and that the decoder stays usable.

The device kernel only ever sees a frame whose parse succeeded, and every
reference it reads is checked for presence first (an absent one predicts
flat or from the other direction), so no corrupted stream reaches the GPU
with an out-of-range index."""
import hashlib
import random

import pytest

pytestmark = pytest.mark.gpu

SPECS = [dict(w=96, h=80, n=4, qp=32, preset=2, profile=1, src="rect"),
         dict(w=128, h=64, n=4, qp=27, preset=2, profile=0, entropy=False, crc=True, src="sin"),
         dict(w=128, h=96, n=6, qp=32, preset=2, profile=1, b_frames=True, src="rect"),
         dict(w=64, h=64, n=3, qp=37, preset=1, profile=0, src="sin", keyframe_interval=2)]
TRIALS = 200
VERSION_AND_SIZE = range(3, 8)   # header bytes: version, width (16 bits), height (16 bits)


@pytest.fixture(scope="module")
def lib():
    from tcodec_b200 import api
    return api.load_library()


def digest(planes):
    return hashlib.sha1(b"".join(p.tobytes() for p in planes)).hexdigest()[:16]


def outcomes(L, packets):
    """Per packet: 'err<code>', 'wait' (display reorder) or the picture's
    digest; then the pictures the final flush drains."""
    from tcodec_b200 import api
    dec = api.Decoder(L)
    out = []
    try:
        for p in packets:
            try:
                f = dec.decode(p)
                out.append("wait" if f is None else digest(f))
            except RuntimeError as e:
                out.append("err%d" % e.args[1])
        try:
            out.extend("flush" + digest(f) for f in dec.flush())
        except RuntimeError as e:
            out.append("flusherr%d" % e.args[1])
    finally:
        dec.close()
    return out


def mutate(rng, p):
    p = bytearray(p)
    kind = rng.choice(["flip1", "flip8", "header", "truncate", "garbage"])
    if kind == "flip1" or kind == "header":
        b = rng.randrange((len(p) if kind == "flip1" else min(len(p), 16)) * 8)
        p[b >> 3] ^= 1 << (b & 7)
    elif kind == "flip8":
        for _ in range(8):
            b = rng.randrange(len(p) * 8)
            p[b >> 3] ^= 1 << (b & 7)
    elif kind == "truncate":
        p = p[:rng.randrange(1, len(p))]
    else:
        o, n = rng.randrange(len(p)), rng.randrange(1, 16)
        p[o:o + n] = bytes(rng.randrange(256) for _ in range(n))
    return bytes(p), kind


@pytest.mark.parametrize("si", range(len(SPECS)))
def test_corrupted_streams_match_reference_decoder(lib, ref_lib, si):
    from tcodec_b200 import api, synth
    s = SPECS[si]
    frames = (synth.sinusoid_clip if s["src"] == "sin" else synth.moving_rects_clip)(s["w"], s["h"], s["n"])
    kw = {k: v for k, v in s.items() if k not in ("w", "h", "n", "src")}
    kw.setdefault("keyframe_interval", 1000)
    pk = api.encode_sequence(lib, api.make_config(lib, s["w"], s["h"], **kw), frames)
    clean = outcomes(lib, pk)
    assert clean == outcomes(ref_lib, pk)
    rng = random.Random(1000 + si)
    compared = robust = 0
    for _ in range(TRIALS):
        i = rng.randrange(len(pk))
        bad, kind = mutate(rng, pk[i])
        seq = list(pk)
        seq[i] = bad
        got = outcomes(lib, seq)
        orig = pk[i]
        if any(k < len(bad) and bad[k] != orig[k] for k in VERSION_AND_SIZE) or len(bad) <= 7:
            robust += 1
            assert len(got) >= len(seq)
            continue
        want = outcomes(ref_lib, seq)
        assert got == want, (si, kind, i, got, want)
        compared += 1
    print(f"spec {si}: {compared} mutated streams equal to the reference decoder, {robust} robustness-only")
    assert compared > TRIALS // 2
    # the decoder (and its device context) is still sound afterwards
    assert outcomes(lib, pk) == clean


def test_malformed_headers_without_crash(lib, ref_lib):
    """The reference's systematic edge cases (test_fuzz_edge_cases): valid
    magic with garbage after the header, zero dimensions, the largest QP
    delta, 65535 x 65535.  Both decoders must return an error code or a
    picture; zero and oversized dimensions are errors in both."""
    from tcodec_b200 import api
    magic = bytes([0x54, 0x43, 0x56])
    garbage = magic + bytes([0, 0, 64, 0, 64, 0x80]) + bytes(23)
    zero = magic + bytes(13)
    qp = magic + bytes([0, 0, 64, 0, 64, 0x80, 0xFF]) + bytes(6)
    huge = magic + bytes([0, 0xFF, 0xFF, 0xFF, 0xFF, 0x80]) + bytes(7)
    for L in (lib, ref_lib):
        for p in (garbage, zero, qp, huge):
            dec = api.Decoder(L)
            try:
                dec.decode(p)
            except RuntimeError:
                pass
            dec.close()
        for p in (zero, huge):
            dec = api.Decoder(L)
            with pytest.raises(RuntimeError) as e:
                dec.decode(p)
            assert e.value.args[1] == api.TC_ERR_BITSTREAM
            dec.close()
