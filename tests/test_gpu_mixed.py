"""Mixed-resolution batched workload against the reference encoder's
digests (tests/golden/mixed_streams.json, made by
tests/golden/make_mixed_golden.py with the reference library): the
streams of the 64-stream mix up to 640x360, all in one batch, must produce
exactly the reference's packets and final reconstruction."""
import hashlib
import json
import os
import struct

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def test_mixed_batch_small_streams_match_reference():
    from tcodec_b200 import api, synth
    gold = json.load(open(os.path.join(HERE, "golden", "mixed_streams.json")))
    lib = api.load_library()
    idx = [i for i, s in enumerate(gold["batch"]) if s["w"] <= 640]
    specs = [gold["batch"][i] for i in idx]
    clips = [synth.stream_clip(s) for s in specs]
    cfgs = [api.make_config(lib, s["w"], s["h"], qp=s["qp"], preset=gold["preset"], profile=gold["profile"],
                            keyframe_interval=1000) for s in specs]
    batch = api.BatchEncoder(lib, cfgs)
    got = [[] for _ in specs]
    for t in range(max(len(c) for c in clips)):
        for i, p in enumerate(batch.encode([c[t] if t < len(c) else None for c in clips])):
            if p is not None:
                got[i].append(p)
    recon = [batch_recon(lib, batch, i) for i in range(len(specs))]
    tail = batch.flush()
    batch.close()
    bad = []
    for i, s in enumerate(specs):
        h = hashlib.sha256()
        for p in got[i] + tail[i]:
            h.update(struct.pack("<I", len(p)) + p)
        if h.hexdigest() != s["digest"] or recon[i] != s["recon"]:
            bad.append((idx[i], s["w"], s["h"], s["qp"]))
    assert not bad, bad


def batch_recon(lib, batch, i):
    """SHA-256 of stream i's host reconstruction (tc_encoder_t.recon)."""
    import ctypes
    from tcodec_b200 import api
    enc = api.EncoderHead.from_address(lib.tcb_batch_encoder(batch.h, i))
    fb = enc.recon.contents
    w, h = fb.width, fb.height
    r = hashlib.sha256()
    for ptr, stride, pw, ph in ((fb.y, fb.stride_y, w, h), (fb.cb, fb.stride_c, w // 2, h // 2),
                                (fb.cr, fb.stride_c, w // 2, h // 2)):
        base = ctypes.cast(ptr, ctypes.c_void_p).value
        for y in range(ph):
            r.update(ctypes.string_at(base + y * stride, pw))
    return r.hexdigest()
