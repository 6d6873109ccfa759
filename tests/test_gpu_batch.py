"""Batched form: N streams of mixed resolution / QP / preset / GOP in
shared CTU-engine launches must produce, per stream, exactly the packets
that stream produces when encoded alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_batch_matches_single_stream_encodes():
    from tcodec_b200 import api, synth
    lib = api.load_library()
    specs = [
        dict(w=320, h=240, qp=32, preset=2, profile=1, src="rect"),
        dict(w=128, h=96, qp=22, preset=2, profile=0, src="sin"),
        dict(w=192, h=128, qp=37, preset=1, profile=0, src="rect"),
        dict(w=256, h=136, qp=27, preset=2, profile=1, src="sin", b_frames=True),
        dict(w=96, h=80, qp=27, preset=0, profile=0, src="rect"),
    ]
    n_frames = 6
    clips = [(synth.sinusoid_clip if s["src"] == "sin" else synth.moving_rects_clip)(s["w"], s["h"], n_frames)
             for s in specs]
    cfgs = [api.make_config(lib, s["w"], s["h"], qp=s["qp"], preset=s["preset"], profile=s["profile"],
                            keyframe_interval=1000, b_frames=s.get("b_frames", False)) for s in specs]
    batch = api.BatchEncoder(lib, cfgs)
    got = [[] for _ in specs]
    for t in range(n_frames):
        # stream 2 skips frame 3 (no input that call) to exercise partial steps
        frames = [None if (i == 2 and t == 3) else clips[i][t] for i in range(len(specs))]
        for i, p in enumerate(batch.encode(frames)):
            if p is not None:
                got[i].append(p)
    tail = batch.flush()
    batch.close()
    for i, s in enumerate(specs):
        frames = [f for t, f in enumerate(clips[i]) if not (i == 2 and t == 3)]
        want = api.encode_sequence(lib, cfgs[i], frames)
        assert got[i] + tail[i] == want, i
