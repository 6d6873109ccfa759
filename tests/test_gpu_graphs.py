"""CUDA-graph replay of the batched step (tcb_batch_set_graphs): the step's
device work captured and replayed as one graph launch per step must give
exactly the packets of the plain launch sequence, across step shapes that
change (key, P and B frames, streams that skip a step, B-frame drain),
and against the reference's own digests for the mixed batch."""
import hashlib
import json
import os
import struct

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def run_batch(lib, cfgs, clips, graphs, skip=None):
    from tcodec_b200 import api
    batch = api.BatchEncoder(lib, cfgs)
    batch.set_graphs(graphs)
    got = [[] for _ in cfgs]
    steps = 0
    for t in range(max(len(c) for c in clips)):
        frames = [c[t] if t < len(c) and (i, t) != skip else None for i, c in enumerate(clips)]
        for i, p in enumerate(batch.encode(frames)):
            if p is not None:
                got[i].append(p)
        steps += 1
    tail = batch.flush()
    stats = batch.graph_stats()
    batch.close()
    return [g + t for g, t in zip(got, tail)], stats


def test_graph_replay_matches_plain_steps():
    from tcodec_b200 import api, synth
    lib = api.load_library()
    specs = [dict(w=320, h=240, qp=32, preset=2, profile=1, b=False),
             dict(w=256, h=136, qp=27, preset=2, profile=1, b=True),
             dict(w=192, h=128, qp=37, preset=1, profile=0, b=True),
             dict(w=128, h=96, qp=22, preset=2, profile=0, b=False)]
    n = 10
    clips = [synth.moving_rects_clip(s["w"], s["h"], n) for s in specs]
    cfgs = [api.make_config(lib, s["w"], s["h"], qp=s["qp"], preset=s["preset"], profile=s["profile"],
                            keyframe_interval=6, b_frames=s["b"]) for s in specs]
    plain, st0 = run_batch(lib, cfgs, clips, False, skip=(3, 4))
    graph, st1 = run_batch(lib, cfgs, clips, True, skip=(3, 4))
    for i in range(len(specs)):
        assert graph[i] == plain[i], i
    assert st0 == (0, 0, 0)
    launches, builds, refused = st1
    print("graph launches", launches, "instantiations", builds, "last refused update", refused)
    assert launches >= n and builds <= launches   # every step replayed a graph


def test_graph_replay_mixed_batch_matches_reference():
    from tcodec_b200 import api, synth
    gold = json.load(open(os.path.join(HERE, "golden", "mixed_streams.json")))
    lib = api.load_library()
    idx = [i for i, s in enumerate(gold["batch"]) if s["w"] <= 640][:24]
    specs = [gold["batch"][i] for i in idx]
    clips = [synth.stream_clip(s) for s in specs]
    cfgs = [api.make_config(lib, s["w"], s["h"], qp=s["qp"], preset=gold["preset"], profile=gold["profile"],
                            keyframe_interval=1000) for s in specs]
    got, (launches, builds, refused) = run_batch(lib, cfgs, clips, True)
    print("graph launches", launches, "instantiations", builds, "last refused update", refused)
    bad = []
    for i, s in enumerate(specs):
        h = hashlib.sha256()
        for p in got[i]:
            h.update(struct.pack("<I", len(p)) + p)
        if h.hexdigest() != s["digest"]:
            bad.append((idx[i], s["w"], s["h"], s["qp"]))
    assert not bad, bad
    # steps of one shape (all streams P after the key frame) reuse one
    # executable graph, updated in place
    assert launches >= 30 and builds <= 4, (launches, builds, refused)
