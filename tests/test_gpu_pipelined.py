"""Pipelined batch steps (tcb_batch_set_pipelined): each call entropy-codes
the previous call's frames while its own run on the device, so packets
arrive one call later.  Every stream's packet sequence must equal the
unpipelined batch's, across key / P / B frames, a stream that skips a
call, the B-frame drain and CUDA-graph replay; rate-controlled streams
are refused."""
import pytest

pytestmark = pytest.mark.gpu


def run_batch(lib, cfgs, clips, pipelined, graphs=False, skip=None):
    from tcodec_b200 import api
    batch = api.BatchEncoder(lib, cfgs)
    if pipelined:
        batch.set_pipelined(True)
    batch.set_graphs(graphs)
    got = [[] for _ in cfgs]
    first = None
    for t in range(max(len(c) for c in clips)):
        frames = [c[t] if t < len(c) and (i, t) != skip else None for i, c in enumerate(clips)]
        out = batch.encode(frames)
        for i, p in enumerate(out):
            if p is not None:
                got[i].append(p)
        if t == 0:
            first = out
    tail = batch.flush()
    batch.close()
    return [g + t for g, t in zip(got, tail)], first


@pytest.mark.parametrize("graphs", [False, True])
def test_pipelined_packets_equal_plain(graphs):
    from tcodec_b200 import api, synth
    lib = api.load_library()
    specs = [dict(w=320, h=240, qp=32, preset=2, profile=1, b=False),
             dict(w=256, h=136, qp=27, preset=2, profile=1, b=True),
             dict(w=192, h=128, qp=37, preset=1, profile=0, b=True),
             dict(w=128, h=96, qp=22, preset=2, profile=0, b=False)]
    n = 11
    clips = [synth.moving_rects_clip(s["w"], s["h"], n) for s in specs]
    cfgs = [api.make_config(lib, s["w"], s["h"], qp=s["qp"], preset=s["preset"], profile=s["profile"],
                            keyframe_interval=6, b_frames=s["b"]) for s in specs]
    plain, _ = run_batch(lib, cfgs, clips, False, skip=(3, 4))
    piped, first = run_batch(lib, cfgs, clips, True, graphs=graphs, skip=(3, 4))
    assert all(p is None for p in first)     # the first call's packets come with the second call
    for i in range(len(specs)):
        assert len(piped[i]) == len(plain[i]) and piped[i] == plain[i], i


def test_drain_returns_pending_packets_only():
    """tcb_batch_drain codes what the last call left pending and runs no new
    frame: P-only streams give exactly one packet each, then nothing."""
    from tcodec_b200 import api, synth
    lib = api.load_library()
    cfgs = [api.make_config(lib, 128, 96, keyframe_interval=1000) for _ in range(2)]
    clips = [synth.moving_rects_clip(128, 96, 3) for _ in cfgs]
    ref = api.BatchEncoder(lib, cfgs)
    want = [[] for _ in cfgs]
    for t in range(3):
        for i, p in enumerate(ref.encode([c[t] for c in clips])):
            want[i].append(p)
    ref.close()
    batch = api.BatchEncoder(lib, cfgs)
    batch.set_pipelined(True)
    got = [[] for _ in cfgs]
    for t in range(3):
        for i, p in enumerate(batch.encode([c[t] for c in clips])):
            if p is not None:
                got[i].append(p)
    last = batch.drain()
    assert all(p is not None for p in last)
    assert all(p is None for p in batch.drain())
    batch.close()
    for i in range(len(cfgs)):
        assert got[i] + [last[i]] == want[i]


def test_pipelined_refuses_rate_control():
    from tcodec_b200 import api
    lib = api.load_library()
    cfg = api.make_config(lib, 128, 96)
    cfg.rc_method = 1          # bitrate control: a frame's QP depends on the previous frame's bits
    cfg.target_bitrate = 500000
    batch = api.BatchEncoder(lib, [cfg])
    with pytest.raises(RuntimeError):
        batch.set_pipelined(True)
    batch.close()
