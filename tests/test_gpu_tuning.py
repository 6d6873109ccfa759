"""The engine knobs change speed only: a batch of streams encodes to the
same bytes under every search-window radius and both wavefront queue orders
(and equal to the reference encoder's bytes), and the autotuner runs end to
end and records one of the combinations it timed."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W, H, N, STREAMS = 256, 192, 6, 3


@pytest.fixture(scope="module")
def lib():
    from tcodec_b200 import api
    return api.bind_b200(api.load_library())


def _clips():
    from tcodec_b200 import synth
    return [synth.moving_rects_clip(W, H, N, motion=(3.5 + s, -1.25), seed_rects=40 + s, seed_noise=50 + s)
            for s in range(STREAMS)]


def _batch_packets(lib, clips, b_frames):
    from tcodec_b200 import api
    cfgs = [api.make_config(lib, W, H, qp=30, preset=2, profile=1, keyframe_interval=1000, b_frames=b_frames)
            for _ in clips]
    b = api.BatchEncoder(lib, cfgs)
    try:
        out = [[] for _ in clips]
        for t in range(N):
            for i, p in enumerate(b.encode([c[t] for c in clips])):
                if p is not None:
                    out[i].append(p)
        for i, tail in enumerate(b.flush()):
            out[i].extend(tail)
        return out
    finally:
        b.close()


@pytest.mark.parametrize("b_frames", [False, True], ids=["p_only", "gop4_b"])
def test_engine_knobs_do_not_change_output(lib, ref_lib, b_frames):
    from tcodec_b200 import api
    clips = _clips()
    want = [api.encode_sequence(ref_lib, api.make_config(ref_lib, W, H, qp=30, preset=2, profile=1,
                                                         keyframe_interval=1000, b_frames=b_frames), c)
            for c in clips]
    try:
        for r, o in ((2, api.QUEUE_DIAGONAL), (3, api.QUEUE_STAGGERED), (5, api.QUEUE_STAGGERED),
                     (4, api.QUEUE_DIAGONAL)):
            api.set_engine_tuning(lib, W, H, r, o)
            assert _batch_packets(lib, clips, b_frames) == want, (r, o)
    finally:
        api.set_engine_tuning(lib, W, H, 0, 0)


def test_autotuner_records_a_timed_choice(lib):
    from tcodec_b200 import api, tuning
    cfg = api.make_config(lib, W, H, qp=30, preset=2, profile=1, keyframe_interval=1000, b_frames=True)
    frames = _clips()[0]
    try:
        res = tuning.tune_engine(lib, cfg, frames, streams=2, steps=1, warmup=2, windows=(3, 4),
                                 orders=(api.QUEUE_DIAGONAL, api.QUEUE_STAGGERED))
        assert set(res["ms_per_step"]) == {(3, 0), (3, 1), (4, 0), (4, 1)}
        assert all(np.isfinite(v) and v > 0 for v in res["ms_per_step"].values())
        assert res["chosen"] in res["ms_per_step"]
        assert api.engine_tuning(lib, W, H) == res["chosen"]
        assert tuning.describe(res)["search_window"] == res["chosen"][0]
    finally:
        api.set_engine_tuning(lib, W, H, 0, 0)
