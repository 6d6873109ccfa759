"""Allocation failures, injected on the host (tcb_debug_fail_allocations_after),
never by exhausting the GPU.  Each device or pinned-host allocation that
creating an encoder, a decoder's first frames, or a batch makes is failed in
turn: the failure must surface as NULL from the create call or TC_ERR_MEMORY
from the decode call (the reference's contract, include/tcodec.h: create
returns NULL, decode TC_ERR_MEMORY), and the same process must then produce
exactly the unfailed output.  A decoder that returned TC_ERR_MEMORY is left
as it was before the call, so retrying the packet gives the unfailed
picture."""
import pytest

pytestmark = pytest.mark.gpu

MAX_ALLOCS = 400      # far above what any object here allocates


@pytest.fixture(scope="module")
def lib():
    from tcodec_b200 import api
    return api.bind_b200(api.load_library())


@pytest.fixture(autouse=True)
def disarm(lib):
    yield
    lib.tcb_debug_fail_allocations_after(-1)


def _failures(lib, attempt):
    """Runs attempt() with the k-th allocation failing, k = 0, 1, ..., until
    an attempt makes fewer than k + 1 allocations; returns the results."""
    results = []
    for k in range(MAX_ALLOCS):
        assert lib.tcb_debug_fail_allocations_after(k) < 0
        res = attempt()
        left = lib.tcb_debug_fail_allocations_after(-1)
        if left >= 0:                      # the armed failure never fired
            return results, k
        results.append(res)
    raise AssertionError("allocation count did not converge")


def test_encoder_create_failures_return_null(lib):
    from tcodec_b200 import api, synth
    frames = synth.sinusoid_clip(128, 64, 5)
    cfg = api.make_config(lib, 128, 64, qp=32, preset=2, profile=1, keyframe_interval=1000, b_frames=True)
    clean = api.encode_sequence(lib, cfg, frames)

    def attempt():
        try:
            enc = api.Encoder(lib, cfg)
        except RuntimeError:
            return "null"
        pk = [enc.encode(*f) for f in frames] + enc.flush()
        enc.close()
        return [p for p in pk if p is not None]

    results, nalloc = _failures(lib, attempt)
    print(f"encoder: {nalloc} allocations, each failed once")
    assert nalloc >= 20 and all(r == "null" for r in results)
    assert api.encode_sequence(lib, cfg, frames) == clean


def test_decoder_memory_errors_leave_state_retryable(lib):
    from tcodec_b200 import api, synth
    frames = synth.moving_rects_clip(128, 64, 4)
    cfg = api.make_config(lib, 128, 64, qp=30, preset=2, profile=1, keyframe_interval=1000)
    pk = api.encode_sequence(lib, cfg, frames)
    clean = api.decode_sequence(lib, pk)

    def attempt():
        dec = api.Decoder(lib)
        out, errors = [], 0
        for p in pk:
            try:
                f = dec.decode(p)
            except RuntimeError as e:
                assert e.args[1] == api.TC_ERR_MEMORY, e.args
                errors += 1
                f = dec.decode(p)          # the injected failure fires once: the retry allocates
            out.append(f)
        dec.close()
        return errors, out

    results, nalloc = _failures(lib, attempt)
    print(f"decoder: {nalloc} allocations over {len(pk)} packets, each failed once")
    assert nalloc >= 5
    for errors, out in results:
        assert errors == 1
        assert len(out) == len(clean)
        for a, b in zip(out, clean):
            for pa, pb in zip(a, b):
                assert (pa == pb).all()


def test_batch_create_failures_return_null(lib):
    from tcodec_b200 import api, synth
    specs = [(128, 64, 30), (96, 80, 34)]
    clips = [synth.sinusoid_clip(w, h, 3) for w, h, _ in specs]
    cfgs = [api.make_config(lib, w, h, qp=q, preset=2, profile=1, keyframe_interval=1000) for w, h, q in specs]

    def run():
        b = api.BatchEncoder(lib, cfgs)
        got = [[] for _ in cfgs]
        for t in range(3):
            for i, p in enumerate(b.encode([c[t] for c in clips])):
                if p is not None:
                    got[i].append(p)
        for i, tail in enumerate(b.flush()):
            got[i] += tail
        b.close()
        return got

    clean = run()

    def attempt():
        try:
            b = api.BatchEncoder(lib, cfgs)
        except RuntimeError:
            return "null"
        b.close()
        return "ok"

    results, nalloc = _failures(lib, attempt)
    print(f"batch: {nalloc} allocations at creation, each failed once")
    assert nalloc >= 40 and all(r == "null" for r in results)
    assert run() == clean
    for c, (w, h, _) in zip(clips, specs):
        assert c[0][0].shape == (h, w)
