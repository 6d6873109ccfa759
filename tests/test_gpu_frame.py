"""Standalone frame entry point of the CTU engine (tcb_ctu_encode_frame).

Driven with a caller-managed DPB over P-only GOPs, its reconstruction must
equal the full encoder's after every frame (the encoder's own output is
pinned to the reference by test_gpu_encoder.py), and it must reject
invalid descriptors and short scratch buffers."""
import ctypes

import numpy as np
import pytest

from tests import ctu_frames

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from tcodec_b200 import api
    return api.bind_b200(api.load_library())


def _entry(lib, w, h):
    import torch
    nbytes = lib.tcb_ctu_scratch_bytes(w, h)
    scratch = torch.empty(nbytes, dtype=torch.uint8, device="cuda")

    def call(desc):
        return lib.tcb_ctu_encode_frame(desc, scratch.data_ptr(), nbytes,
                                        torch.cuda.current_stream().cuda_stream)
    call.scratch = scratch
    return call


@pytest.mark.parametrize("case", ctu_frames.clips(), ids=lambda c: c[0])
def test_frame_entry_matches_encoder(lib, case):
    from tcodec_b200 import api
    name, frames, qp, preset, profile = case
    h, w = frames[0][0].shape
    cfg = api.make_config(lib, w, h, qp=qp, preset=preset, profile=profile, keyframe_interval=1000)
    _, recons = api.encode_sequence(lib, cfg, frames, with_recon=True)
    got = ctu_frames.FrameRun(lib, frames, qp, preset, profile, _entry(lib, w, h)).run()
    assert len(got) == len(recons)
    for t, (g, want) in enumerate(zip(got, recons)):
        for k in range(3):
            assert np.array_equal(g[k], want[k]), (name, t, k)


def test_frame_entry_rejects_bad_input(lib):
    import torch
    from tcodec_b200 import api
    w, h = 128, 64
    buf = torch.zeros(w * h * 2, dtype=torch.uint8, device="cuda")
    p = buf.data_ptr()
    d = api.FrameDesc()
    d.width, d.height, d.stride_y, d.stride_c = w, h, w, w // 2
    d.src_y = d.src_cb = d.src_cr = d.rec_y = d.rec_cb = d.rec_cr = p
    d.cur_mv_grid = d.ctu_records = p
    d.qp, d.preset, d.profile = 32, 2, 1
    need = lib.tcb_ctu_scratch_bytes(w, h)
    st = torch.cuda.current_stream().cuda_stream
    assert lib.tcb_ctu_encode_frame(ctypes.byref(d), p, need - 1, st) == api.TC_ERR_PARAM
    for field, bad in (("width", 0), ("width", 127), ("height", 5000), ("stride_y", 64), ("qp", 64),
                       ("frame_type", 3), ("preset", 4)):
        old = getattr(d, field)
        setattr(d, field, bad)
        assert lib.tcb_ctu_encode_frame(ctypes.byref(d), p, need, st) == api.TC_ERR_PARAM, field
        setattr(d, field, old)
    assert lib.tcb_ctu_encode_frame(None, p, need, st) == api.TC_ERR_PARAM
    assert lib.tcb_ctu_scratch_bytes(0, 64) == 0
