"""tcb_ctu_encode_frame_static: the frame entry point whose scratch is a
fixed device array inside the library.  Called through the C ABI on
consecutive frames (key frame, then P-frames that read the previous
calls' reconstructions and MV grids), its reconstruction, MV grid and CTU
records must equal those of tcb_ctu_encode_frame with caller scratch,
exactly (the encoder is integer throughout).  Collected last so that it
also runs after every other test in one process."""
import ctypes

import numpy as np
import pytest

from tests import ctu_frames

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from tcodec_b200 import api
    return api.bind_b200(api.load_library())


def _with_scratch(lib, w, h):
    import torch
    nbytes = lib.tcb_ctu_scratch_bytes(w, h)
    scratch = torch.empty(nbytes, dtype=torch.uint8, device="cuda")

    def call(desc):
        return lib.tcb_ctu_encode_frame(desc, scratch.data_ptr(), nbytes, torch.cuda.current_stream().cuda_stream)
    call.scratch = scratch
    return call


def _static(lib):
    import torch

    def call(desc):
        return lib.tcb_ctu_encode_frame_static(desc, torch.cuda.current_stream().cuda_stream)
    return call


@pytest.mark.parametrize("case", ctu_frames.clips()[:2], ids=lambda c: c[0])
def test_static_scratch_matches_caller_scratch(lib, case):
    name, frames, qp, preset, profile = case
    frames = frames[:3]
    h, w = frames[0][0].shape
    want = ctu_frames.FrameRun(lib, frames, qp, preset, profile, _with_scratch(lib, w, h)).run()
    got = ctu_frames.FrameRun(lib, frames, qp, preset, profile, _static(lib)).run()
    assert len(got) == len(want) == len(frames)
    for t, (g, r) in enumerate(zip(got, want)):
        for k, what in enumerate(("y", "cb", "cr", "records", "mv grid")):
            assert np.array_equal(g[k], r[k]), (name, t, what)


def test_static_scratch_rejects_oversize_frames(lib):
    import torch
    from tcodec_b200 import api
    buf = torch.zeros(256, dtype=torch.uint8, device="cuda")
    p = buf.data_ptr()
    d = api.FrameDesc()
    d.src_y = d.src_cb = d.src_cr = d.rec_y = d.rec_cb = d.rec_cr = p
    d.cur_mv_grid = d.ctu_records = p
    d.qp, d.preset, d.profile = 32, 2, 1
    st = torch.cuda.current_stream().cuda_stream
    # 4096x2160 is 64 x 34 = 2176 CTUs, above the 2048-CTU static scratch:
    # rejected before anything is launched.
    d.width, d.height, d.stride_y, d.stride_c = 4096, 2160, 4096, 2048
    assert lib.tcb_ctu_encode_frame_static(ctypes.byref(d), st) == api.TC_ERR_MEMORY
    d.width = 4095                      # odd width: invalid descriptor
    assert lib.tcb_ctu_encode_frame_static(ctypes.byref(d), st) == api.TC_ERR_PARAM
    assert lib.tcb_ctu_encode_frame_static(None, st) == api.TC_ERR_PARAM
