"""Failure detection in the CTU wavefront, without a GPU fault.

Every CTU waits for its left and above neighbours' publish flags with a
bounded back-off (tcb_set_neighbor_wait_limit).  The test hook launches a
frame's queue without its first CTU, so two waits are for a flag that
nothing sets: with a short limit they run out, the kernel records the
error and finishes, and tcb_ctu_frame_result reports TC_ERR_INTERNAL.
The same process then encodes the same frame normally, with the same
output as the library's fixed-scratch entry point."""
import ctypes
import time

import numpy as np
import pytest

from tests import ctu_frames

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from tcodec_b200 import api
    return api.bind_b200(api.load_library())


def test_expired_neighbor_wait_is_reported_and_context_survives(lib):
    import torch
    from tcodec_b200 import api
    name, frames, qp, preset, profile = ctu_frames.clips()[0]
    frames = frames[:1]                          # a key frame: intra only, 4 x 3 CTUs
    h, w = frames[0][0].shape
    nbytes = lib.tcb_ctu_scratch_bytes(w, h)
    scratch = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream().cuda_stream

    def without_first(desc):
        return lib.tcb_debug_ctu_encode_frame_without_first(desc, scratch.data_ptr(), nbytes, st)

    def whole(desc):
        return lib.tcb_ctu_encode_frame(desc, scratch.data_ptr(), nbytes, st)

    def static(desc):
        return lib.tcb_ctu_encode_frame_static(desc, st)

    default = ctypes.c_longlong()
    assert lib.tcb_get_neighbor_wait_limit(ctypes.byref(default)) == api.TC_OK
    assert default.value == 1 << 22
    assert lib.tcb_set_neighbor_wait_limit(0) == api.TC_ERR_PARAM
    try:
        # at most 4,096 back-offs of <= 2,048 ns: under 10 ms per wait
        assert lib.tcb_set_neighbor_wait_limit(1 << 12) == api.TC_OK
        run = ctu_frames.FrameRun(lib, frames, qp, preset, profile, without_first)
        t0 = time.perf_counter()
        run.run()
        assert lib.tcb_ctu_frame_result(scratch.data_ptr(), st) == api.TC_ERR_INTERNAL
        elapsed = time.perf_counter() - t0
        print(f"expired waits reported after {elapsed * 1e3:.1f} ms")
        assert elapsed < 5.0                     # the default bound alone is ~8.6 s
    finally:
        assert lib.tcb_set_neighbor_wait_limit(default.value) == api.TC_OK
    # the device context is still usable: the whole queue completes
    got = ctu_frames.FrameRun(lib, frames, qp, preset, profile, whole).run()
    assert lib.tcb_ctu_frame_result(scratch.data_ptr(), st) == api.TC_OK
    want = ctu_frames.FrameRun(lib, frames, qp, preset, profile, static).run()
    assert lib.tcb_ctu_frame_result_static(st) == api.TC_OK
    for k, what in enumerate(("y", "cb", "cr", "records", "mv grid")):
        assert np.array_equal(got[0][k], want[0][k]), what
    assert lib.tcb_ctu_frame_result(None, st) == api.TC_ERR_PARAM
