"""tcb_ctu_encode_frame_static: the frame entry point whose scratch is a
fixed device array inside the library, for callers that cannot allocate
device memory themselves (a pool allocator owns the GPU, a plugin host
only lends its frame buffers, a real-time loop forbids cudaMalloc / cudaFree
and the device synchronisation they imply).  Called through the C ABI on
consecutive frames (key frame, then P-frames that read the previous
calls' reconstructions and MV grids), its reconstruction, MV grid and CTU
records must equal those of tcb_ctu_encode_frame with caller scratch,
exactly (the encoder is integer throughout), and the calls must allocate
nothing.  Collected last so that it also runs after every other test in one
process."""
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


def _static_armed(lib, seen):
    """The static entry point with the library's allocation fault injector
    armed at 0 around every call: the library's next device or pinned-host
    allocation would fail.  Records, per call, the injector's pending count
    afterwards (0: nothing was allocated) and the drop in the device's free
    memory across the call."""
    import torch

    def call(desc):
        st = torch.cuda.current_stream().cuda_stream
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        lib.tcb_debug_fail_allocations_after(0)
        r = lib.tcb_ctu_encode_frame_static(desc, st)
        pending = lib.tcb_debug_fail_allocations_after(-1)
        if r == 0:
            r = lib.tcb_ctu_frame_result_static(st)
        torch.cuda.synchronize()
        seen.append((pending, free0 - torch.cuda.mem_get_info()[0]))
        return r
    return call


def test_static_scratch_allocates_nothing(lib):
    """With the fault injector armed, every call returns TC_OK, leaves the
    armed failure pending, takes no device memory, and still matches the
    caller-scratch entry point bit for bit.  The caller-scratch run goes
    first, so the kernels' module and the driver's local-memory reservation
    for the engine's stack exist before the static calls are watched."""
    lib.tcb_debug_fail_allocations_after.argtypes = [ctypes.c_longlong]
    lib.tcb_debug_fail_allocations_after.restype = ctypes.c_longlong
    name, frames, qp, preset, profile = ctu_frames.clips()[0]
    frames = frames[:3]
    h, w = frames[0][0].shape
    want = ctu_frames.FrameRun(lib, frames, qp, preset, profile, _with_scratch(lib, w, h)).run()
    seen = []
    got = ctu_frames.FrameRun(lib, frames, qp, preset, profile, _static_armed(lib, seen)).run()
    assert len(seen) == len(frames)
    for t, (pending, drop) in enumerate(seen):
        assert pending == 0, (t, "an allocation was attempted")
        assert drop == 0, (t, drop)
    for t, (g, r) in enumerate(zip(got, want)):
        for k, what in enumerate(("y", "cb", "cr", "records", "mv grid")):
            assert np.array_equal(g[k], r[k]), (name, t, what)
