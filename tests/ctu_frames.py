"""Drives a CTU-engine frame entry point over a clip the way the v2 frame
encoder does for a P-only GOP: device-resident DPB with the newest
reconstruction in slot 0, the previous frame's MV grid as the temporal
predictor, and the global-motion hint computed by the oracle restatement
(reference src/encoder.c:171-202) on the host copies of the source and
slot-0 reference.  Test helper; every buffer is a torch CUDA tensor."""
import ctypes

import numpy as np
import torch

from tcodec_b200 import api
from tests import orabind


def _dev(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint8)).cuda()


def _ptr(t: torch.Tensor) -> int:
    return t.data_ptr()


class FrameRun:
    """Holds the device state of one clip: sources, DPB, MV grids, records.

    `call(desc)` is the entry point under test (it receives a
    ctypes.POINTER(api.FrameDesc) and returns a tc_error_t); `step(t)`
    encodes frame t and returns its outputs as host copies."""

    def __init__(self, lib, frames, qp, preset, profile, call):
        self.lib = api.bind_b200(lib)
        self.frames = frames
        self.qp, self.preset, self.profile = qp, preset, profile
        self.call = call
        self.h, self.w = frames[0][0].shape
        self.gw, self.gh = (self.w + 7) // 8, (self.h + 7) // 8
        self.nctu = ((self.w + 63) // 64) * ((self.h + 63) // 64)
        cell = lib.tcb_mv_cell_bytes()
        init = np.zeros((self.gw * self.gh, cell), np.uint8)
        init[:, 4] = 1                                  # intra, zero vector
        self.grids = [_dev(init.reshape(-1)), _dev(init.reshape(-1))]
        self.records = torch.zeros(self.nctu * lib.tcb_ctu_record_bytes(), dtype=torch.uint8, device="cuda")
        self.dpb = []                                   # newest first: (y, cb, cr, poc)
        self.oracle = orabind.port()

    def step(self, t):
        y, cb, cr = (_dev(p) for p in self.frames[t])
        rec = [torch.empty_like(y), torch.empty_like(cb), torch.empty_like(cr)]
        d = api.FrameDesc()
        d.width, d.height, d.stride_y, d.stride_c = self.w, self.h, self.w, self.w // 2
        d.src_y, d.src_cb, d.src_cr = _ptr(y), _ptr(cb), _ptr(cr)
        d.rec_y, d.rec_cb, d.rec_cr = (_ptr(p) for p in rec)
        for i, (ry, rcb, rcr, poc) in enumerate(self.dpb):
            d.ref_y[i], d.ref_cb[i], d.ref_cr[i], d.ref_poc[i] = _ptr(ry), _ptr(rcb), _ptr(rcr), poc
        d.frame_type = 0 if t == 0 else 1
        d.prev_mv_grid = _ptr(self.grids[1]) if t > 0 else None
        d.cur_mv_grid = _ptr(self.grids[0])
        d.ctu_records = _ptr(self.records)
        d.poc, d.qp, d.preset, d.profile = t, self.qp, self.preset, self.profile
        if d.frame_type == 1:
            cur = np.ascontiguousarray(self.frames[t][0], dtype=np.uint8)
            ref = self.dpb[0][0].cpu().numpy()
            gx, gy = ctypes.c_int(), ctypes.c_int()
            self.oracle.or_global_mv(orabind.P(cur), orabind.P(ref), self.w, self.h, self.w,
                                     ctypes.byref(gx), ctypes.byref(gy))
            d.global_mv_valid, d.global_mv_x, d.global_mv_y = 1, gx.value, gy.value
        self.records.zero_()
        torch.cuda.synchronize()
        r = self.call(ctypes.byref(d))
        assert r == 0, f"frame entry point -> {r}"
        torch.cuda.synchronize()
        out = tuple(p.cpu().numpy() for p in rec) + (self.records.cpu().numpy(), self.grids[0].cpu().numpy())
        self.dpb = [(rec[0], rec[1], rec[2], t)] + self.dpb[:api.REF_FRAMES - 1]
        self.grids.reverse()
        return out

    def run(self):
        return [self.step(t) for t in range(len(self.frames))]


def clips():
    """(name, frames, qp, preset, profile) cases: non-aligned sizes, a
    motion large enough to enable the global-motion candidate, multiref."""
    from tcodec_b200 import synth
    return [
        ("sin200x136", synth.sinusoid_clip(200, 136, 4), 32, 2, 1),
        ("rect256x128_glob", synth.moving_rects_clip(256, 128, 3, motion=(6.0, -3.0)), 27, 2, 1),
        ("rect136x72_p0", synth.moving_rects_clip(136, 72, 3, motion=(7.0, 5.0)), 37, 1, 0),
    ]
