"""Standalone motion compensation (tcb_mc_frames) against the oracle
restatement of tc_inter_predict / tc_inter_predict_chroma, bit-exact:
several frames per launch, partial blocks at the right / bottom border,
unaligned strides, and vectors that exercise all three luma paths
(integer copy, full six-tap block, per-sample edge-safe)."""
import ctypes

import numpy as np
import pytest

from tcodec_b200.api import McFrame
from tests import orabind

pytestmark = pytest.mark.gpu


def bind(lib):
    from tcodec_b200 import api
    return api.bind_b200(lib)


def make_case(rng, w, h, pad, kind):
    from tcodec_b200 import synth
    y, cb, cr = synth.moving_rects_clip(w, h, 1, seed_luma=int(rng.integers(1 << 20)))[0]
    gw, gh = (w + 7) // 8, (h + 7) // 8
    if kind == "random":       # quarter-pel vectors within +-24 px, some far outside the frame
        mv = rng.integers(-96, 97, (gh, gw, 2))
        far = rng.random((gh, gw)) < 0.05
        mv[far] = rng.integers(-4 * w, 4 * w, (int(far.sum()), 2))
    elif kind == "integer":    # whole-sample vectors: the copy path inside the frame
        mv = rng.integers(-16, 17, (gh, gw, 2)) * 4
    else:                      # one global fractional motion (+2.5, +0.75) px
        mv = np.broadcast_to(np.array([10, 3]), (gh, gw, 2)).copy()
    return dict(w=w, h=h, pad=pad, y=y, cb=cb, cr=cr, mv=mv.astype(np.int16))


def padded(a, pad):
    h, w = a.shape
    out = np.zeros((h, w + pad), np.uint8)
    out[:, :w] = a
    return out


def run_gpu(lib, cases):
    import torch
    frames = (McFrame * len(cases))()
    keep = []
    for f, c in zip(frames, cases):
        w, h, pad = c["w"], c["h"], c["pad"]
        ry, rcb, rcr = (torch.from_numpy(padded(c[k], pad)).cuda() for k in ("y", "cb", "cr"))
        py = torch.full_like(ry, 7)
        pcb, pcr = torch.full_like(rcb, 7), torch.full_like(rcr, 7)
        tmv = torch.from_numpy(np.ascontiguousarray(c["mv"])).cuda()
        keep.append((ry, rcb, rcr, py, pcb, pcr, tmv))
        f.width, f.height, f.stride_y, f.stride_c = w, h, ry.shape[1], rcb.shape[1]
        f.ref_y, f.ref_cb, f.ref_cr = ry.data_ptr(), rcb.data_ptr(), rcr.data_ptr()
        f.pred_y, f.pred_cb, f.pred_cr = py.data_ptr(), pcb.data_ptr(), pcr.data_ptr()
        f.mv = tmv.data_ptr()
    torch.cuda.synchronize()
    assert lib.tcb_mc_frames(frames, len(cases), torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    return [tuple(t.cpu().numpy() for t in k[3:6]) for k in keep]


def run_oracle(c):
    L = orabind.port()
    w, h = c["w"], c["h"]
    wc, hc = w // 2, h // 2
    y, cb, cr = (np.ascontiguousarray(c[k]) for k in ("y", "cb", "cr"))
    py, pcb, pcr = np.zeros((h, w), np.uint8), np.zeros((hc, wc), np.uint8), np.zeros((hc, wc), np.uint8)
    tl, tc = np.zeros((8, 8), np.uint8), np.zeros((4, 4), np.uint8)
    for by in range(0, h, 8):
        for bx in range(0, w, 8):
            dx, dy = (int(v) for v in c["mv"][by // 8, bx // 8])
            mx, my = bx * 4 + dx, by * 4 + dy
            L.or_pred_luma(orabind.P(y), w, w, h, mx, my, orabind.P(tl), 8, 8)
            py[by:by + 8, bx:bx + 8] = tl[:min(8, h - by), :min(8, w - bx)]
            for src, dst in ((cb, pcb), (cr, pcr)):
                L.or_pred_chroma(orabind.P(src), wc, wc, hc, mx, my, orabind.P(tc), 4, 4)
                cy, cx = by // 2, bx // 2
                dst[cy:cy + 4, cx:cx + 4] = tc[:min(4, hc - cy), :min(4, wc - cx)]
    return py, pcb, pcr


CASES = [(1920, 1080, 0, "global"), (200, 136, 0, "random"), (130, 70, 6, "random"), (256, 128, 0, "integer"),
         (96, 80, 2, "random")]


@pytest.mark.parametrize("threads", [0, 64, 128, 256])
def test_mc_frames_match_oracle(threads):
    """Every CTA-size variant (recorded for the first frame's size, the
    size a launch is tuned by) against the oracle."""
    from tcodec_b200 import api
    lib = bind(api.load_library())
    rng = np.random.default_rng(9)
    cases = [make_case(rng, *c) for c in CASES]
    if threads:
        assert lib.tcb_autotune_set_threads(api.KERNEL_MC, cases[0]["w"], cases[0]["h"], threads) == 0
    try:
        got = run_gpu(lib, cases)
    finally:
        lib.tcb_autotune_set_threads(api.KERNEL_MC, cases[0]["w"], cases[0]["h"], 0)
    for c, g in zip(cases, got):
        want = run_oracle(c)
        w, h = c["w"], c["h"]
        for k, (gp, wp) in enumerate(zip(g, want)):
            ww = w if k == 0 else w // 2
            assert np.array_equal(gp[:, :ww], wp), (w, h, c["pad"], k)
