"""Counters of the CTU engine on the batched 1080p GOP4-B workload, read
from the profiling build (`make -C tcodec_b200 prof`, which compiles the
same kernels with -DTCB_PHASE_PROFILE):

* per-phase cycles of each CTU (thread 0's clock64 deltas summed over CTUs);
* each CTA's residency and the cycles it waited for a left or above
  neighbour's publish flag;
* work counts: integer-search SAD pixel differences, quarter-sample SAD
  pixels, and 8x8 / 4x4 transform units coded.  The encode is deterministic,
  so these counts hold for the production build too.

    python -m tcodec_b200.profile_engine --streams 32 --ops-out profiles/ctu_engine_ops.txt

Needs a CUDA device.  The profiling counters slow the engine: its timings
are for shares, not for throughput."""
import argparse
import ctypes
import json
import os
import time

from . import api, synth

PHASES = ["refs/mvp", "ME", "MC", "resid jobs", "skip chk", "scan", "CfL", "replay", "decide(total)",
          "write pass", "deblock+sao", "me0:int", "me0:subpel"]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--streams", type=int, default=32)
    ap.add_argument("--steps", type=int, default=12)
    ap.add_argument("--ops-out", default=None, help="write the per-frame work counts (JSON) here")
    args = ap.parse_args()
    lib = api.load_library(os.path.join(os.path.dirname(os.path.abspath(__file__)), "libtcodec_b200_prof.so"))
    lib.tcb_debug_phase_cycles.argtypes = [ctypes.c_void_p]
    lib.tcb_debug_op_counts.argtypes = [ctypes.c_void_p]
    S, W, H = args.streams, 1920, 1080
    clip = synth.workload("rects_lines", frames=12)
    cfgs = [api.make_config(lib, W, H, qp=32, preset=api.PRESET_MEDIUM, profile=1, keyframe_interval=1000,
                            b_frames=True) for _ in range(S)]
    batch = api.BatchEncoder(lib, cfgs)
    cyc, ops = (ctypes.c_ulonglong * 16)(), (ctypes.c_ulonglong * 4)()
    tot, steady = [0, 0, 0, 0], 0
    for t in range(args.steps):
        t0 = time.time()
        pk = batch.encode([clip[(t + s) % len(clip)] for s in range(S)])
        dt = time.time() - t0
        lib.tcb_debug_phase_cycles(cyc)
        lib.tcb_debug_op_counts(ops)
        coded = sum(p is not None for p in pk)
        enc = cyc[8] + cyc[9] + cyc[10]
        print(f"step {t} {dt * 1000:.0f} ms, {coded} frames: residency {cyc[14] / 1e9:.2f} Gcyc, encode "
              f"{100 * enc / max(1, cyc[14]):.1f} %, neighbour wait {100 * cyc[13] / max(1, cyc[14]):.1f} %; "
              f"int SAD px {ops[0] / 1e9:.3f} G, qpel SAD px {ops[1] / 1e9:.3f} G, "
              f"TU8 {ops[2] / 1e6:.2f} M, TU4 {ops[3] / 1e6:.2f} M")
        if t == args.steps - 1:
            for i, n in enumerate(PHASES):
                print(f"   {n:14s} {cyc[i] / 1e6:10.1f} Mcyc  {100 * cyc[i] / max(1, enc):5.1f} %")
        if t >= 4 and coded == S:          # steady GOP4-B steps (after the first anchor)
            steady += 1
            for i in range(4):
                tot[i] += ops[i]
    batch.close()
    per_frame = {k: tot[i] / max(1, steady * S) for i, k in enumerate(("int_sad_px", "qpel_sad_px", "tu8", "tu4"))}
    print("per frame:", json.dumps(per_frame))
    if args.ops_out:
        out = {"workload": f"1920x1080 GOP4-B, CQP 32, preset medium, profile 1, {S} streams, "
                           f"mean over {steady} steady steps",
               "per_frame": per_frame,
               "int32_lanes_per_sm_clock": 64,
               "peak_note": "integer peak taken as 64 INT32 lane operations per SM per clock (half the 128 "
                            "FP32 lanes), an assumption; a packed SAD (vsadu4) counts 4 byte differences",
               "command": "python -m tcodec_b200.profile_engine --streams %d --ops-out <file>" % S}
        with open(args.ops_out, "w") as f:
            f.write(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
