"""Generates tests/golden/bench_1080p_gop4b.json: SHA-256 of the first
packets (coding order) the reference encoder emits for bench.py's
workload (1920x1080 GOP4 B, QP32, medium, profile 1, synthetic 'rects_lines'
source).  bench.py compares its own stream against these to report
bit-exactness.  Run from the repository root (needs oracle/_ref):
    python tests/golden/make_bench_golden.py
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

N_INPUT = 12   # inputs fed; GOP4 emits 9 packets for 12 inputs


def main():
    import bench
    from oracle import tcref
    from tcodec_b200 import api
    lib = tcref.ref_lib()
    enc = api.Encoder(lib, bench.make_cfg(lib))
    pk = []
    for f in bench.make_clip(N_INPUT):
        p = enc.encode(*f)
        if p is not None:
            pk.append(p)
    enc.close()
    out = {"inputs": N_INPUT, "packets": [hashlib.sha256(p).hexdigest() for p in pk],
           "sizes": [len(p) for p in pk]}
    json.dump(out, open(os.path.join(HERE, "bench_1080p_gop4b.json"), "w"), indent=1)
    print(out["sizes"])


if __name__ == "__main__":
    main()
