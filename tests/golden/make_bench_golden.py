"""Generates tests/golden/bench_1080p_gop4b.json: what the reference encoder
emits for bench.py's workload (1920x1080 GOP4 B, QP32, medium, profile 1,
synthetic 'rects_lines' source):

  packets / sizes   SHA-256 and length of the first packets (coding order)
                    of one stream fed clip frames 0..11 (GOP4 emits 9
                    packets for 12 inputs);
  streams           for every one of the bench's STREAMS streams, the
                    digest of its whole packet sequence when stream s is fed
                    clip frames s .. s + INPUTS - 1 and then flushed, which
                    is exactly what bench.py's batched run encodes with
                    --warmup W --steps K, W + K = INPUTS (the defaults:
                    5 + 20).  The digest is SHA-256 over every packet
                    prefixed by its 4-byte little-endian length.

bench.py compares every stream of its own run against `streams`.  Run from
the repository root (needs oracle/_ref; about 15 minutes on 8 cores):
    python tests/golden/make_bench_golden.py [--procs N]
"""
import argparse
import hashlib
import json
import multiprocessing as mp
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "bench_1080p_gop4b.json")
N_INPUT = 12     # prefix check of stream 0
STREAMS = 32     # bench.py's default streams per GPU
INPUTS = 25      # bench.py's default warm-up + steps


def stream_digest(packets):
    h = hashlib.sha256()
    for p in packets:
        h.update(len(p).to_bytes(4, "little") + p)
    return h.hexdigest()


def _encode_stream(s):
    import bench
    from oracle import tcref
    from tcodec_b200 import api
    lib = tcref.ref_lib()
    frames = bench.make_clip(s + INPUTS)[s:s + INPUTS]
    pk = api.encode_sequence(lib, bench.make_cfg(lib), frames)
    return s, stream_digest(pk), len(pk)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--procs", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
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
    with mp.get_context("spawn").Pool(args.procs) as pool:
        res = sorted(pool.map(_encode_stream, range(STREAMS), chunksize=1))
    out["streams"] = {"inputs": INPUTS, "count": STREAMS, "digests": [r[1] for r in res],
                      "packets": [r[2] for r in res],
                      "what": "stream s: clip frames s .. s+inputs-1, then flushed; SHA-256 over length-prefixed "
                              "packets"}
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print(out["sizes"], [r[2] for r in res])


if __name__ == "__main__":
    main()
