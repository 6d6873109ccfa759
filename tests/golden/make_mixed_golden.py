"""Generates tests/golden/mixed_streams.json: for every stream of the
mixed-resolution batched workload (synth.mixed_streams(): 64 streams,
32 frames, P-only, preset MEDIUM, profile 1) and for the first sessions of
the served workload (synth.served_sessions()), the SHA-256 over the
reference encoder's length-prefixed packets and the final reconstruction.
bench.py and the GPU tests compare against these digests.  Run from the
repository root (needs oracle/_ref; spawns one process per core):
    python tests/golden/make_mixed_golden.py [n_served]
    python tests/golden/make_mixed_golden.py --served-sample STOP STEP
The second form adds, to the existing file, the digests of a seeded sample
of the served schedule (sessions 0, STEP, 2 STEP, ... below STOP; key
"served_sample", by session index), which bench.py --served-sessions uses to
check a long served run without a reference run of every session.
"""
import hashlib
import json
import multiprocessing as mp
import os
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

PRESET, PROFILE = 2, 1


def stream_digest(lib, spec, frames):
    """(packet digest, final-recon digest, total bytes) of one P-only stream."""
    from tcodec_b200 import api
    cfg = api.make_config(lib, spec["w"], spec["h"], qp=spec["qp"], preset=PRESET, profile=PROFILE,
                          keyframe_interval=1000)
    enc = api.Encoder(lib, cfg)
    h = hashlib.sha256()
    total = 0
    try:
        for f in frames:
            p = enc.encode(*f)
            if p is not None:
                h.update(struct.pack("<I", len(p)) + p)
                total += len(p)
        for p in enc.flush():
            h.update(struct.pack("<I", len(p)) + p)
            total += len(p)
        r = hashlib.sha256()
        for pl in enc.recon():
            r.update(pl.tobytes())
    finally:
        enc.close()
    return h.hexdigest(), r.hexdigest(), total


def _work(item):
    kind, idx, spec = item
    from oracle import tcref
    from tcodec_b200 import synth
    lib = tcref.ref_lib()
    d, r, n = stream_digest(lib, spec, synth.stream_clip(spec))
    return kind, idx, dict(spec, digest=d, recon=r, bytes=n)


def served_sample(stop, step):
    from tcodec_b200 import synth
    path = os.path.join(HERE, "mixed_streams.json")
    out = json.load(open(path))
    sessions = synth.served_sessions()
    items = [("served_sample", j, sessions[j]) for j in range(0, stop, step)]
    items.sort(key=lambda it: -it[2]["w"] * it[2]["h"] * it[2]["frames"])
    sample = {}
    with mp.get_context("spawn").Pool(os.cpu_count()) as pool:
        for _, idx, rec in pool.imap_unordered(_work, items):
            sample[str(idx)] = rec
            print("served_sample", idx, rec["w"], rec["h"], rec["frames"], flush=True)
    out["served_sample"] = {k: sample[k] for k in sorted(sample, key=int)}
    json.dump(out, open(path, "w"), indent=0)


def main():
    from tcodec_b200 import synth
    if len(sys.argv) > 1 and sys.argv[1] == "--served-sample":
        served_sample(int(sys.argv[2]), int(sys.argv[3]))
        return
    n_served = int(sys.argv[1]) if len(sys.argv) > 1 else 64
    items = [("batch", i, s) for i, s in enumerate(synth.mixed_streams())]
    items += [("served", j, s) for j, s in enumerate(synth.served_sessions()[:n_served])]
    # longest first keeps the pool busy to the end
    items.sort(key=lambda it: -it[2]["w"] * it[2]["h"] * it[2]["frames"])
    out = {"preset": PRESET, "profile": PROFILE, "batch": [None] * 64, "served": [None] * n_served}
    with mp.get_context("spawn").Pool(os.cpu_count()) as pool:
        for kind, idx, rec in pool.imap_unordered(_work, items):
            out[kind][idx] = rec
            print(kind, idx, rec["w"], rec["h"], rec["frames"], flush=True)
    json.dump(out, open(os.path.join(HERE, "mixed_streams.json"), "w"), indent=0)


if __name__ == "__main__":
    main()
