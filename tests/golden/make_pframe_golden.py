"""Generates tests/golden/pframes_v2.json: known answers for P-frame (and
B-frame) v2 streams, produced by the reference encoder (oracle/_ref) on the
seeded synthetic sources of tcodec_b200.synth.

The reference repository pins only one-frame (keyframe) streams, so these
hashes are the inter-frame pins: per case the SHA-256 of every packet and
of the final reconstruction.  Regenerate from the repository root with
    python tests/golden/make_pframe_golden.py
(needs oracle/_ref built from the reference tree).
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "pframes_v2.json")

# (id, source, W, H, frames, qp, preset, profile, keyint, entropy, crc, b_frames)
CASES = [
    ("sin320_q32_med", "sin", 320, 240, 6, 32, 2, 0, 1000, 1, 0, 0),
    ("rect320_q27_med_mref", "rect", 320, 240, 6, 27, 2, 1, 1000, 1, 0, 0),
    ("rect320_q27_fast", "rect", 320, 240, 5, 27, 1, 1, 1000, 1, 0, 0),
    ("rect256x136_q37_slow_crc", "rect", 256, 136, 4, 37, 3, 1, 1000, 1, 1, 0),
    ("rect192x128_q22_raw", "rect", 192, 128, 4, 22, 2, 1, 1000, 0, 0, 0),
    ("sin96x80_q42_ufast", "sin", 96, 80, 5, 42, 0, 0, 1000, 1, 0, 0),
    ("rect320_q32_kint3", "rect", 320, 240, 7, 32, 2, 1, 3, 1, 0, 0),
    ("rect640x360_q32_med_mref", "rect", 640, 360, 3, 32, 2, 1, 1000, 1, 0, 0),
    ("rect320_q32_gop4b", "rect", 320, 240, 9, 32, 2, 1, 1000, 1, 0, 1),
    ("sin128_q27_gop4b_tail", "sin", 128, 128, 6, 27, 2, 1, 1000, 1, 0, 1),
]


def source(kind, w, h, n):
    from tcodec_b200 import synth
    return synth.sinusoid_clip(w, h, n) if kind == "sin" else synth.moving_rects_clip(w, h, n)


def digest_planes(planes):
    h = hashlib.sha256()
    for p in planes:
        h.update(p.tobytes())
    return h.hexdigest()


def run_case(lib, case):
    from tcodec_b200 import api
    cid, kind, w, h, n, qp, preset, prof, kint, ent, crc, b = case
    cfg = api.make_config(lib, w, h, qp=qp, preset=preset, profile=prof, keyframe_interval=kint,
                          entropy=bool(ent), crc=bool(crc), b_frames=bool(b))
    enc = api.Encoder(lib, cfg)
    pkts = []
    try:
        for f in source(kind, w, h, n):
            p = enc.encode(*f)
            if p is not None:
                pkts.append(p)
        pkts.extend(enc.flush())
        recon = digest_planes(enc.recon())
    finally:
        enc.close()
    return {"packets": [hashlib.sha256(p).hexdigest() for p in pkts],
            "sizes": [len(p) for p in pkts], "final_recon": recon}


def main():
    from oracle import tcref
    lib = tcref.ref_lib()
    out = {}
    for case in CASES:
        out[case[0]] = {"case": list(case[1:]), **run_case(lib, case)}
        print(case[0], out[case[0]]["sizes"])
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
