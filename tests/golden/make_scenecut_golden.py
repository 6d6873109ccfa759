"""Generates tests/golden/scenecut_v2.json: the reference encoder's packets
(SHA-256, sizes, key-frame flags) and final reconstruction digest for
P-only clips with hard scene cuts, so the encoder's scene-cut keyframe
decision is exercised (reference src/encoder.c:2650-2679: chi-square
distance of 16-bin luma histograms of consecutive source frames against
SCENE_CUT_THRESHOLD 0.5, src/encoder.c:161).

Each clip switches between two scenes: A, moving rectangles over the
sinusoid background, and B, a different sinusoid texture with its luma
compressed to the dark quarter of the range (so the histograms of A and B
barely overlap and the distance is far above the threshold).

Run from the repository root (needs oracle/_ref, about a minute):
    python tests/golden/make_scenecut_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

OUT = os.path.join(HERE, "scenecut_v2.json")
# name: (width, height, frames, scene of each frame, qp, profile)
CASES = {
    "cut320": (320, 240, 8, "AAAABBBB", 32, 0),
    "cut720": (1280, 720, 8, "AAABBBAA", 27, 1),
}


def clip(name):
    """Frames of a scene-cut case: scene A frames are frame i of the moving
    rectangles clip, scene B frames frame i of a second sinusoid clip whose
    luma is mapped to 16 + y / 4."""
    from tcodec_b200 import synth
    w, h, n, scenes, _, _ = CASES[name]
    a = synth.moving_rects_clip(w, h, n, seed_rects=31, seed_noise=32)
    b = synth.sinusoid_clip(w, h, n, motion=(-1.5, 1.0), seed_luma=41, seed_chroma=42, seed_noise=43)
    out = []
    for i, sc in enumerate(scenes):
        if sc == "A":
            out.append(a[i])
        else:
            y, cb, cr = b[i]
            out.append(((16 + y.astype(np.int32) // 4).astype(np.uint8), cb, cr))
    return out


def run(lib, name):
    """Packets, key-frame flags and final reconstruction of one case."""
    from tcodec_b200 import api
    from tests.golden.make_pframe_golden import digest_planes
    w, h, n, scenes, qp, prof = CASES[name]
    cfg = api.make_config(lib, w, h, qp=qp, preset=api.PRESET_MEDIUM, profile=prof, keyframe_interval=1000)
    enc = api.Encoder(lib, cfg)
    pk, keys = [], []
    try:
        for f in clip(name):
            pk.append(enc.encode(*f))
            keys.append(enc.last_key_frame)
        recon = digest_planes(enc.recon())
    finally:
        enc.close()
    return {"packets": [hashlib.sha256(p).hexdigest() for p in pk], "sizes": [len(p) for p in pk],
            "key_frames": keys, "final_recon": recon}


def main():
    from oracle import tcref
    lib = tcref.ref_lib()
    out = {}
    for name in CASES:
        out[name] = {"case": list(CASES[name]), **run(lib, name)}
        print(name, out[name]["key_frames"], out[name]["sizes"], flush=True)
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
