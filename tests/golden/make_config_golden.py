"""Generates tests/golden/configs_v2.json: the reference encoder's packets
(SHA-256 and sizes) and final reconstruction digest for the two
single-stream workloads at their full length, as this repository declares
them for parity (preset MEDIUM, P-only, keyframe interval above the clip):
  cfg0  320x240, 30 frames, QP 32, profile 0 (1 searched reference),
        sinusoid source (synth.workload("sinusoid"))
  cfg1  1280x720, 60 frames, QP 27, profile 1 (2 searched references),
        sinusoid + moving rectangles (synth.workload("rects"))
Run from the repository root (needs oracle/_ref, a few CPU minutes):
    python tests/golden/make_config_golden.py
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

OUT = os.path.join(HERE, "configs_v2.json")
CONFIGS = {   # name: (workload, width, height, frames, qp, profile)
    "cfg0": ("sinusoid", 320, 240, 30, 32, 0),
    "cfg1": ("rects", 1280, 720, 60, 27, 1),
}


def run(lib, name):
    from tcodec_b200 import api, synth
    from tests.golden.make_pframe_golden import digest_planes
    wl, w, h, n, qp, prof = CONFIGS[name]
    cfg = api.make_config(lib, w, h, qp=qp, preset=api.PRESET_MEDIUM, profile=prof, keyframe_interval=1000)
    enc = api.Encoder(lib, cfg)
    pk = []
    try:
        for f in synth.workload(wl, frames=n):
            p = enc.encode(*f)
            if p is not None:
                pk.append(p)
        pk.extend(enc.flush())
        recon = digest_planes(enc.recon())
    finally:
        enc.close()
    return {"packets": [hashlib.sha256(p).hexdigest() for p in pk], "sizes": [len(p) for p in pk],
            "final_recon": recon}


def main():
    from oracle import tcref
    lib = tcref.ref_lib()
    out = {}
    for name in CONFIGS:
        out[name] = {"config": list(CONFIGS[name]), **run(lib, name)}
        print(name, sum(out[name]["sizes"]), "bytes", flush=True)
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
