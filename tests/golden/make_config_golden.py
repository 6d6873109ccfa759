"""Generates tests/golden/configs_v2.json: the reference encoder's packets
(SHA-256 and sizes) and final reconstruction digest for the two
single-stream workloads at their full length, as this repository declares
them for parity (preset MEDIUM, P-only, keyframe interval above the clip):
  cfg0  320x240, 30 frames, QP 32, profile 0 (1 searched reference),
        sinusoid source (synth.workload("sinusoid"))
  cfg1  1280x720, 60 frames, QP 27, profile 1 (2 searched references),
        sinusoid + moving rectangles (synth.workload("rects"))
  cfg2  1920x1080, 120 frames, QP 32, profile 1, GOP4 hierarchical B
        frames, rectangles + 1-px lines (synth.workload("rects_lines"))
Run from the repository root (needs oracle/_ref; cfg2 alone is about 20
minutes of one CPU core, the configurations run in parallel):
    python tests/golden/make_config_golden.py [name ...]
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

OUT = os.path.join(HERE, "configs_v2.json")
CONFIGS = {   # name: (workload, width, height, frames, qp, profile, B frames)
    "cfg0": ("sinusoid", 320, 240, 30, 32, 0, False),
    "cfg1": ("rects", 1280, 720, 60, 27, 1, False),
    "cfg2": ("rects_lines", 1920, 1080, 120, 32, 1, True),
}


def run(lib, name, entropy_threads=None):
    """Encode configuration `name` with `lib`; `entropy_threads` (B200
    library only) sets the encoder's host threads for entry-point rows."""
    from tcodec_b200 import api, synth
    from tests.golden.make_pframe_golden import digest_planes
    wl, w, h, n, qp, prof, bf = CONFIGS[name]
    cfg = api.make_config(lib, w, h, qp=qp, preset=api.PRESET_MEDIUM, profile=prof, keyframe_interval=1000,
                          b_frames=bf)
    enc = api.Encoder(lib, cfg)
    if entropy_threads is not None:
        lib.tcb_encoder_set_entropy_threads(enc.h, entropy_threads)
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


def _run_ref(name):
    from oracle import tcref
    return name, run(tcref.ref_lib(), name)


def main():
    import multiprocessing as mp
    names = sys.argv[1:] or list(CONFIGS)
    out = json.load(open(OUT)) if os.path.exists(OUT) else {}
    with mp.get_context("spawn").Pool(len(names)) as pool:
        for name, res in pool.imap_unordered(_run_ref, names):
            out[name] = {"config": list(CONFIGS[name]), **res}
            print(name, sum(out[name]["sizes"]), "bytes", flush=True)
    with open(OUT, "w") as f:
        json.dump({k: out[k] for k in sorted(out)}, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
