"""Builds tests/golden/golden_v2.sha256 and provides the golden clips.

The reference commits SHA-256 hashes of its conformance streams
(golden/MANIFEST.sha256, produced by its tools/gen_golden.sh).  This
script copies the v2 lines of that manifest (v2 raw, v2e range coded,
v2m profile-1 multiref syntax, v2b B-frame stream) into
tests/golden/golden_v2.sha256, so the hashes travel without the reference
tree.  `clip()` regenerates each one-frame test pattern with the same
per-pixel rules as the reference generator (gradient, checkerboard,
per-pixel-seeded noise from Python's `random`, line patterns; chroma 128).

Run from the repository root:  python tests/golden/make_golden.py [REFERENCE_TREE | MANIFEST]
(default: the tree oracle/Makefile reads, `make -s -C oracle refdir`).
"""
import os
import random
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "golden_v2.sha256")
OUT_LEGACY = os.path.join(HERE, "golden_legacy.sha256")


def reference_manifest() -> str:
    if len(sys.argv) > 1:
        if os.path.isfile(sys.argv[1]):      # a manifest file given directly
            return sys.argv[1]
        ref = sys.argv[1]
    else:
        root = os.path.dirname(os.path.dirname(HERE))
        ref = subprocess.run(["make", "-s", "-C", os.path.join(root, "oracle"), "refdir"], check=True,
                             capture_output=True, text=True).stdout.strip()
    return os.path.join(ref, "golden", "MANIFEST.sha256")

PATTERNS = {"gradient", "checkerboard", "noise", "hlines", "vlines", "diagonal"}
# tcenc flags of each variant (reference tools/gen_golden.sh:111-147).
VARIANTS = {
    "v2": dict(entropy=True, profile=0, b_frames=False),
    "v2e": dict(entropy=True, profile=0, b_frames=False),
    "v2m": dict(entropy=True, profile=1, b_frames=False),
    "v2b": dict(entropy=True, profile=1, b_frames=True),
}
# Legacy 8x8 block syntax (tools/gen_golden.sh:87-111): `--bs-version 0`,
# `--bs-version 1`, `--bs-version 1 --entropy`; default worker count.
LEGACY_VARIANTS = {
    "v0": dict(version=0, entropy=False),
    "v1": dict(version=1, entropy=False),
    "v1e": dict(version=1, entropy=True),
}


def clip(pattern: str, w: int, h: int):
    """One frame of a golden pattern as (y, cb, cr) bytes."""
    y = bytearray()
    for row in range(h):
        for col in range(w):
            if pattern == "gradient":
                v = (row * 255 // h + col * 255 // w) // 2
            elif pattern == "checkerboard":
                v = 255 if ((col // 16) + (row // 16)) % 2 else 0
            elif pattern == "noise":
                random.seed(row * w + col)
                v = random.randint(0, 255)
            elif pattern == "hlines":
                v = 255 if row % 16 < 8 else 0
            elif pattern == "vlines":
                v = 255 if col % 16 < 8 else 0
            elif pattern == "diagonal":
                v = 255 if (row + col) % 32 < 16 else 0
            else:
                v = 128
            y.append(v)
    c = bytes([128]) * ((w // 2) * (h // 2))
    return bytes(y), c, c


def parse_name(name: str):
    """'gradient_96x80_qp32_v2m.tcv' -> ('gradient', 96, 80, 32, 'v2m')."""
    stem = name[:-4]
    parts = stem.split("_")
    pat, dims, qp, var = parts[0], parts[1], parts[2], parts[3]
    w, h = (int(v) for v in dims.split("x"))
    return pat, w, h, int(qp[2:]), var


def load(path: str = OUT):
    """[(sha256, name, pattern, w, h, qp, variant)] from golden_v2.sha256
    (or the legacy file)."""
    out = []
    with open(path) as f:
        for line in f:
            digest, name = line.split()
            out.append((digest, name) + parse_name(name))
    return out


def main():
    src = reference_manifest()
    lines, legacy = [], []
    with open(src) as f:
        for line in f:
            digest, name = line.split()
            if not name.endswith(".tcv"):
                continue
            var = name[:-4].split("_")[-1]
            if var in VARIANTS:
                lines.append(f"{digest}  {name}\n")
            elif var in LEGACY_VARIANTS:
                legacy.append(f"{digest}  {name}\n")
    for path, ls in ((OUT, lines), (OUT_LEGACY, legacy)):
        with open(path, "w") as f:
            f.writelines(ls)
        print(f"wrote {len(ls)} hashes to {path}")


if __name__ == "__main__":
    main()
