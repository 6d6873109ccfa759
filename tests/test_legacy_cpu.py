"""CPU check of the legacy (v0 / v1) block path's device source.

tests/legacy_emu.cpp compiles tcodec_b200/csrc/tcb_legacy.cuh as plain C++
(a team of one lane) with the library's host syntax writer and links the
reference encoder from its own sources (oracle/_ref/obj, built by
`make -C oracle ref`).  These tests run it over a configuration matrix and
over the reference's 72 legacy conformance streams; in the matrix every
reference packet is also decoded with the library's host parser
(tcb_parse.h) and the same source's reconstruction and compared with the
reference decoder.  The GPU tests (test_gpu_legacy.py) then check the same
source on the device.
"""
import glob
import hashlib
import os
import subprocess

import pytest

from tests.golden import make_golden as golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_OBJS = sorted(glob.glob(os.path.join(ROOT, "oracle", "_ref", "obj", "*.o")))


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    if not REF_OBJS:
        pytest.skip("reference objects oracle/_ref/obj not built (make -C oracle ref)")
    exe = str(tmp_path_factory.mktemp("legacy") / "legacy_emu")
    subprocess.run(["g++", "-O2", "-std=c++17", "-w", "-o", exe, os.path.join(ROOT, "tests", "legacy_emu.cpp"),
                    os.path.join(ROOT, "tcodec_b200", "csrc", "tcb_entropy.cpp")] + REF_OBJS + ["-lm", "-lpthread"],
                   check=True)
    return exe


MATRIX = [
    # W H frames qp preset version entropy crc threads profile seed
    "128 128 6 22 2 0 0 0 0 0 1",
    "128 128 6 42 2 1 0 1 0 0 2",
    "128 128 6 32 2 1 1 1 0 0 3",
    "96 80 6 32 1 1 0 0 0 0 4",
    "320 240 4 27 3 1 1 0 0 1 5",
    "320 240 4 27 3 1 0 0 0 1 6",
    "100 60 5 32 0 1 0 0 0 0 7",
    "104 72 5 12 2 1 1 1 1 0 8",
    "200 136 33 37 2 1 0 0 0 0 9",
    "64 64 4 50 3 0 0 0 4 2 10",
]


@pytest.mark.parametrize("args", MATRIX)
def test_sequence_matches_reference(emu, args):
    r = subprocess.run([emu] + args.split(), capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("identical")


def test_legacy_golden_hashes(emu, tmp_path):
    rows = golden.load(golden.OUT_LEGACY)
    assert len(rows) == 72
    yuv, out = str(tmp_path / "clip.yuv"), str(tmp_path / "out.tcv")
    bad = []
    for (digest, name, pat, w, h, qp, var) in rows:
        y, cb, cr = golden.clip(pat, w, h)
        with open(yuv, "wb") as f:
            f.write(y + cb + cr)
        kw = golden.LEGACY_VARIANTS[var]
        r = subprocess.run([emu, str(w), str(h), "1", str(qp), "2", str(kw["version"]),
                            "1" if kw["entropy"] else "0", "0", "0", "0", "1", yuv, out],
                           capture_output=True, text=True, timeout=120)
        with open(out, "rb") as f:
            d = hashlib.sha256(f.read()).hexdigest()
        if r.returncode != 0 or d != digest:
            bad.append(name)
    assert not bad, bad
