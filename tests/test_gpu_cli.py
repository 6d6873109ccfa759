"""The reference's own command-line tools driving this library: tcenc and
tcdec compiled from the reference sources and linked against
libtcodec_b200 (oracle/Makefile `suite`) must write the same .tcv and .yuv
files as the same tools linked against the reference library, for a P-only
and a GOP4 B-frame clip."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
TOOLS = ["tcenc", "tcdec", "tcenc_b200", "tcdec_b200"]


@pytest.mark.skipif(not all(os.path.exists(os.path.join(REF, t)) for t in TOOLS),
                    reason="oracle/_ref tools not built (make -C oracle ref suite)")
@pytest.mark.parametrize("extra", [[], ["-b"]], ids=["p_only", "gop4_b"])
def test_reference_cli_through_library(tmp_path, extra):
    from tcodec_b200 import synth
    w, h, n = 320, 240, 9
    yuv = tmp_path / "in.yuv"
    with open(yuv, "wb") as f:
        for y, cb, cr in synth.moving_rects_clip(w, h, n):
            f.write(np.ascontiguousarray(y).tobytes() + cb.tobytes() + cr.tobytes())
    args = ["-w", str(w), "-h", str(h), "-q", "30", "-p", "2", "--profile", "1", "-k", "1000", "--v2"] + extra
    out = {}
    for suffix in ("", "_b200"):
        tcv = tmp_path / f"out{suffix}.tcv"
        dec = tmp_path / f"dec{suffix}.yuv"
        subprocess.run([os.path.join(REF, "tcenc" + suffix)] + args + ["-o", str(tcv), str(yuv)], check=True,
                       stdout=subprocess.DEVNULL, timeout=600)
        subprocess.run([os.path.join(REF, "tcdec" + suffix), str(tcv), str(dec)], check=True,
                       stdout=subprocess.DEVNULL, timeout=600)
        out[suffix] = (tcv.read_bytes(), dec.read_bytes())
    assert len(out[""][0]) > 0 and out["_b200"][0] == out[""][0], "tcenc output differs"
    assert len(out[""][1]) == w * h * 3 // 2 * n and out["_b200"][1] == out[""][1], "tcdec output differs"
