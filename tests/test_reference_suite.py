"""The reference's own C regression tests (its test/test_tcodec.c).

The whole suite (53 tests in its fast mode: the default-configuration
legacy v1 encodes and decodes, v0 / v1 / v2 bitstreams, presets, B-frames,
malformed-stream fuzzing, the range coder, transforms, SAO) runs as the
reference builds it, linked with the reference's objects on the CPU and
with libtcodec_b200.so on the GPU (oracle/Makefile `suite`).

The v2 bitstream and the modules beneath it also run alone, through
tests/reference_suite_v2.c:

* linked with the reference library's objects, on the CPU: the harness and
  the selection of tests are sound (every selected test passes on the
  reference itself);
* linked with libtcodec_b200.so, on the GPU: the same tests pass with this
  library behind the reference's API (multiref, CfL, B-frame GOP order with
  bit-exact decode, quadtree round trip, fast / medium replay parity, the
  systematic malformed-stream fuzz, SAO band offset, range coder and
  transform round trips).
"""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
N_TESTS = 16
N_FULL = 53


def _run(binary):
    path = os.path.join(REF, binary)
    if not os.path.exists(path):
        pytest.skip(f"oracle/_ref/{binary} not built (make -C oracle suite)")
    out = subprocess.run([path], capture_output=True, text=True, timeout=1200,
                         env=dict(os.environ, TCODEC_TEST_FAST="1"))
    m = re.search(r"Results: (\d+)/(\d+) passed", out.stdout)
    assert m, out.stdout[-2000:] + out.stderr[-2000:]
    return out.returncode, int(m.group(1)), int(m.group(2)), out.stdout


def test_reference_suite_on_reference_library():
    rc, passed, run, log = _run("test_v2_suite_ref")
    assert (rc, passed, run) == (0, N_TESTS, N_TESTS), log[-3000:]


@pytest.mark.gpu
def test_reference_suite_on_b200_library():
    rc, passed, run, log = _run("test_v2_suite_b200")
    assert (rc, passed, run) == (0, N_TESTS, N_TESTS), log[-3000:]


def test_full_reference_suite_on_reference_library():
    rc, passed, run, log = _run("test_tcodec_ref")
    assert (rc, passed, run) == (0, N_FULL, N_FULL), log[-3000:]


@pytest.mark.gpu
def test_full_reference_suite_on_b200_library():
    rc, passed, run, log = _run("test_tcodec_b200")
    assert (rc, passed, run) == (0, N_FULL, N_FULL), log[-3000:]
