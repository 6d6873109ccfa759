"""The frame kernels' packed 16-bit lane routines (MC six-tap / bilinear,
deblocking work items, SAO band SSE) are __host__ __device__: this builds
them for the CPU with nvcc, together with the oracle's C restatement, and
checks them bit-exact against it (tests/packed_lanes_check.cu).  No GPU is
needed; the same routines run inside the sm_100a kernels, whose outputs the
gpu-marked tests compare with the oracle frame by frame."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        pytest.skip("nvcc not found")
    return path


def test_packed_lanes_match_oracle(tmp_path):
    exe = str(tmp_path / "packed_lanes_check")
    subprocess.run([nvcc(), "-std=c++17", "-O2", "-Wno-deprecated-gpu-targets", "-o", exe,
                    os.path.join(HERE, "packed_lanes_check.cu"), os.path.join(ROOT, "oracle", "tcoracle.c")],
                   check=True, timeout=300)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "mismatching samples 0" in r.stdout
