"""Host-side checks that need no GPU: the product library builds, loads and
exports every C entry point its headers declare; without a CUDA device the
encoder refuses to start instead of falling back to the CPU; seeded
sources are deterministic."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "tcodec_b200", "libtcodec_b200.so")


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    inline = set(re.findall(r"static\s+inline\s+[\w\s\*]*?\b(tcb?_[a-z0-9_]+)\s*\(", text))   # defined in the header
    return sorted(set(re.findall(r"\b(tcb?_[a-z0-9_]+)\s*\(", text)) - inline)


def _exported():
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_library_built_and_loads():
    assert os.path.exists(LIB), "run make -C tcodec_b200"
    from tcodec_b200 import api
    L = api.load_library()
    assert L.tc_version() == (0 << 16) | (1 << 8)


@pytest.mark.parametrize("header", ["tcodec.h", "tcodec_b200.h", "tcodec_b200_common.h"])
def test_every_declared_symbol_is_exported(header):
    names = _declared(header)
    assert names
    missing = [n for n in names if n not in _exported()]
    assert not missing, missing


def test_config_defaults_match_reference_values():
    from tcodec_b200 import api
    L = api.load_library()
    cfg = api.Config()
    L.tc_config_defaults(ctypes.byref(cfg), 1280, 720)
    assert (cfg.preset, cfg.rc_method, cfg.qp, cfg.fps_num, cfg.fps_den, cfg.keyframe_interval,
            cfg.bitstream_version, cfg.profile) == (2, 0, 32, 60, 1, 30, 1, 0)
    assert L.tc_error_string(-6) == b"Unknown error" or L.tc_error_string(-1) == b"Out of memory"


def test_invalid_configs_rejected():
    from tcodec_b200 import api
    L = api.load_library()
    cfg = api.make_config(L, 65, 64)
    assert not L.tc_encoder_create(ctypes.byref(cfg))          # odd width
    cfg = api.make_config(L, 64, 64)
    cfg.use_v2 = 0
    assert not L.tc_encoder_create(ctypes.byref(cfg))          # legacy v0/v1 not built


def test_no_cpu_fallback_without_device():
    """On a machine without a CUDA device, creation fails (NULL) instead of
    silently encoding on the host."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from tcodec_b200 import api
    L = api.load_library()
    cfg = api.make_config(L, 64, 64)
    assert not L.tc_encoder_create(ctypes.byref(cfg))


def test_synthetic_sources_deterministic():
    from tcodec_b200 import synth
    a = synth.moving_rects_clip(160, 96, 3)
    b = synth.moving_rects_clip(160, 96, 3)
    for fa, fb in zip(a, b):
        for pa, pb in zip(fa, fb):
            assert np.array_equal(pa, pb)
    assert a[0][0].shape == (96, 160) and a[0][1].shape == (48, 80)


def test_autotune_choice_table():
    """The frame-kernel autotuner's choice table (no GPU needed to read or
    record choices): valid variants per kernel, TMA staging for deblocking
    only, 0 clears, other sizes untouched; invalid variants are refused."""
    from tcodec_b200 import api
    L = api.bind_b200(api.load_library())
    w, h = 1234, 566
    assert L.tcb_autotune_threads(api.KERNEL_DEBLOCK, w, h) == 0
    for k, good, bad in ((api.KERNEL_DEBLOCK, [64, 128, 256, 64 | api.STAGING_TMA, 256 | api.STAGING_TMA], [32, 512]),
                         (api.KERNEL_SAO, [64, 128], [256, 128 | api.STAGING_TMA]),
                         (api.KERNEL_MC, [64, 128, 256], [96, 64 | api.STAGING_TMA])):
        for t in good:
            assert L.tcb_autotune_set_threads(k, w, h, t) == 0
            assert L.tcb_autotune_threads(k, w, h) == t
            assert L.tcb_autotune_threads(k, w + 2, h) == 0
        for t in bad:
            assert L.tcb_autotune_set_threads(k, w, h, t) == api.TC_ERR_PARAM
        assert L.tcb_autotune_set_threads(k, w, h, 0) == 0
        assert L.tcb_autotune_threads(k, w, h) == 0
    assert L.tcb_autotune_set_threads(7, w, h, 128) == api.TC_ERR_PARAM
    assert L.tcb_autotune_frame_kernels(w + 1, h, 4) == api.TC_ERR_PARAM     # odd width
    assert L.tcb_autotune_frame_kernels(w, h, 0) == api.TC_ERR_PARAM         # no frames


def test_engine_tuning_choice_table():
    """The engine autotuner's choice table (no GPU needed): defaults R = 4
    and diagonal order, every radius 2..5 and both orders recorded per frame
    size, other sizes untouched, invalid values refused, (0, 0) restores the
    defaults."""
    from tcodec_b200 import api
    L = api.bind_b200(api.load_library())
    w, h = 1922, 1084
    assert api.engine_tuning(L, w, h) == (4, api.QUEUE_DIAGONAL)
    for r in range(api.SEARCH_WINDOW_MIN, api.SEARCH_WINDOW_MAX + 1):
        for o in (api.QUEUE_DIAGONAL, api.QUEUE_STAGGERED):
            assert L.tcb_engine_set_tuning(w, h, r, o) == 0
            assert api.engine_tuning(L, w, h) == (r, o)
            assert api.engine_tuning(L, w + 2, h) == (4, api.QUEUE_DIAGONAL)
    for r, o in ((1, 0), (6, 0), (4, 2), (4, -1), (0, 1)):
        assert L.tcb_engine_set_tuning(w, h, r, o) == api.TC_ERR_PARAM, (r, o)
    assert L.tcb_engine_set_tuning(0, h, 4, 0) == api.TC_ERR_PARAM
    assert L.tcb_engine_get_tuning(w, h, None, None) == api.TC_ERR_PARAM
    assert L.tcb_engine_set_tuning(w, h, 0, 0) == 0
    assert api.engine_tuning(L, w, h) == (4, api.QUEUE_DIAGONAL)


def test_transform_dc_paths(tmp_path):
    """The reference's transform checks (test/test_tcodec.c:3074-3149) on
    the library's residual transforms and the DC-only helpers of
    include/tcodec_b200_common.h: DC gains, the +-2 round-trip bound, and
    exact DC-only parity for every DC in [-2000, 2000]."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    libdir = os.path.join(ROOT, "tcodec_b200")
    exe = str(tmp_path / "transform_dc_check")
    subprocess.run([cc, "-std=c99", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "transform_dc_check.c"), "-L", libdir, "-ltcodec_b200",
                    "-Wl,-rpath," + libdir, "-o", exe], check=True, timeout=120)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
