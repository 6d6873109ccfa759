"""ctypes binding of the TCodec C API (include/tcodec.h).

The same binding drives any library that exports the reference's
include/tcodec.h ABI: libtcodec_b200.so (this package's CUDA build) or the
reference C library built by oracle/Makefile for checking.  The product
path is libtcodec_b200.so; `load_library()` raises if it is missing, there is
no fallback.
"""
from __future__ import annotations

import ctypes
import os
from typing import List, Optional, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtcodec_b200.so")

TC_OK, TC_ERR_MEMORY, TC_ERR_PARAM, TC_ERR_BITSTREAM, TC_ERR_EOF, TC_ERR_INTERNAL, TC_ERR_NEED_MORE = (
    0, -1, -2, -3, -4, -5, -6)
PRESET_ULTRAFAST, PRESET_FAST, PRESET_MEDIUM, PRESET_SLOW = 0, 1, 2, 3


class Config(ctypes.Structure):
    """tc_config_t (reference include/tcodec_types.h:333-355)."""
    _fields_ = [
        ("width", ctypes.c_int32), ("height", ctypes.c_int32),
        ("preset", ctypes.c_int), ("rc_method", ctypes.c_int),
        ("qp", ctypes.c_int32), ("target_bitrate", ctypes.c_int32),
        ("fps_num", ctypes.c_int32), ("fps_den", ctypes.c_int32),
        ("keyframe_interval", ctypes.c_int32), ("threads", ctypes.c_int32),
        ("tile_cols", ctypes.c_int32), ("tile_rows", ctypes.c_int32),
        ("bitstream_version", ctypes.c_uint8), ("profile", ctypes.c_uint8),
        ("level_idx", ctypes.c_uint8),
        ("enable_crc", ctypes.c_int), ("enable_entropy_coded", ctypes.c_int),
        ("enable_b_frames", ctypes.c_int), ("use_v2", ctypes.c_int),
    ]


class Packet(ctypes.Structure):
    """tc_packet_t (reference include/tcodec_types.h:324-329)."""
    _fields_ = [("data", ctypes.POINTER(ctypes.c_uint8)), ("size", ctypes.c_size_t),
                ("pts", ctypes.c_int64), ("key_frame", ctypes.c_int)]


class FrameBuf(ctypes.Structure):
    """tc_frame_buf_t (reference include/tcodec_types.h:309-320)."""
    _fields_ = [("y", ctypes.POINTER(ctypes.c_uint8)), ("cb", ctypes.POINTER(ctypes.c_uint8)),
                ("cr", ctypes.POINTER(ctypes.c_uint8)), ("stride_y", ctypes.c_int32),
                ("stride_c", ctypes.c_int32), ("width", ctypes.c_int32), ("height", ctypes.c_int32),
                ("poc", ctypes.c_int32), ("qp_avg", ctypes.c_uint8), ("owned", ctypes.c_int)]


class EncoderHead(ctypes.Structure):
    """Leading members of tc_encoder_t shared by both implementations
    (reference include/tcodec_common.h:609-612)."""
    _fields_ = [("cfg", Config), ("cur", ctypes.POINTER(FrameBuf)), ("recon", ctypes.POINTER(FrameBuf))]


def bind(lib: ctypes.CDLL) -> ctypes.CDLL:
    """Attach argtypes/restype of the include/tcodec.h entry points."""
    P = ctypes.POINTER
    u8p = P(ctypes.c_uint8)
    lib.tc_config_defaults.argtypes = [P(Config), ctypes.c_int32, ctypes.c_int32]
    lib.tc_config_defaults.restype = None
    lib.tc_encoder_create.argtypes = [P(Config)]
    lib.tc_encoder_create.restype = ctypes.c_void_p
    lib.tc_encoder_destroy.argtypes = [ctypes.c_void_p]
    lib.tc_encoder_destroy.restype = None
    lib.tc_encoder_encode.argtypes = [ctypes.c_void_p, u8p, ctypes.c_int, u8p, ctypes.c_int, u8p,
                                      ctypes.c_int, P(Packet)]
    lib.tc_encoder_encode.restype = ctypes.c_int
    lib.tc_encoder_flush_tail.argtypes = [ctypes.c_void_p, P(Packet)]
    lib.tc_encoder_flush_tail.restype = ctypes.c_int
    lib.tc_encoder_force_keyframe.argtypes = [ctypes.c_void_p]
    lib.tc_encoder_force_keyframe.restype = None
    lib.tc_encoder_get_stats.argtypes = [ctypes.c_void_p, P(ctypes.c_int64), P(ctypes.c_int32),
                                         P(ctypes.c_double)]
    lib.tc_encoder_get_stats.restype = None
    lib.tc_error_string.argtypes = [ctypes.c_int]
    lib.tc_error_string.restype = ctypes.c_char_p
    return lib


_lib: Optional[ctypes.CDLL] = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libtcodec_b200.so (RTLD_LOCAL so it can sit next to the
    reference library in one process).  Raises if the build is missing."""
    global _lib
    if path == LIB_PATH and _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is not built; run `make -C tcodec_b200` (no CPU fallback exists)")
    lib = bind(ctypes.CDLL(path, mode=os.RTLD_LOCAL | os.RTLD_NOW))
    if path == LIB_PATH:
        _lib = lib
    return lib


def make_config(lib: ctypes.CDLL, width: int, height: int, qp: int = 32, preset: int = PRESET_MEDIUM,
                profile: int = 0, keyframe_interval: int = 30, entropy: bool = True,
                b_frames: bool = False, crc: bool = False) -> Config:
    """tc_config_defaults + the fields `tcenc --v2` sets (reference
    tools/tcenc.c:127-185)."""
    cfg = Config()
    lib.tc_config_defaults(ctypes.byref(cfg), width, height)
    cfg.preset = preset
    cfg.qp = qp
    cfg.keyframe_interval = keyframe_interval
    cfg.profile = profile
    cfg.use_v2 = 1
    cfg.enable_entropy_coded = 1 if entropy else 0
    cfg.enable_b_frames = 1 if b_frames else 0
    cfg.enable_crc = 1 if crc else 0
    return cfg


class Encoder:
    """One v2 encode session through the C ABI."""

    def __init__(self, lib: ctypes.CDLL, cfg: Config):
        self.lib = lib
        self.cfg = cfg
        self.h = lib.tc_encoder_create(ctypes.byref(cfg))
        if not self.h:
            raise RuntimeError("tc_encoder_create failed (no CUDA device or invalid config)")
        self.w, self.hgt = cfg.width, cfg.height

    def close(self) -> None:
        if self.h:
            self.lib.tc_encoder_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _ptr(a: np.ndarray):
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))

    def encode(self, y: np.ndarray, cb: np.ndarray, cr: np.ndarray) -> Optional[bytes]:
        """Encode one frame; returns the packet, or None while a B-frame GOP
        is still filling.  Raises on any other error code."""
        y, cb, cr = (np.ascontiguousarray(a, dtype=np.uint8) for a in (y, cb, cr))
        pkt = Packet()
        r = self.lib.tc_encoder_encode(self.h, self._ptr(y), y.shape[1], self._ptr(cb), cb.shape[1],
                                       self._ptr(cr), cr.shape[1], ctypes.byref(pkt))
        if r == TC_ERR_NEED_MORE:
            return None
        if r != TC_OK:
            raise RuntimeError(f"tc_encoder_encode -> {r}")
        return ctypes.string_at(pkt.data, pkt.size)

    def flush(self) -> List[bytes]:
        out = []
        while True:
            pkt = Packet()
            r = self.lib.tc_encoder_flush_tail(self.h, ctypes.byref(pkt))
            if r == TC_ERR_EOF:
                return out
            if r != TC_OK:
                raise RuntimeError(f"tc_encoder_flush_tail -> {r}")
            out.append(ctypes.string_at(pkt.data, pkt.size))

    def force_keyframe(self) -> None:
        self.lib.tc_encoder_force_keyframe(self.h)

    def stats(self) -> Tuple[int, int, float]:
        b, f, p = ctypes.c_int64(), ctypes.c_int32(), ctypes.c_double()
        self.lib.tc_encoder_get_stats(self.h, ctypes.byref(b), ctypes.byref(f), ctypes.byref(p))
        return b.value, f.value, p.value

    def recon(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Copy of encoder->recon (the reconstruction of the last frame)."""
        head = ctypes.cast(self.h, ctypes.POINTER(EncoderHead)).contents
        fb = head.recon.contents
        w, h = self.w, self.hgt

        def plane(p, stride, pw, ph):
            buf = ctypes.string_at(p, stride * ph)
            return np.frombuffer(buf, dtype=np.uint8).reshape(ph, stride)[:, :pw].copy()

        return (plane(fb.y, fb.stride_y, w, h), plane(fb.cb, fb.stride_c, w // 2, h // 2),
                plane(fb.cr, fb.stride_c, w // 2, h // 2))


def encode_sequence(lib: ctypes.CDLL, cfg: Config, frames, with_recon: bool = False):
    """Encode a list of (y, cb, cr) frames; returns the packets (coding
    order, B-frame tail drained) and optionally the recon after each call."""
    enc = Encoder(lib, cfg)
    pkts, recons = [], []
    try:
        for f in frames:
            p = enc.encode(*f)
            if p is not None:
                pkts.append(p)
                if with_recon:
                    recons.append(enc.recon())
        tail = enc.flush()
        pkts.extend(tail)
    finally:
        enc.close()
    return (pkts, recons) if with_recon else pkts
