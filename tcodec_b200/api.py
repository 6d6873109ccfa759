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
KERNEL_DEBLOCK, KERNEL_SAO, KERNEL_MC = 0, 1, 2   # tcb_autotune_* kernel ids
QUEUE_DIAGONAL, QUEUE_STAGGERED = 0, 1            # tcb_engine_set_tuning queue orders
SEARCH_WINDOW_MIN, SEARCH_WINDOW_MAX = 2, 5
STAGING_TMA = 0x10000                             # TCB_STAGING_TMA: deblocking tiles staged by TMA


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
    pp = P(P(ctypes.c_uint8))
    ip = P(ctypes.c_int)
    lib.tc_decoder_create.argtypes = [ctypes.c_int32, ctypes.c_int32]
    lib.tc_decoder_create.restype = ctypes.c_void_p
    lib.tc_decoder_destroy.argtypes = [ctypes.c_void_p]
    lib.tc_decoder_set_threads.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.tc_decoder_destroy.restype = None
    lib.tc_decoder_decode.argtypes = [ctypes.c_void_p, u8p, ctypes.c_size_t, pp, ip, pp, ip, pp, ip]
    lib.tc_decoder_decode.restype = ctypes.c_int
    lib.tc_decoder_flush_tail.argtypes = [ctypes.c_void_p, pp, ip, pp, ip, pp, ip]
    lib.tc_decoder_flush_tail.restype = ctypes.c_int
    lib.tc_decoder_crc_valid.argtypes = [ctypes.c_void_p]
    lib.tc_decoder_crc_valid.restype = ctypes.c_int
    lib.tc_decoder_entropy_coded.argtypes = [ctypes.c_void_p]
    lib.tc_decoder_entropy_coded.restype = ctypes.c_int
    lib.tc_decoder_get_info.argtypes = [ctypes.c_void_p, P(ctypes.c_int32), P(ctypes.c_int32)]
    lib.tc_decoder_get_info.restype = None
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
                b_frames: bool = False, crc: bool = False, version: int = 2, threads: int = 0) -> Config:
    """tc_config_defaults + the fields `tcenc` sets (reference
    tools/tcenc.c:127-185): `version` 2 is `--v2` (quadtree syntax), 0 and 1
    are `--bs-version 0/1` (legacy 8x8 block syntax); `threads` 0 is the
    default worker count, which lays legacy rows out as separate runs."""
    cfg = Config()
    lib.tc_config_defaults(ctypes.byref(cfg), width, height)
    cfg.preset = preset
    cfg.qp = qp
    cfg.keyframe_interval = keyframe_interval
    cfg.profile = profile
    cfg.threads = threads
    if version == 2:
        cfg.use_v2 = 1
    else:
        cfg.use_v2 = 0
        cfg.bitstream_version = version
    cfg.enable_entropy_coded = 1 if entropy else 0
    cfg.enable_b_frames = 1 if b_frames else 0
    cfg.enable_crc = 1 if crc else 0
    return cfg


class Encoder:
    """One encode session through the C ABI (v2 or legacy, as `cfg` says)."""

    def __init__(self, lib: ctypes.CDLL, cfg: Config):
        self.lib = lib
        self.cfg = cfg
        self.h = lib.tc_encoder_create(ctypes.byref(cfg))
        if not self.h:
            raise RuntimeError("tc_encoder_create failed (no CUDA device or invalid config)")
        self.w, self.hgt = cfg.width, cfg.height
        self.last_key_frame = None   # key_frame flag of the last packet encode() returned

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
        self.last_key_frame = int(pkt.key_frame)
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


class Decoder:
    """One decode session through the C ABI (tc_decoder_*)."""

    def __init__(self, lib: ctypes.CDLL, width: int = 0, height: int = 0, threads: Optional[int] = None):
        self.lib = lib
        self.h = lib.tc_decoder_create(width, height)
        if not self.h:
            raise RuntimeError("tc_decoder_create failed")
        if threads is not None:
            lib.tc_decoder_set_threads(self.h, threads)

    def close(self) -> None:
        if self.h:
            self.lib.tc_decoder_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _planes(self, y, ys, cb, cbs, cr, crs):
        w, h = ctypes.c_int32(), ctypes.c_int32()
        self.lib.tc_decoder_get_info(self.h, ctypes.byref(w), ctypes.byref(h))
        W, H = w.value, h.value

        def plane(p, stride, pw, ph):
            buf = ctypes.string_at(p, stride * ph)
            return np.frombuffer(buf, dtype=np.uint8).reshape(ph, stride)[:, :pw].copy()

        return (plane(y, ys.value, W, H), plane(cb, cbs.value, W // 2, H // 2),
                plane(cr, crs.value, W // 2, H // 2))

    def decode(self, packet: bytes):
        """Returns (y, cb, cr), None while a B-frame reorder waits, or
        raises on an error code (the code is in the exception args)."""
        P = ctypes.POINTER(ctypes.c_uint8)
        y, cb, cr = P(), P(), P()
        ys, cbs, crs = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        buf = (ctypes.c_uint8 * max(1, len(packet))).from_buffer_copy(packet or b"\0")
        r = self.lib.tc_decoder_decode(self.h, buf, len(packet), ctypes.byref(y), ctypes.byref(ys),
                                       ctypes.byref(cb), ctypes.byref(cbs), ctypes.byref(cr), ctypes.byref(crs))
        if r == TC_ERR_NEED_MORE:
            return None
        if r != TC_OK:
            raise RuntimeError("tc_decoder_decode", r)
        return self._planes(y, ys, cb, cbs, cr, crs)

    def flush(self):
        out = []
        P = ctypes.POINTER(ctypes.c_uint8)
        while True:
            y, cb, cr = P(), P(), P()
            ys, cbs, crs = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
            r = self.lib.tc_decoder_flush_tail(self.h, ctypes.byref(y), ctypes.byref(ys), ctypes.byref(cb),
                                               ctypes.byref(cbs), ctypes.byref(cr), ctypes.byref(crs))
            if r != TC_OK:
                return out
            out.append(self._planes(y, ys, cb, cbs, cr, crs))

    def crc_valid(self) -> int:
        return self.lib.tc_decoder_crc_valid(self.h)


REF_FRAMES = 4


class FrameDesc(ctypes.Structure):
    """tcb_frame_desc_t: one frame for the CTU engine (device pointers)."""
    _fields_ = [("width", ctypes.c_int), ("height", ctypes.c_int),
                ("stride_y", ctypes.c_int), ("stride_c", ctypes.c_int),
                ("src_y", ctypes.c_void_p), ("src_cb", ctypes.c_void_p), ("src_cr", ctypes.c_void_p),
                ("rec_y", ctypes.c_void_p), ("rec_cb", ctypes.c_void_p), ("rec_cr", ctypes.c_void_p),
                ("ref_y", ctypes.c_void_p * REF_FRAMES), ("ref_cb", ctypes.c_void_p * REF_FRAMES),
                ("ref_cr", ctypes.c_void_p * REF_FRAMES), ("ref_poc", ctypes.c_int * REF_FRAMES),
                ("prev_mv_grid", ctypes.c_void_p), ("cur_mv_grid", ctypes.c_void_p),
                ("ctu_records", ctypes.c_void_p),
                ("frame_type", ctypes.c_int), ("poc", ctypes.c_int), ("qp", ctypes.c_int),
                ("preset", ctypes.c_int), ("profile", ctypes.c_int),
                ("global_mv_valid", ctypes.c_int), ("global_mv_x", ctypes.c_int),
                ("global_mv_y", ctypes.c_int)]


class FilterFrame(ctypes.Structure):
    """tcb_filter_frame_t: one frame for tcb_deblock_frames / tcb_sao_frames."""
    _fields_ = [("width", ctypes.c_int), ("height", ctypes.c_int), ("stride_y", ctypes.c_int),
                ("stride_c", ctypes.c_int), ("y", ctypes.c_void_p), ("cb", ctypes.c_void_p), ("cr", ctypes.c_void_p),
                ("src_y", ctypes.c_void_p), ("stride_src", ctypes.c_int), ("qp", ctypes.c_int),
                ("sao_params", ctypes.c_void_p)]


class McFrame(ctypes.Structure):
    """tcb_mc_frame_t: one frame for tcb_mc_frames."""
    _fields_ = [("width", ctypes.c_int), ("height", ctypes.c_int), ("stride_y", ctypes.c_int),
                ("stride_c", ctypes.c_int), ("ref_y", ctypes.c_void_p), ("ref_cb", ctypes.c_void_p),
                ("ref_cr", ctypes.c_void_p), ("pred_y", ctypes.c_void_p), ("pred_cb", ctypes.c_void_p),
                ("pred_cr", ctypes.c_void_p), ("mv", ctypes.c_void_p)]


def bind_b200(lib: ctypes.CDLL) -> ctypes.CDLL:
    """Attach argtypes of the include/tcodec_b200.h encoder extensions."""
    vp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)
    lib.tcb_encoder_encode_device.argtypes = [vp] + [vp, ctypes.c_int] * 3 + [ctypes.POINTER(Packet)]
    lib.tcb_encoder_encode_device.restype = ctypes.c_int
    lib.tcb_encoder_stream.argtypes = [vp]
    lib.tcb_encoder_stream.restype = vp
    lib.tcb_encoder_set_timing.argtypes = [vp, ctypes.c_int]
    lib.tcb_encoder_get_timing.argtypes = [vp] + [vp] * 5
    lib.tcb_encoder_set_recon_readback.argtypes = [vp, ctypes.c_int]
    lib.tcb_encoder_set_entropy_threads.argtypes = [vp, ctypes.c_int]
    lib.tcb_batch_create.argtypes = [ctypes.POINTER(Config), ctypes.c_int]
    lib.tcb_batch_create.restype = vp
    lib.tcb_batch_destroy.argtypes = [vp]
    lib.tcb_batch_encoder.argtypes = [vp, ctypes.c_int]
    lib.tcb_batch_encoder.restype = vp
    lib.tcb_batch_stream.argtypes = [vp]
    lib.tcb_batch_stream.restype = vp
    lib.tcb_batch_encode.argtypes = [vp, ctypes.POINTER(vp), ip, ctypes.POINTER(vp), ip, ctypes.POINTER(vp), ip,
                                     ctypes.c_int, ctypes.POINTER(Packet), ip]
    lib.tcb_batch_encode.restype = ctypes.c_int
    lib.tcb_batch_flush.argtypes = [vp, ctypes.POINTER(Packet), ip]
    lib.tcb_batch_flush.restype = ctypes.c_int
    lib.tcb_batch_set_timing.argtypes = [vp, ctypes.c_int]
    lib.tcb_batch_get_timing.argtypes = [vp] + [vp] * 5
    lib.tcb_batch_get_host_timing.argtypes = [vp] + [vp] * 3
    lib.tcb_batch_set_graphs.argtypes = [vp, ctypes.c_int]
    lib.tcb_batch_set_pipelined.argtypes = [vp, ctypes.c_int]
    lib.tcb_batch_set_pipelined.restype = ctypes.c_int
    lib.tcb_batch_drain.argtypes = [vp, ctypes.POINTER(Packet), ip]
    lib.tcb_batch_drain.restype = ctypes.c_int
    lib.tcb_batch_get_graph_stats.argtypes = [vp, vp, vp]
    lib.tcb_batch_get_graph_stats.restype = ctypes.c_int
    lib.tcb_ctu_record_bytes.restype = ctypes.c_size_t
    lib.tcb_mv_cell_bytes.restype = ctypes.c_size_t
    lib.tcb_ctu_scratch_bytes.argtypes = [ctypes.c_int, ctypes.c_int]
    lib.tcb_ctu_scratch_bytes.restype = ctypes.c_size_t
    lib.tcb_ctu_encode_frame.argtypes = [ctypes.POINTER(FrameDesc), vp, ctypes.c_size_t, vp]
    lib.tcb_ctu_encode_frame.restype = ctypes.c_int
    lib.tcb_ctu_encode_frame_static.argtypes = [ctypes.POINTER(FrameDesc), vp]
    lib.tcb_ctu_encode_frame_static.restype = ctypes.c_int
    lib.tcb_ctu_frame_result.argtypes = [vp, vp]
    lib.tcb_ctu_frame_result.restype = ctypes.c_int
    lib.tcb_ctu_frame_result_static.argtypes = [vp]
    lib.tcb_ctu_frame_result_static.restype = ctypes.c_int
    lib.tcb_set_neighbor_wait_limit.argtypes = [ctypes.c_longlong]
    lib.tcb_set_neighbor_wait_limit.restype = ctypes.c_int
    lib.tcb_get_neighbor_wait_limit.argtypes = [ctypes.POINTER(ctypes.c_longlong)]
    lib.tcb_get_neighbor_wait_limit.restype = ctypes.c_int
    lib.tcb_debug_ctu_encode_frame_without_first.argtypes = [ctypes.POINTER(FrameDesc), vp, ctypes.c_size_t, vp]
    lib.tcb_debug_ctu_encode_frame_without_first.restype = ctypes.c_int
    lib.tcb_debug_fail_allocations_after.argtypes = [ctypes.c_longlong]
    lib.tcb_debug_fail_allocations_after.restype = ctypes.c_longlong
    for fn in (lib.tcb_deblock_frames, lib.tcb_sao_frames):
        fn.argtypes = [ctypes.POINTER(FilterFrame), ctypes.c_int, vp]
        fn.restype = ctypes.c_int
    lib.tcb_mc_frames.argtypes = [ctypes.POINTER(McFrame), ctypes.c_int, vp]
    lib.tcb_mc_frames.restype = ctypes.c_int
    lib.tcb_autotune_frame_kernels.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.tcb_autotune_frame_kernels.restype = ctypes.c_int
    lib.tcb_autotune_threads.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.tcb_autotune_threads.restype = ctypes.c_int
    lib.tcb_autotune_set_threads.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.tcb_autotune_set_threads.restype = ctypes.c_int
    lib.tcb_engine_set_tuning.argtypes = [ctypes.c_int] * 4
    lib.tcb_engine_set_tuning.restype = ctypes.c_int
    lib.tcb_engine_get_tuning.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    lib.tcb_engine_get_tuning.restype = ctypes.c_int
    lib.tcb_frame_kernels_errors.argtypes = []
    lib.tcb_frame_kernels_errors.restype = ctypes.c_uint
    return lib


class BatchEncoder:
    """N independent v2 streams sharing every CTU-engine launch
    (tcb_batch_*).  `encode(frames)` takes one (y, cb, cr) per stream —
    numpy arrays (host) or (ptr, stride) device-pointer triples — or None
    to skip a stream; returns a list of packets (None while buffering)."""

    def __init__(self, lib: ctypes.CDLL, cfgs: List[Config]):
        self.lib = bind_b200(lib)
        self.n = len(cfgs)
        arr = (Config * self.n)(*cfgs)
        self.h = lib.tcb_batch_create(arr, self.n)
        if not self.h:
            raise RuntimeError("tcb_batch_create failed")
        self.cfgs = cfgs

    def set_graphs(self, on: bool = True):
        """Replay each step's device work as one CUDA graph (tcb_batch_set_graphs)."""
        self.lib.tcb_batch_set_graphs(self.h, 1 if on else 0)

    def set_pipelined(self, on: bool = True):
        """Entropy-code each call's frames during the next call's device step
        (tcb_batch_set_pipelined): packets arrive one call later, `flush`
        returns the last ones."""
        r = self.lib.tcb_batch_set_pipelined(self.h, 1 if on else 0)
        if r != TC_OK:
            raise RuntimeError(f"tcb_batch_set_pipelined -> {r}")

    def drain(self):
        """Pipelined batch: the packets still pending from the last call (per
        stream, None where none), without running new frames."""
        pk = (Packet * self.n)()
        st = (ctypes.c_int * self.n)()
        r = self.lib.tcb_batch_drain(self.h, pk, st)
        if r not in (TC_OK, TC_ERR_EOF):
            raise RuntimeError(f"tcb_batch_drain -> {r}")
        return [ctypes.string_at(pk[i].data, pk[i].size) if r == TC_OK and st[i] == TC_OK else None
                for i in range(self.n)]

    def graph_stats(self):
        """(graph launches, graph instantiations, last refused-update result)
        since the last call."""
        a, b = ctypes.c_int64(), ctypes.c_int64()
        r = self.lib.tcb_batch_get_graph_stats(self.h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value, r

    def close(self):
        if self.h:
            self.lib.tcb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _call(self, planes, on_device):
        n = self.n
        VP = ctypes.c_void_p * n
        I = ctypes.c_int * n
        y, cb, cr, sy, scb, scr = VP(), VP(), VP(), I(), I(), I()
        keep = []
        for i, f in enumerate(planes):
            if f is None:
                continue
            if on_device:
                (y[i], sy[i]), (cb[i], scb[i]), (cr[i], scr[i]) = f
            else:
                a = [np.ascontiguousarray(p, dtype=np.uint8) for p in f]
                keep.append(a)
                y[i], cb[i], cr[i] = (p.ctypes.data for p in a)
                sy[i], scb[i], scr[i] = (p.shape[1] for p in a)
        pk = (Packet * n)()
        st = I()
        r = self.lib.tcb_batch_encode(self.h, y, sy, cb, scb, cr, scr, 1 if on_device else 0, pk, st)
        return r, pk, st

    def encode(self, planes, on_device: bool = False):
        r, pk, st = self._call(planes, on_device)
        if r not in (TC_OK, TC_ERR_NEED_MORE):
            raise RuntimeError(f"tcb_batch_encode -> {r}", list(st))
        return [ctypes.string_at(pk[i].data, pk[i].size) if st[i] == TC_OK else None for i in range(self.n)]

    def flush(self):
        """All remaining packets, per stream."""
        out = [[] for _ in range(self.n)]
        while True:
            pk = (Packet * self.n)()
            st = (ctypes.c_int * self.n)()
            r = self.lib.tcb_batch_flush(self.h, pk, st)
            if r == TC_ERR_EOF:
                return out
            if r != TC_OK:
                raise RuntimeError(f"tcb_batch_flush -> {r}")
            for i in range(self.n):
                if st[i] == TC_OK:
                    out[i].append(ctypes.string_at(pk[i].data, pk[i].size))


def decode_sequence(lib: ctypes.CDLL, packets, width: int = 0, height: int = 0, threads: Optional[int] = None):
    """Decode packets (coding order) into display-order frames
    (`threads`: tc_decoder_set_threads, when given)."""
    dec = Decoder(lib, width, height, threads)
    out = []
    try:
        for p in packets:
            f = dec.decode(p)
            if f is not None:
                out.append(f)
        out.extend(dec.flush())
    finally:
        dec.close()
    return out


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


class ServerPacket(ctypes.Structure):
    _fields_ = [("session", ctypes.c_int), ("status", ctypes.c_int), ("packet", Packet)]


SESSION_WAITING, SESSION_ACTIVE, SESSION_DONE = 0, 1, 2
SERVER_QUEUE = 2


def bind_server(lib: ctypes.CDLL) -> ctypes.CDLL:
    """Attach argtypes of the include/tcodec_b200.h served-form entry points."""
    vp = ctypes.c_void_p
    lib.tcb_server_create.argtypes = [ctypes.c_size_t, ctypes.c_int]
    lib.tcb_server_create.restype = vp
    lib.tcb_server_destroy.argtypes = [vp]
    lib.tcb_server_session_bytes.argtypes = [ctypes.POINTER(Config)]
    lib.tcb_server_session_bytes.restype = ctypes.c_size_t
    lib.tcb_server_open.argtypes = [vp, ctypes.POINTER(Config)]
    lib.tcb_server_open.restype = ctypes.c_int
    lib.tcb_server_push.argtypes = [vp, ctypes.c_int] + [vp, ctypes.c_int] * 3
    lib.tcb_server_push.restype = ctypes.c_int
    lib.tcb_server_finish.argtypes = [vp, ctypes.c_int]
    lib.tcb_server_finish.restype = ctypes.c_int
    lib.tcb_server_session_state.argtypes = [vp, ctypes.c_int]
    lib.tcb_server_session_state.restype = ctypes.c_int
    lib.tcb_server_step.argtypes = [vp, ctypes.POINTER(ServerPacket), ctypes.c_int]
    lib.tcb_server_step.restype = ctypes.c_int
    lib.tcb_server_stats.argtypes = [vp] + [vp] * 5
    lib.tcb_server_set_graphs.argtypes = [vp, ctypes.c_int]
    lib.tcb_server_get_timing.argtypes = [vp, vp, vp, vp]
    lib.tcb_server_get_timing.restype = None
    return lib


class Server:
    """Served form (tcb_server_*): sessions opened at any time, admitted
    under an HBM budget, advanced together one frame per step."""

    def __init__(self, lib: ctypes.CDLL, hbm_budget_bytes: int, max_active: int = 64):
        self.lib = bind_server(lib)
        self.h = lib.tcb_server_create(int(hbm_budget_bytes), int(max_active))
        if not self.h:
            raise RuntimeError("tcb_server_create failed")
        self.max_active = max_active
        self._out = (ServerPacket * max_active)()

    def set_graphs(self, on: bool = True):
        """Replay each step's device work as one CUDA graph (tcb_server_set_graphs)."""
        self.lib.tcb_server_set_graphs(self.h, 1 if on else 0)

    def close(self):
        if self.h:
            self.lib.tcb_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def session_bytes(self, cfg: Config) -> int:
        return self.lib.tcb_server_session_bytes(ctypes.byref(cfg))

    def open(self, cfg: Config) -> int:
        sid = self.lib.tcb_server_open(self.h, ctypes.byref(cfg))
        if sid < 0:
            raise RuntimeError(f"tcb_server_open -> {sid}")
        return sid

    def push(self, sid: int, frame) -> bool:
        """Queue one (y, cb, cr) frame; False when the session's queue is full."""
        y, cb, cr = (np.ascontiguousarray(p, dtype=np.uint8) for p in frame)
        r = self.lib.tcb_server_push(self.h, sid, y.ctypes.data, y.shape[1], cb.ctypes.data, cb.shape[1],
                                     cr.ctypes.data, cr.shape[1])
        if r == TC_ERR_NEED_MORE:
            return False
        if r != TC_OK:
            raise RuntimeError(f"tcb_server_push -> {r}")
        return True

    def finish(self, sid: int) -> None:
        self.lib.tcb_server_finish(self.h, sid)

    def state(self, sid: int) -> int:
        return self.lib.tcb_server_session_state(self.h, sid)

    def step(self):
        """One step; returns [(session, status, packet bytes or None)]."""
        n = self.lib.tcb_server_step(self.h, self._out, self.max_active)
        if n < 0:
            raise RuntimeError(f"tcb_server_step -> {n}")
        res = []
        for i in range(n):
            e = self._out[i]
            data = ctypes.string_at(e.packet.data, e.packet.size) if e.status == TC_OK else None
            res.append((e.session, e.status, data))
        return res

    def timing(self):
        """Host ms in admission and in whole steps since creation, sessions
        admitted (tcb_server_get_timing)."""
        a, st, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_longlong()
        self.lib.tcb_server_get_timing(self.h, ctypes.byref(a), ctypes.byref(st), ctypes.byref(n))
        return dict(admit_ms=a.value, step_ms=st.value, admitted=n.value)

    def stats(self):
        w, a, d = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        used, cap = ctypes.c_size_t(), ctypes.c_size_t()
        self.lib.tcb_server_stats(self.h, ctypes.byref(w), ctypes.byref(a), ctypes.byref(d), ctypes.byref(used),
                                  ctypes.byref(cap))
        return dict(waiting=w.value, active=a.value, retired=d.value, bytes_in_use=used.value,
                    bytes_budget=cap.value)


def engine_tuning(lib: ctypes.CDLL, width: int, height: int) -> Tuple[int, int]:
    """(search_window, queue_order) the engine uses for this frame size."""
    w, q = ctypes.c_int(), ctypes.c_int()
    r = lib.tcb_engine_get_tuning(width, height, ctypes.byref(w), ctypes.byref(q))
    if r != TC_OK:
        raise RuntimeError(f"tcb_engine_get_tuning -> {r}")
    return w.value, q.value


def set_engine_tuning(lib: ctypes.CDLL, width: int, height: int, search_window: int, queue_order: int) -> None:
    """tcb_engine_set_tuning; (0, 0) restores the defaults."""
    r = lib.tcb_engine_set_tuning(width, height, search_window, queue_order)
    if r != TC_OK:
        raise RuntimeError(f"tcb_engine_set_tuning({width}, {height}, {search_window}, {queue_order}) -> {r}")
