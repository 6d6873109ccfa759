"""ctypes bindings of oracle/liboracle.so (the C restatement) and of the
reference kernels exported by oracle/_ref/libtcref.so.  Test-only."""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PORT = os.path.join(ROOT, "oracle", "liboracle.so")
REF = os.path.join(ROOT, "oracle", "_ref", "libtcref.so")

u8p = ctypes.POINTER(ctypes.c_uint8)
i16p = ctypes.POINTER(ctypes.c_int16)
ip = ctypes.POINTER(ctypes.c_int)
c_int = ctypes.c_int


class MV(ctypes.Structure):
    _fields_ = [("x", ctypes.c_int32), ("y", ctypes.c_int32)]


def P(a):
    """Pointer to a numpy array's data (uint8 or int16)."""
    if a.dtype == np.uint8:
        return a.ctypes.data_as(u8p)
    if a.dtype == np.int16:
        return a.ctypes.data_as(i16p)
    if a.dtype == np.int32:
        return a.ctypes.data_as(ip)
    raise TypeError(a.dtype)


def PO(a, off):
    """Pointer to a[off] (flat element offset) of a uint8 array."""
    return ctypes.cast(a.ctypes.data + off * a.itemsize, u8p if a.dtype == np.uint8 else i16p)


def port():
    if not os.path.exists(PORT):
        raise RuntimeError("oracle/liboracle.so not built (make -C oracle port)")
    L = ctypes.CDLL(PORT, mode=os.RTLD_LOCAL | os.RTLD_NOW)
    L.or_sad.restype = c_int
    L.or_lambda.restype = c_int
    L.or_eff_scale.restype = c_int
    L.or_qscale.restype = c_int
    L.or_quant.restype = c_int
    L.or_dequant.restype = c_int
    L.or_freq_band.restype = c_int
    L.or_code_tu.restype = ctypes.c_longlong
    L.or_code_tu.argtypes = [c_int, u8p, c_int, u8p, c_int, c_int, ctypes.c_longlong, i16p, u8p, c_int, ip]
    L.or_sao_choose.restype = c_int
    return L


def ref():
    if not os.path.exists(REF):
        return None
    L = ctypes.CDLL(REF, mode=os.RTLD_LOCAL | os.RTLD_NOW)
    L.tc_motion_est.restype = MV
    L.tc_motion_est.argtypes = [u8p, c_int, c_int, c_int, u8p, c_int, c_int, c_int, c_int, c_int, ip]
    L.tc_inter_predict.argtypes = [u8p, c_int, c_int, c_int, MV, u8p, c_int, c_int]
    L.tc_inter_predict_chroma.argtypes = [u8p, c_int, c_int, c_int, MV, u8p, c_int, c_int]
    L.tc_sad.restype = c_int
    L.tc_lambda.restype = c_int
    L.tc_qscale.restype = c_int
    L.tc_freq_band.restype = c_int
    L.tc_sao_choose_bo.restype = c_int
    return L
