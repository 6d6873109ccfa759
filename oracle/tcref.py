"""Loader for the reference TCodec C library compiled by oracle/Makefile.

Test infrastructure only: tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use it as the checker.  The reference exports the same
include/tcodec.h ABI, so tcodec_b200.api.Encoder drives both libraries.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libtcref.so")
REF_TCENC = os.path.join(HERE, "_ref", "tcenc")
REF_TCDEC = os.path.join(HERE, "_ref", "tcdec")
PORT_LIB = os.path.join(HERE, "liboracle.so")

_ref = None


def available() -> bool:
    return os.path.exists(REF_LIB)


def ref_lib():
    """ctypes handle of the reference library (RTLD_LOCAL, -Bsymbolic build)."""
    global _ref
    if _ref is None:
        from tcodec_b200.api import bind
        if not os.path.exists(REF_LIB):
            raise RuntimeError("oracle/_ref/libtcref.so is not built (make -C oracle ref)")
        _ref = bind(ctypes.CDLL(REF_LIB, mode=os.RTLD_LOCAL | os.RTLD_NOW))
    return _ref
