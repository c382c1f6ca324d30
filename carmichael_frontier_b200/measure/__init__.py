"""Measurement tooling for bench.py and the profiles: ceilings of the running GPU (micro.py).

Its kernels are built into libcfmicro.so next to libcfmitm.so, from measure/cf_micro.cu, and are
not part of the library's C ABI (include/cfmitm.h).
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG, "libcfmicro.so")
_lib = None
_lock = threading.Lock()


def load() -> C.CDLL:
    """Load libcfmicro.so (built with libcfmitm.so by carmichael_frontier_b200._build)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m carmichael_frontier_b200._build`")
            lib = C.CDLL(LIB_PATH)
            vp, u64, u32 = C.c_void_p, C.c_uint64, C.c_uint32
            lib.cf_micro_l2_probe.restype = C.c_int
            lib.cf_micro_l2_probe.argtypes = [vp, u64, C.c_int, u32, vp, vp]
            lib.cf_micro_mulhi.restype = C.c_int
            lib.cf_micro_mulhi.argtypes = [C.c_int, u32, vp, vp]
            _lib = lib
    return _lib
