"""Loads libmach2d_b200.so (built in-tree by mach2d_b200/build.py).

There is no CPU fallback: if the library is missing or a call reports a CUDA
failure, the error propagates to the caller.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmach2d_b200.so")

M2D_OK = 0
ERRORS = {
    1: "CUDA error",
    2: "invalid argument",
    3: "NaN detected",
    4: "iteration or wait limit reached",
    5: "device allocation failed",
    6: "grid larger than supported",
    7: "zero or non-finite pivot",
}

_lib = None


class M2DError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"mach2d_b200 error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


def lib():
    """The loaded shared library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: run `python mach2d_b200/build.py`")
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.m2d_last_error.restype = ctypes.c_char_p
    return _lib


def check(rc):
    if rc != M2D_OK:
        raise M2DError(rc, lib().m2d_last_error().decode(errors="replace"))
    return rc


def dptr(a):
    """Pointer to a C-contiguous float64 numpy array (no copy)."""
    if not isinstance(a, np.ndarray) or a.dtype != np.float64 or not a.flags.c_contiguous:
        raise TypeError("expected a C-contiguous float64 numpy array")
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def call(name, *args):
    """Calls a by-reference C entry point: ints and floats are passed as
    pointers to c_int / c_double, numpy arrays as data pointers."""
    conv = []
    keep = []
    for a in args:
        if isinstance(a, np.ndarray):
            conv.append(dptr(a))
        elif isinstance(a, (bool, int, np.integer)):
            v = ctypes.c_int(int(a))
            keep.append(v)
            conv.append(ctypes.byref(v))
        elif isinstance(a, (float, np.floating)):
            v = ctypes.c_double(float(a))
            keep.append(v)
            conv.append(ctypes.byref(v))
        elif isinstance(a, (ctypes._SimpleCData, ctypes.Structure)):
            conv.append(ctypes.byref(a))
        else:
            raise TypeError(f"unsupported argument {type(a)}")
    return check(getattr(lib(), name)(*conv))


def exported_symbols():
    """Names of the entry points declared in include/mach2d_b200.h."""
    import re
    hdr = os.path.join(HERE, "..", "include", "mach2d_b200.h")
    text = open(hdr).read()
    return sorted(set(re.findall(r"\b(m2d_[a-z0-9_]+)\s*\(", text)))
