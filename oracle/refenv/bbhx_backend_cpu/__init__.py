"""ctypes bindings of oracle/_ref/libbbhx_ref.so, laid out as the five compiled
extension modules the reference's CPU backend imports (cutils/__init__.py:60-78)."""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "..", "..", "_ref", "libbbhx_ref.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(os.path.abspath(_LIB_PATH))
    return _lib


def P(a, dtype=None):
    """Address of a C-contiguous numpy array (checked), or an int passed through."""
    if isinstance(a, (int, np.integer)) and not isinstance(a, bool):
        return ctypes.c_void_p(int(a))
    if not isinstance(a, np.ndarray):
        raise TypeError(f"expected numpy array, got {type(a)}")
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    if dtype is not None and a.dtype != dtype:
        raise TypeError(f"expected {dtype}, got {a.dtype}")
    return ctypes.c_void_p(a.__array_interface__["data"][0])


I = ctypes.c_int
D = ctypes.c_double
