"""ctypes binding of ``libbbhx_b200.so`` (the C ABI declared in ``include/bbhx_b200.h``).

There is no fallback: if the library or a CUDA device is missing, the first call raises.
Device arrays are torch CUDA tensors; host arrays are numpy arrays.  Every call is issued
on torch's current CUDA stream.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbbhx_b200.so")

_VP = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_LL = ctypes.c_longlong

# name -> argument types (every function returns int status unless listed in _RESTYPES)
_SIGS = {
    "bbhx_version": [],
    "bbhx_stream_synchronize": [_VP],
    "bbhx_take_status": [_VP],
    "bbhx_pointer_is_device": [_VP],
    "bbhx_mode_coeffs_bytes": [],
    "bbhx_response_mode_bytes": [],
    "bbhx_selftest_sincos": [_VP, _VP, _I, _VP],
    "bbhx_selftest_recurrence": [_VP, _D, _D, _D, _I, _I, _VP, _VP],
    "bbhx_count_point_ops": [_VP] * 5 + [_I, _VP, _I, _VP, _I, _D, _I, _I, _I, _VP],
    "bbhx_get_phenomhm_ringdown_frequencies": [_VP] * 8 + [_I, _I, _VP],
    "bbhx_get_phenomd_ringdown_frequencies": [_VP] * 6 + [_I] + [_VP] * 8 + [_D, _VP],
    "bbhx_ringdown_frequencies_all": [_VP] * 8 + [_I, _I, _VP, _I, _D, _I, _VP],
    "bbhx_waveform_amp_phase": [_VP] * 10 + [_I, _I, _I, _VP, _VP, _I, _VP],
    "bbhx_waveform_amp_phase_noalloc": [_VP] * 10 + [_I, _I, _I, _VP, _VP, _I, _VP],
    "bbhx_phenomhm_setup": [_VP] * 10 + [_I, _I, _I, _VP],
    "bbhx_phenomhm_points": [_VP, _VP, _VP, _VP, _D, _I, _I, _I, _VP],
    "bbhx_phenomhm_tf": [_VP, _VP, _VP, _VP, _I, _I, _I, _VP],
    "bbhx_default_freqs": [_VP, _VP, _VP, _VP, _D, _D, _I, _I, _I, _VP],
    "bbhx_tf_window_regrid": [_VP, _VP, _VP, _VP, _VP, _I, _LL, _VP, _VP],
    "bbhx_orbits_create": [ctypes.POINTER(_VP)],
    "bbhx_orbits_add_orbit_information": [_VP, _D, _I] + [_VP] * 6 + [_D],
    "bbhx_orbits_destroy": [_VP],
    "bbhx_LISA_response": [_VP] * 10 + [_I] * 8 + [_VP],
    "bbhx_waveform_response_fused": [_VP] * 12 + [_D, _I, _I, _I, _I, _I, _I, _VP],
    "bbhx_interpolate": [_VP] * 6 + [_I] * 4 + [_VP],
    "bbhx_InterpTDI": [_VP] * 9 + [_I] * 4 + [_VP] * 3 + [_VP],
    "bbhx_direct_sum": [_VP, _VP, _I, _I, _I, _I, _VP, _VP, _VP],
    "bbhx_fill_templates": [_VP, _VP, _VP, _VP, _I, _I, _I, _VP],
    "bbhx_direct_like": [_VP] * 7 + [_I, _I, _VP],
    "bbhx_hdyn": [_VP] * 5 + [_I, _I, _I, _VP],
    "bbhx_hdyn_constants": [_VP, _VP, _VP, _VP, _I, _VP, _I, _VP, _I, _I, _VP, _I, _D, _VP],
    "bbhx_template_support": [_VP, _VP, _VP, _I, _I, _I, _VP, _I, _VP],
    "bbhx_step_front": [_VP] * 10 + [_I, _I, _D, _D, _VP, _I, _VP],
    "bbhx_tf_range_check": [_VP, _LL, _D, _D, _VP, _VP],
    "bbhx_pack_lnl": [_VP, _VP, _VP, _D, _I, _I, _VP, _I, _VP],
    "bbhx_tssb_from_lframe": [_VP, _VP, _VP, _VP, _I, _D, _I, _VP],
    "bbhx_frame_transform": [_VP] * 8 + [_I, _D, _I, _VP],
    "bbhx_sky_mode_transform": [_VP] + [_I] * 8 + [_VP],
    "bbhx_direct_like_fused": [_VP] * 5 + [_I] + [_VP] * 7 + [_I, _I, _I, _I, _VP, _VP, _VP],
    "bbhx_hdyn_fused": [_VP] * 12 + [_D] + [_VP] * 5 + [_I] * 7 + [_VP],
    "bbhx_hdyn_grad": [_VP] * 9 + [_I, _D, _D] + [_VP] * 5 + [_I] * 7 + [_VP],
    "bbhx_direct_like_multi": [_VP, _I, _I, _I, _I, _VP],
    "bbhx_uneven_like": [_VP, _I, _VP, _I, _I, _I, _I, _VP],
    "bbhx_uneven_batch": [_VP, _I, _VP, _I, _I, _I, _I, _VP],
    "bbhx_workspace_set": [_VP, ctypes.c_size_t],
    "bbhx_workspace_peak": [],
    "bbhx_direct_like_grad": [_VP] * 8 + [_I, _D, _D] + [_VP] * 3 + [_I] + [_VP] * 9 + [_D, _D] + [_I] * 7 + [_VP],
}
_RESTYPES = {
    "bbhx_workspace_peak": ctypes.c_size_t,
    "bbhx_mode_coeffs_bytes": ctypes.c_size_t,
    "bbhx_response_mode_bytes": ctypes.c_size_t,
}


class BBHxCudaError(RuntimeError):
    """A CUDA-side failure reported by the library (status 2..6)."""


_lib = None


def lib():
    """Load the library (once).  Raises if it is missing or no CUDA device is present."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.isfile(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m bbhx_b200.build_ext` "
            "(bbhx_b200 has no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    for name, args in _SIGS.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, ctypes.c_int)
    L.bbhx_last_error_string.restype = ctypes.c_char_p
    L.bbhx_last_error_string.argtypes = []
    _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS) + ["bbhx_last_error_string"]


def check(status, name=""):
    if status == 0:
        return
    msg = lib().bbhx_last_error_string().decode(errors="replace")
    if status == 1:
        raise ValueError(f"{name}: {msg}")
    raise BBHxCudaError(f"{name} failed with status {status}: {msg}")


def call(name, *args):
    check(getattr(lib(), name)(*args), name)


def stream():
    import torch

    return _VP(torch.cuda.current_stream().cuda_stream)


def dptr(t, dtype=None):
    """Device address of a contiguous torch CUDA tensor (checked)."""
    import torch

    if t is None:
        return _VP(0)
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError("expected a torch CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("tensor must be contiguous")
    if dtype is not None and t.dtype != dtype:
        raise TypeError(f"expected {dtype}, got {t.dtype}")
    return _VP(t.data_ptr())


def hptr(a, dtype=None):
    """Host address of a C-contiguous numpy array (checked)."""
    if not isinstance(a, np.ndarray):
        raise TypeError("expected a numpy array")
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    if dtype is not None and a.dtype != dtype:
        raise TypeError(f"expected {dtype}, got {a.dtype}")
    return _VP(a.__array_interface__["data"][0])
