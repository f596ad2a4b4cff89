"""BBHx backend methods on ``libbbhx_b200.so``.

BBHx's drivers (``PhenomHMAmpPhase``, ``LISATDIResponse``, ``CubicSplineInterpolant``,
``BBHWaveformFD``, ``Likelihood``, ``HeterodynedLikelihood``) call every compiled kernel through
a backend object with nine methods plus ``xp`` (src/bbhx/cutils/__init__.py:13-23; the Cython
wrappers in src/bbhx/cutils/{phenomhm,lisaresponse,interp,bbhwaveformbuild,bbhlikelihood}.pyx
define their positional arguments).  ``b200_methods()`` returns those nine methods bound to this
library's C entry points, with the same positional arguments, so the unmodified BBHx drivers run
their GPU path on the sm_100a kernels once a maintainer registers it as a backend.

Array arguments are converted to addresses the way BBHx's ``wrapper`` does: torch CUDA tensors
and objects exposing ``__cuda_array_interface__`` (cupy) give device addresses, numpy arrays give
host addresses, plain integers are taken as addresses.  Unlike a raw cast, every slot is checked
against what the C entry point reads there: a device slot refuses host memory and a host slot
(the pointer arrays of ``InterpTDI`` / ``direct_like`` and ``direct_like``'s ``d_h`` / ``h_h``,
as in the reference) refuses device memory, so a wrong array raises ``TypeError`` instead of
reaching a kernel.  Status codes map to exceptions as in ``bbhx_b200._lib.check``.
"""
import ctypes

import numpy as np

from . import _lib

# slot codes: D<dtype> device array, H<dtype> host array, i int, d double, b bool (as int)
_SLOT_DTYPES = {"f8": (np.float64, "torch.float64"), "i4": (np.int32, "torch.int32"),
                "i8": (np.int64, "torch.int64"), "c16": (np.complex128, "torch.complex128")}

# positional arguments of each backend method (reference .pyx order) -> C entry point
_METHODS = {
    # phenomhm.pyx:61-114 -> PhenomHMWaveform.hh:354-371
    "waveform_amp_phase_wrap": ("bbhx_waveform_amp_phase",
                                ["Df8", "Di4", "Di4", "Df8", "Df8", "Df8", "Df8", "Df8", "Df8",
                                 "Df8", "i", "i", "i", "Df8", "Df8", "b"]),
    # phenomhm.pyx -> PhenomHMWaveform.hh:322-333
    "get_phenomhm_ringdown_frequencies": ("bbhx_get_phenomhm_ringdown_frequencies",
                                          ["Df8"] * 6 + ["Di4", "Di4", "i", "i"]),
    # phenomhm.pyx -> PhenomHMWaveform.hh:335-352
    "get_phenomd_ringdown_frequencies": ("bbhx_get_phenomd_ringdown_frequencies",
                                         ["Df8"] * 6 + ["i"] + ["Df8"] * 8 + ["d"]),
    # interp.pyx:14-31 -> Interpolate.hh:4-6
    "interpolate_wrap": ("bbhx_interpolate", ["Df8"] * 6 + ["i"] * 4),
    # bbhwaveformbuild.pyx:18-35 -> WaveformBuild.hh:6
    "InterpTDI_wrap": ("bbhx_InterpTDI",
                       ["Hi8", "Df8", "Df8", "Df8", "Df8", "Df8", "Df8", "Hf8", "Hf8", "i", "i",
                        "i", "i", "Hi8", "Hi4", "Hi4"]),
    # bbhwaveformbuild.pyx:37-49 -> WaveformBuild.hh:8-10
    "direct_sum_wrap": ("bbhx_direct_sum", ["Dc16", "Df8", "i", "i", "i", "i", "Df8", "Df8"]),
    # bbhlikelihood.pyx:43-56 -> Likelihood.hh:11
    "direct_like_wrap": ("bbhx_direct_like",
                         ["Hc16", "Hc16", "Dc16", "Df8", "Hi8", "Hi4", "Hi4", "i", "i"]),
    # bbhlikelihood.pyx:21-41 -> Likelihood.hh:6-9
    "hdyn_wrap": ("bbhx_hdyn", ["Dc16", "Dc16", "Dc16", "Dc16", "Df8", "i", "i", "i"]),
}
# lisaresponse.pyx:78-121 -> Response.hh:27-41 (after the orbit handle)
_RESPONSE_SLOTS = ["Df8", "Di4", "Di4", "Df8", "Df8", "Df8", "Df8", "Df8", "Df8", "i", "b", "b",
                   "i", "i", "i", "i", "i"]


def _torch():
    import torch

    return torch


def _is_device_address(addr):
    return addr != 0 and _lib.lib().bbhx_pointer_is_device(ctypes.c_void_p(addr)) == 1


def _device_addr(a, dt, where):
    """Device address of a device array in slot ``where`` (dtype ``dt``)."""
    torch = _torch()
    np_dtype, torch_name = _SLOT_DTYPES[dt]
    if isinstance(a, torch.Tensor):
        if not a.is_cuda:
            raise TypeError(f"{where}: expected device memory, got a CPU tensor")
        if str(a.dtype) != torch_name:
            raise TypeError(f"{where}: expected {torch_name}, got {a.dtype}")
        if not a.is_contiguous():
            raise ValueError(f"{where}: tensor must be contiguous")
        return a.data_ptr()
    cai = getattr(a, "__cuda_array_interface__", None)
    if cai is not None:
        if np.dtype(cai["typestr"]) != np.dtype(np_dtype):
            raise TypeError(f"{where}: expected {np.dtype(np_dtype)}, got {cai['typestr']}")
        return int(cai["data"][0])
    if isinstance(a, np.ndarray):
        raise TypeError(f"{where}: expected device memory, got a numpy (host) array")
    if isinstance(a, (int, np.integer)) and not isinstance(a, bool):
        addr = int(a)
        if addr != 0 and not _is_device_address(addr):
            raise TypeError(f"{where}: address {addr:#x} is not device memory")
        return addr
    raise TypeError(f"{where}: cannot take a device address of {type(a).__name__}")


def _host_array(a, dt, where):
    """Host (numpy) array for slot ``where``; device arrays are refused.  The returned array
    must stay referenced until the call returns."""
    torch = _torch()
    np_dtype, _ = _SLOT_DTYPES[dt]
    if isinstance(a, torch.Tensor):
        if a.is_cuda:
            raise TypeError(f"{where}: expected host memory, got a CUDA tensor")
        a = a.numpy()
    if hasattr(a, "__cuda_array_interface__"):
        raise TypeError(f"{where}: expected host memory, got a device array")
    if not isinstance(a, np.ndarray):
        raise TypeError(f"{where}: expected a numpy array, got {type(a).__name__}")
    if a.dtype != np_dtype or not a.flags["C_CONTIGUOUS"]:
        raise TypeError(f"{where}: expected a C-contiguous {np.dtype(np_dtype)} array")
    return a


def _convert(slots, args, name):
    """ctypes arguments for ``args`` per ``slots``; also returns the host arrays to keep alive
    and the host pointer arrays (whose entries are checked to be device addresses)."""
    if len(args) != len(slots):
        raise TypeError(f"{name}: expected {len(slots)} positional arguments, got {len(args)}")
    out, keep = [], []
    for k, (slot, a) in enumerate(zip(slots, args)):
        where = f"{name} argument {k}"
        if slot[0] == "D":
            out.append(ctypes.c_void_p(_device_addr(a, slot[1:], where)))
        elif slot[0] == "H":
            h = _host_array(a, slot[1:], where)
            keep.append(h)
            out.append(ctypes.c_void_p(h.__array_interface__["data"][0]))
        elif slot == "i":
            out.append(ctypes.c_int(int(a)))
        elif slot == "b":
            out.append(ctypes.c_int(1 if bool(a) else 0))
        elif slot == "d":
            out.append(ctypes.c_double(float(a)))
        else:  # pragma: no cover - table error
            raise AssertionError(slot)
    return out, keep


def _check_pointer_arrays(name, args):
    """The int64 pointer arrays of InterpTDI / direct_like hold device addresses of per-binary
    templates and segment indices (waveformbuild.py:188-216, likelihood.py:186-194)."""
    idx = {"InterpTDI_wrap": (0, 13), "direct_like_wrap": (4,)}.get(name, ())
    for k in idx:
        for addr in np.asarray(args[k]).ravel():
            if int(addr) != 0 and not _is_device_address(int(addr)):
                raise TypeError(f"{name} argument {k}: entry {int(addr):#x} is not device memory")


def _method(name):
    cname, slots = _METHODS[name]

    def call(*args):
        cargs, keep = _convert(slots, args, name)
        _check_pointer_arrays(name, args)
        fn = getattr(_lib.lib(), cname)
        _lib.check(fn(*cargs, _lib.stream()), cname)  # direct_like returns with d_h, h_h on the host
        del keep

    call.__name__ = name
    call.__doc__ = f"BBHx backend method {name} on {cname} (include/bbhx_b200.h)."
    return call


class pyFastLISAResponse:
    """The response object of BBHx's backend (lisaresponse.pyx:34-121): orbit tables set by
    ``add_orbit_information`` (host or device arrays; the library keeps its own device copy)
    and ``LISA_response_wrap`` on them."""

    def __init__(self):
        self._h = ctypes.c_void_p()
        _lib.call("bbhx_orbits_create", ctypes.byref(self._h))

    def add_orbit_information(self, dt, N, n_arr, L_arr, x_arr, links, sc_r, sc_e, armlength):
        def host(a, dtype):
            torch = _torch()
            if isinstance(a, torch.Tensor):
                a = a.detach().cpu().numpy()
            elif hasattr(a, "get") and hasattr(a, "__cuda_array_interface__"):
                a = a.get()
            return np.ascontiguousarray(a, dtype=dtype)

        arrs = [host(n_arr, np.float64), host(L_arr, np.float64), host(x_arr, np.float64),
                host(links, np.int32), host(sc_r, np.int32), host(sc_e, np.int32)]
        _lib.call("bbhx_orbits_add_orbit_information", self._h, ctypes.c_double(float(dt)),
                  ctypes.c_int(int(N)), *[_lib.hptr(a) for a in arrs],
                  ctypes.c_double(float(armlength)))

    def LISA_response_wrap(self, *args):
        cargs, keep = _convert(_RESPONSE_SLOTS, args, "LISA_response_wrap")
        _lib.check(_lib.lib().bbhx_LISA_response(self._h, *cargs, _lib.stream()),
                   "bbhx_LISA_response")
        del keep

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().bbhx_orbits_destroy(h)
            except Exception:
                pass
            self._h = None


class B200BackendMethods:
    """The nine backend methods and ``xp`` (attribute names of BBHxBackendMethods,
    src/bbhx/cutils/__init__.py:13-23)."""

    def __init__(self):
        for name in _METHODS:
            setattr(self, name, _method(name))
        self.pyFastLISAResponse = pyFastLISAResponse
        self.xp = _torch()

    def as_dict(self):
        return {name: getattr(self, name) for name in list(_METHODS) + ["pyFastLISAResponse", "xp"]}


def b200_methods():
    """The BBHx backend methods bound to libbbhx_b200.so (one object per call)."""
    return B200BackendMethods()


METHOD_NAMES = tuple(_METHODS) + ("pyFastLISAResponse",)
