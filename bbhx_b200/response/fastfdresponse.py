"""Fast frequency-domain LISA TDI response on the GPU.

Drop-in for the reference's ``LISATDIResponse`` (src/bbhx/response/fastfdresponse.py:26-531):
same constructor keywords (TDItag, orbits, rescaled, tdi2, order_fresnel_stencil), same
``__call__`` arguments and checks, the same flat response buffer with optional amplitude
slot ((8 | 9), B, M, L), and the ``transferL1..3`` / ``phase`` / ``tf`` views.  The orbit
tables are uploaded once, when the object is built (the reference copies them to the
device on every call, Response.cu:700-725).
"""
import ctypes

import numpy as np

from .. import _lib
from ..orbits import EqualArmlengthOrbits, Orbits
from ..utils.arrays import atleast_1d, device, to_dev, torch

ALLOWABLE_MODES = [(2, 2), (3, 3), (4, 4), (2, 1), (3, 2), (4, 3)]


class OrbitHandle:
    """Device copy of an orbit table (``bbhx_orbits_*``)."""

    def __init__(self, orbits):
        self._h = ctypes.c_void_p(0)
        _lib.call("bbhx_orbits_create", ctypes.byref(self._h))
        dt, N, n_arr, L_arr, x_arr, links, sc_r, sc_e, armlength = orbits.pycppdetector_args
        arrs = [np.ascontiguousarray(a) for a in (n_arr, L_arr, x_arr)]
        ints = [np.ascontiguousarray(a, dtype=np.int32) for a in (links, sc_r, sc_e)]
        _lib.call("bbhx_orbits_add_orbit_information", self._h, float(dt), int(N),
                  _lib.hptr(arrs[0], np.float64), _lib.hptr(arrs[1], np.float64),
                  _lib.hptr(arrs[2], np.float64), _lib.hptr(ints[0]), _lib.hptr(ints[1]),
                  _lib.hptr(ints[2]), float(armlength))

    @property
    def ptr(self):
        return self._h

    def __del__(self):
        try:
            if self._h:
                _lib.lib().bbhx_orbits_destroy(self._h)
        except Exception:
            pass


class LISATDIResponse:
    def __init__(self, TDItag="AET", orbits=None, rescaled=False, tdi2=False,
                 order_fresnel_stencil=0, force_backend=None):
        t = torch()
        self.rescaled = rescaled
        self.tdi2 = tdi2
        if order_fresnel_stencil > 0:
            raise NotImplementedError
        self.order_fresnel_stencil = order_fresnel_stencil
        self.TDItag = TDItag
        self.TDItag_int = 1 if TDItag == "XYZ" else 2
        self.allowable_modes = list(ALLOWABLE_MODES)
        self.ells_default = to_dev([2, 3, 4, 2, 3, 4], t.int32)
        self.mms_default = to_dev([2, 3, 4, 1, 2, 3], t.int32)
        self.orbits = orbits
        self.orbit_handle = OrbitHandle(self._orbits)

    @property
    def xp(self):
        return torch()

    @property
    def orbits(self):
        return self._orbits

    @orbits.setter
    def orbits(self, orbits):
        if orbits is None:
            self._orbits = EqualArmlengthOrbits()
        elif not isinstance(orbits, Orbits):
            raise ValueError("Input orbits must be of type Orbits.")
        else:
            self._orbits = orbits
        self._orbits.configure(linear_interp_setup=True)

    def _sanity_check_modes(self, ells, mms):
        for ell, mm in zip(ells, mms):
            if (int(ell), int(mm)) not in self.allowable_modes:
                raise ValueError(
                    "Requested mode [(l,m) = ({},{})] is not available. Allowable modes include {}"
                    .format(ell, mm, self.allowable_modes))

    def _slot(self, k):
        n = self.num_per_param
        return self.response_carrier[(self.includes_amps + k) * n:(self.includes_amps + k + 1) * n]

    def _shape(self, a):
        return a.reshape(self.num_bin_all, self.num_modes, self.length)

    @property
    def transferL1(self):
        return self._shape(self._slot(2)) + 1j * self._shape(self._slot(3))

    @property
    def transferL2(self):
        return self._shape(self._slot(4)) + 1j * self._shape(self._slot(5))

    @property
    def transferL3(self):
        return self._shape(self._slot(6)) + 1j * self._shape(self._slot(7))

    @property
    def phase(self):
        return self._shape(self._slot(0))

    @property
    def tf(self):
        return self._shape(self._slot(1))

    def __call__(self, freqs, inc, lam, beta, psi, phi_ref, length, modes=None, phase=None,
                 tf=None, out_buffer=None, adjust_phase=True, direct=False):
        t = torch()
        inc = to_dev(atleast_1d(inc)).clone()
        lam = to_dev(atleast_1d(lam)).clone()
        beta = to_dev(atleast_1d(beta)).clone()
        psi = to_dev(atleast_1d(psi)).clone()
        phi_ref = to_dev(atleast_1d(phi_ref)).clone()
        if modes is not None:
            ells = to_dev([ell for ell, mm in modes], t.int32)
            mms = to_dev([mm for ell, mm in modes], t.int32)
            self._sanity_check_modes([e for e, _ in modes], [m for _, m in modes])
            self.modes = list(modes)
        else:
            ells, mms = self.ells_default, self.mms_default
            self.modes = list(self.allowable_modes)
        num_modes = len(ells)
        num_bin_all = len(inc)
        self.length = length
        self.num_modes = num_modes
        self.num_bin_all = num_bin_all
        self.num_per_param = length * num_modes * num_bin_all
        self.num_per_bin = length * num_modes
        self.nresponse_params = 6
        if out_buffer is None and phase is None and tf is None:
            raise ValueError("Must provide either out_buffer or both phase and tf.")
        if out_buffer is None:
            includes_amps = 0
            self.nparams = includes_amps + 2 + self.nresponse_params
            self.response_carrier = t.zeros(self.nparams * self.num_per_param, dtype=t.float64,
                                            device=device())
        else:
            nparams_empirical = len(out_buffer) / (self.num_bin_all * self.num_modes * self.length)
            if np.allclose(nparams_empirical, np.round(nparams_empirical)) and int(nparams_empirical) in [8, 9]:
                self.nparams = int(nparams_empirical)
            else:
                raise ValueError(
                    f"out_buffer incorrect length. The length should be equivalent to (8 or 9) * "
                    f"{self.num_bin_all * self.num_modes * self.length}. Given length is {len(out_buffer)}.")
            includes_amps = 1 if self.nparams == 9 else 0
            self.response_carrier = out_buffer
        self.includes_amps = includes_amps
        freqs = to_dev(freqs)
        if freqs.ndim > 1:
            if tuple(freqs.shape) != (self.num_bin_all, self.num_modes, self.length):
                raise ValueError(
                    f"freqs have incorrect shape. Shape should be {(self.num_bin_all, self.num_modes, self.length)}. "
                    f"Current shape is {tuple(freqs.shape)}.")
            freqs = freqs.flatten()
        elif len(freqs) != self.num_per_param:
            raise ValueError(
                f"freqs incorrect length. The length should be equivalent to {self.num_per_param}. "
                f"Given length is {len(freqs)}.")
        self.freqs = freqs
        tmin, tmax = float(self.orbits.t_base.min()), float(self.orbits.t_base.max())
        use_phase_tf = False
        if phase is not None and tf is not None:
            use_phase_tf = True
            tf_d = to_dev(tf)
            ph_d = to_dev(phase)
            if not direct and (float(tf_d.min()) < tmin or float(tf_d.max()) > tmax):
                raise ValueError(
                    f"Orbital information does not cover minimum ({float(tf_d.min())}) and maximum "
                    f"({float(tf_d.max())}) tf. Orbital information begins at {tmin} and ends at {tmax}.")
            if tuple(ph_d.shape) != tuple(tf_d.shape):
                raise ValueError("Shape of phase array and tf array need to be the same shape.")
            if ph_d.numel() != self.num_per_param:
                raise ValueError(f"phase incorrect length. The length should be equivalent to {self.num_per_param}.")
            self._slot(0).copy_(ph_d.flatten())
            self._slot(1).copy_(tf_d.flatten())
        elif phase is not None or tf is not None:
            raise ValueError("If provided phase or tf, need to provide both.")
        else:
            if not direct:
                tfs = self._slot(1)
                lo, hi = float(tfs.min()), float(tfs.max())
                if lo < tmin or hi > tmax:
                    raise ValueError(
                        f"Orbital information does not cover minimum ({lo}) and maximum ({hi}) tf. "
                        f"Orbital information begins at {tmin} and ends at {tmax}.")
        _lib.call("bbhx_LISA_response", self.orbit_handle.ptr, _lib.dptr(self.response_carrier),
                  _lib.dptr(ells), _lib.dptr(mms), _lib.dptr(self.freqs), _lib.dptr(phi_ref),
                  _lib.dptr(inc), _lib.dptr(lam), _lib.dptr(beta), _lib.dptr(psi), self.TDItag_int,
                  int(self.rescaled), int(self.tdi2), self.order_fresnel_stencil, num_modes, length,
                  num_bin_all, includes_amps, _lib.stream())
        if use_phase_tf and adjust_phase and isinstance(phase, t.Tensor) and phase.is_cuda:
            phase.copy_(self._slot(0).reshape(phase.shape))
