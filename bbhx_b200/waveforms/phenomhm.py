"""PhenomHM / PhenomD in the amplitude-phase representation on the GPU.

Drop-in for the reference's ``PhenomHMAmpPhase`` (src/bbhx/waveforms/phenomhm.py:32-614):
same constructor keywords, ``run_wave`` / ``__call__`` arguments, flat
``waveform_carrier`` layout ``[3, B, M, L]`` (amp, phase, t(f)) and the ``amp`` /
``phase`` / ``tf`` / ``freqs`` / ``freqs_shaped`` views.  Arrays are torch CUDA tensors.

Differences in mechanism (not in results): the per-(binary, mode) model setup runs once
and is shared by the two evaluations of ``__call__`` (the reference re-runs the whole
model on the regridded frequencies), the first pass evaluates t(f) only, the t_ref shift
is fused into the evaluation kernel, and the observation-window regrid runs on the GPU.
"""
import numpy as np

from .. import _lib
from ..utils.arrays import atleast_1d, device, to_dev, torch
from ..utils.constants import YRSID_SI
from .ringdownphenomd import QNMData_a, QNMData_fdamp, QNMData_fring, dspin

ALLOWABLE_MODES = [(2, 2), (3, 3), (4, 4), (2, 1), (3, 2), (4, 3)]


def qnm_spline_table():
    """(8, 1001) device table: y, c1, c2, c3 of the not-a-knot spline of the ringdown and of
    the damping frequency over final spin (phenomhm.py:148-163), built with the library's
    spline kernel."""
    t = torch()
    x = to_dev(QNMData_a).reshape(1, -1)
    y = to_dev(np.stack([QNMData_fring, QNMData_fdamp])).reshape(2, 1, -1).contiguous()
    n = x.shape[1]
    c1 = t.empty((2, 1, n), dtype=t.float64, device=device())
    c2 = t.empty_like(c1)
    c3 = t.empty_like(c1)
    _lib.call("bbhx_interpolate", _lib.dptr(x), _lib.dptr(y), _lib._VP(0), _lib.dptr(c1),
              _lib.dptr(c2), _lib.dptr(c3), n, 2, 1, 1, _lib.stream())
    tab = t.stack([y[0, 0], c1[0, 0], c2[0, 0], c3[0, 0], y[1, 0], c1[1, 0], c2[1, 0], c3[1, 0]])
    return tab.contiguous()


CHI1_MSG = "chi1z array contains values with abs(chi1z) > 1.0 which is not allowed."
CHI2_MSG = "chi2z array contains values with abs(chi2z) > 1.0 which is not allowed."


def raise_chi_flag(code):
    """The reference's spin-range errors (phenomhm.py:168-185) from the flag bits set by the
    step front end (1: chi1z, 2: chi2z; chi1z is reported first, as the reference checks it
    first)."""
    if code & 1:
        raise ValueError(CHI1_MSG)
    if code & 2:
        raise ValueError(CHI2_MSG)


def step_front(m1, m2, chi1z, chi2z, lam=None, beta=None, num_modes=1, t_obs=(0.0, 0.0),
               flags=None):
    """Per-binary front end of a step in one kernel (bbhx_step_front): m1 >= m2 ordering with
    the spins swapped alongside, SI masses and the |chi| <= 1 check (phenomhm.py:175-199), and,
    when lam / beta are given, the SSB observation limits (waveformbuild.py:477-484) and the
    per-(binary, mode) spans the window regrid reads.  ``flags`` (device int32 [3]) is cleared
    and receives the spin check (flags[2] bits 1 / 2); without it the check raises here.
    Returns (pars [6, B] = m1, m2, chi1z, chi2z, m1_SI, m2_SI; t_start, t_end, tobs_rows)."""
    t = torch()
    cols = [to_dev(atleast_1d(v)).contiguous() for v in (m1, m2, chi1z, chi2z)]
    B = cols[0].numel()
    if any(c.numel() != B for c in cols):
        raise ValueError("all parameter arrays must have the same length")
    pars = t.empty((6, B), dtype=t.float64, device=device())
    own = flags is None
    fl = t.empty(3, dtype=t.int32, device=device()) if own else flags
    ts = te = tob = None
    if lam is not None:
        lam = to_dev(atleast_1d(lam)).contiguous()
        beta = to_dev(atleast_1d(beta)).contiguous()
        ts = t.empty(B, dtype=t.float64, device=device())
        te = t.empty(B, dtype=t.float64, device=device())
        tob = t.empty(B * num_modes, dtype=t.float64, device=device())
    _lib.call("bbhx_step_front", _lib.dptr(pars), _lib.dptr(ts), _lib.dptr(te), _lib.dptr(tob),
              *[_lib.dptr(c) for c in cols], _lib.dptr(lam), _lib.dptr(beta), B, num_modes,
              float(t_obs[0] * YRSID_SI), float(t_obs[1] * YRSID_SI), _lib.dptr(fl),
              int(fl.numel()), _lib.stream())
    if own:
        raise_chi_flag(int(fl[2].item()))
    return pars, ts, te, tob


class PhenomHMAmpPhase:
    """PhenomHM amplitude, phase and t(f) for batches of binaries.

    Args:
        force_backend: accepted for call compatibility; only the CUDA backend exists.
        run_phenomd (bool): run PhenomD (only the (2,2) mode).
        mf_min, mf_max (float): dimensionless frequency range of the default grid.
        initial_t_val (float): start of the time window; shifts the phase only.
    """

    def __init__(self, force_backend=None, run_phenomd=False, mf_min=1e-4, mf_max=0.6,
                 initial_t_val=0.0):
        t = torch()
        self.run_phenomd = run_phenomd
        self.allowable_modes = [(2, 2)] if run_phenomd else list(ALLOWABLE_MODES)
        self.ells_default = to_dev([ell for ell, _ in self.allowable_modes], t.int32)
        self.mms_default = to_dev([mm for _, mm in self.allowable_modes], t.int32)
        self.mf_min = mf_min
        self.mf_max = mf_max
        self.initial_t_val = initial_t_val
        self._init_phenomd_fring_spline()
        self._coeffs = None

    @property
    def xp(self):
        return torch()

    def _init_phenomd_fring_spline(self):
        self.qnm_table = qnm_spline_table()
        (self.y_rd, self.c1_rd, self.c2_rd, self.c3_rd,
         self.y_dm, self.c1_dm, self.c2_dm, self.c3_dm) = self.qnm_table

    # ------------------------------------------------------------------ checks
    def _sanity_check_modes(self, ells, mms):
        for ell, mm in zip(ells, mms):
            if (int(ell), int(mm)) not in self.allowable_modes:
                raise ValueError(
                    "Requested mode [(l,m) = ({},{})] is not available. Allowable modes include {}"
                    .format(ell, mm, self.allowable_modes))

    # ------------------------------------------------------------------ views
    @property
    def amp(self):
        return self.waveform_carrier[0: self.num_per_param].reshape(
            self.num_bin_all, self.num_modes, self.length)

    @property
    def phase(self):
        return self.waveform_carrier[self.num_per_param: 2 * self.num_per_param].reshape(
            self.num_bin_all, self.num_modes, self.length)

    @property
    def tf(self):
        return self.waveform_carrier[2 * self.num_per_param: 3 * self.num_per_param].reshape(
            self.num_bin_all, self.num_modes, self.length)

    @property
    def freqs_shaped(self):
        return self._freqs.reshape(self.num_bin_all, self.num_modes, self.length)

    @property
    def freqs(self):
        return self._freqs

    @freqs.setter
    def freqs(self, f):
        self._freqs = f.flatten() if f.ndim > 1 else f

    # ------------------------------------------------------------------ core
    def _prepare(self, m1, m2, chi1z, chi2z, distance, phi_ref, f_ref, t_ref, length, freqs,
                 out_buffer, modes, flags=None, front=None):
        """Shared front half of run_wave: parameter checks, modes, buffers, ringdown
        frequencies and the per-(binary, mode) model records."""
        t = torch()
        self._setup_records(m1, m2, chi1z, chi2z, distance, t_ref, modes, flags, front)
        m1, m2 = self._m1, self._m2
        num_modes, num_bin_all, mms = self.num_modes, self.num_bin_all, self.mms
        self.length = length
        self.nparams = 3
        self.num_per_param = length * num_modes * num_bin_all
        self.num_per_bin = length * num_modes
        if out_buffer is None:
            self.waveform_carrier = t.zeros(self.nparams * self.num_per_param, dtype=t.float64,
                                            device=device())
        else:
            self.waveform_carrier = out_buffer
        if freqs is None:
            f = t.empty(self.num_per_param, dtype=t.float64, device=device())
            _lib.call("bbhx_default_freqs", _lib.dptr(f), _lib.dptr(m1), _lib.dptr(m2),
                      _lib.dptr(mms), float(self.mf_min), float(self.mf_max), num_modes, length,
                      num_bin_all, _lib.stream())
            self.freqs = f
        else:
            freqs = to_dev(freqs)
            if freqs.ndim == 1:
                self.freqs = freqs.reshape(1, 1, -1).expand(num_bin_all, num_modes, -1).flatten()
            elif freqs.ndim == 3:
                self.freqs = freqs.flatten().clone()
            else:
                raise ValueError(
                    "If providing freqs, must be 1D array (length,) or 3D array (length, num_modes, length).")

    def _setup_records(self, m1, m2, chi1z, chi2z, distance, t_ref, modes, flags=None,
                       front=None):
        """Parameter checks, mode list, ringdown frequencies and the per-(binary, mode)
        model records (``self._coeffs``), without any frequency grid or output buffer.
        ``front``: the [6, B] output of step_front when the caller already ran it."""
        t = torch()
        pars = front if front is not None else step_front(m1, m2, chi1z, chi2z, flags=flags)[0]
        m1, m2, chi1z, chi2z, m1_SI, m2_SI = pars
        ells, mms = self.mode_tensors(modes)
        self.modes = modes if (modes is not None and not self.run_phenomd) else self.allowable_modes
        self.ells, self.mms = ells, mms
        num_modes = len(ells)
        num_bin_all = len(m1)
        self.num_modes = num_modes
        self.num_bin_all = num_bin_all
        distance = to_dev(atleast_1d(distance))
        self.t_ref_dev = to_dev(atleast_1d(t_ref))
        if distance.numel() != num_bin_all or self.t_ref_dev.numel() != num_bin_all:
            raise ValueError("all parameter arrays must have the same length")
        ncol = 1 if self.run_phenomd else num_modes + 1
        self.fringdown = t.empty(num_bin_all * ncol, dtype=t.float64, device=device())
        self.fdamp = t.empty_like(self.fringdown)
        tab = self.qnm_table
        _lib.call("bbhx_ringdown_frequencies_all", _lib.dptr(self.fringdown), _lib.dptr(self.fdamp),
                  _lib.dptr(m1), _lib.dptr(m2), _lib.dptr(chi1z), _lib.dptr(chi2z), _lib.dptr(ells),
                  _lib.dptr(mms), num_modes, num_bin_all, _lib.dptr(tab), tab.shape[1],
                  float(dspin), int(self.run_phenomd), _lib.stream())
        nbytes = int(_lib.lib().bbhx_mode_coeffs_bytes())
        self._coeffs = t.empty(num_bin_all * num_modes * nbytes, dtype=t.uint8, device=device())
        _lib.call("bbhx_phenomhm_setup", _lib.dptr(self._coeffs), _lib.dptr(ells), _lib.dptr(mms),
                  _lib.dptr(m1_SI), _lib.dptr(m2_SI), _lib.dptr(chi1z), _lib.dptr(chi2z),
                  _lib.dptr(distance), _lib.dptr(self.fringdown), _lib.dptr(self.fdamp), num_modes,
                  num_bin_all, int(self.run_phenomd), _lib.stream())
        self._m1, self._m2 = m1, m2

    def mode_tensors(self, modes):
        """Device (ells, mms) int32 tensors of a mode list (None: all allowable modes; (2, 2)
        only for PhenomD), made once per list so that no host copy happens inside a CUDA graph
        capture."""
        t = torch()
        cache = self.__dict__.setdefault("_mode_tensors", {})
        key = None
        if modes is not None:
            key = tuple(tuple(md) for md in modes)
            if key not in cache:
                self._sanity_check_modes([e for e, _ in modes], [m for _, m in modes])
                cache[key] = (to_dev([ell for ell, mm in modes], t.int32),
                              to_dev([mm for ell, mm in modes], t.int32))
        if self.run_phenomd:
            if "phenomd" not in cache:
                cache["phenomd"] = (to_dev([2], t.int32), to_dev([2], t.int32))
            return cache["phenomd"]
        return cache[key] if key is not None else (self.ells_default, self.mms_default)

    def _evaluate(self):
        _lib.call("bbhx_phenomhm_points", _lib.dptr(self.waveform_carrier), _lib.dptr(self._freqs),
                  _lib.dptr(self._coeffs), _lib.dptr(self.t_ref_dev), float(self.initial_t_val),
                  self.num_modes, self.length, self.num_bin_all, _lib.stream())

    def run_wave(self, m1, m2, chi1z, chi2z, distance, phi_ref, f_ref, t_ref, length, freqs=None,
                 out_buffer=None, modes=None):
        """Generate amplitude, phase and t(f) (phenomhm.py:270-507 semantics)."""
        self._prepare(m1, m2, chi1z, chi2z, distance, phi_ref, f_ref, t_ref, length, freqs,
                      out_buffer, modes)
        self._evaluate()

    def _tobs_rows(self, Tobs):
        t = torch()
        B, M = self.num_bin_all, self.num_modes
        if Tobs is None:
            return t.full((B * M,), 1e300, dtype=t.float64, device=device())
        if isinstance(Tobs, float):
            return t.full((B * M,), Tobs, dtype=t.float64, device=device())
        Tobs_np = Tobs
        if isinstance(Tobs, np.ndarray) or isinstance(Tobs, t.Tensor):
            To = to_dev(Tobs)
            if To.ndim == 1:
                assert To.shape[0] == B
                return To.reshape(B, 1).expand(B, M).flatten().contiguous()
            if To.ndim == 2:
                assert tuple(To.shape) == (B, M)
                return To.flatten().contiguous()
        raise ValueError(f"Tobs entered incorrectly: {type(Tobs_np)}")

    def __call__(self, *args, Tobs=None, direct=False, **kwargs):
        """``run_wave`` plus, unless ``direct``, the regrid onto the frequency band where
        0 <= t(f) <= Tobs (phenomhm.py:509-614)."""
        t = torch()
        names = ["m1", "m2", "chi1z", "chi2z", "distance", "phi_ref", "f_ref", "t_ref", "length"]
        kw = dict(zip(names, args))
        kw.update(kwargs)
        kw.setdefault("freqs", None)
        kw.setdefault("out_buffer", None)
        kw.setdefault("modes", None)
        self._prepare(**kw)
        if direct:
            self._evaluate()
            return
        n = self.num_per_param
        tf0 = t.empty(n, dtype=t.float64, device=device())
        _lib.call("bbhx_phenomhm_tf", _lib.dptr(tf0), _lib.dptr(self._freqs), _lib.dptr(self._coeffs),
                  _lib.dptr(self.t_ref_dev), self.num_modes, self.length, self.num_bin_all,
                  _lib.stream())
        rows = self.num_bin_all * self.num_modes
        new_f = t.empty(n, dtype=t.float64, device=device())
        fminmax = t.empty(2 * rows, dtype=t.float64, device=device())
        err = t.zeros(1, dtype=t.int32, device=device())
        tobs_rows = self._tobs_rows(Tobs)
        _lib.call("bbhx_tf_window_regrid", _lib.dptr(new_f), _lib.dptr(fminmax), _lib.dptr(self._freqs),
                  _lib.dptr(tf0), _lib.dptr(tobs_rows), self.length, rows,
                  _lib.dptr(err), _lib.stream())
        e = int(err.item())
        if e == 1:
            raise ValueError(
                "The search for a window at x_min did not run correctly. If t_ref is close to zero, "
                "the time-frequency correspondence may be crossing zero twice.")
        if e == 2:
            raise ValueError(
                "The search for a window at x_max did not run correctly. If t_ref is close to the "
                "observation time, the time-frequency correspondence may be crossing zero twice.")
        self._freqs = new_f
        self._evaluate()
