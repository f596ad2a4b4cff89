"""Waveform assembly: PhenomHM -> TDI response -> spline -> data grid.

Drop-ins for the reference's ``TemplateInterpFD`` and ``BBHWaveformFD``
(src/bbhx/waveformbuild.py:36-700) with the same call signatures, keyword branches
(direct / compress / squeeze / fill / combine) and return shapes.  Arrays are torch CUDA
tensors.

``BBHWaveformFD.inner_products`` is the fused device path the likelihood uses: the
PhenomHM records are built once, the first pass evaluates only t(f), the window regrid,
waveform and response run in one fused kernel, the spline solve in one kernel, and the
interpolation, mode sum, noise weighting and <d|h>, <h|h> reduction in one kernel; no
template is ever stored and no host synchronisation happens before the caller reads the
results.
"""
import warnings

import numpy as np

from . import _lib
from .response.fastfdresponse import LISATDIResponse
from .utils.arrays import atleast_1d, device, to_dev, to_np, torch
from .utils.constants import YRSID_SI
from .utils.interpolate import CubicSplineInterpolant
from .waveforms.phenomhm import PhenomHMAmpPhase, step_front


# arithmetic of the fused direct likelihood: "fp64" (parity form) or "mixed" (FP64 phase,
# t(f) and accumulations; FP32 amplitude, transfer functions and per-bin products)
PRECISIONS = {"fp64": 0, "mixed": 1}


class TemplateInterpFD:
    """Interpolate the sparse (amp, phase, t(f), transfer) representation onto a data grid
    (waveformbuild.py:36-239)."""

    def __init__(self, force_backend=None):
        pass

    @property
    def xp(self):
        return torch()

    @property
    def template_channels(self):
        return [self.template_carrier[i].reshape(self.num_channels, int(self.lengths[i]))
                for i in range(self.num_bin_all)]

    def __call__(self, data_freqs, interp_container, t_start, t_end, length, num_modes,
                 num_channels):
        t = torch()
        num_bin_all = len(t_start)
        self.length = length
        self.num_modes = num_modes
        self.num_bin_all = num_bin_all
        self.data_length = len(data_freqs)
        self.num_channels = num_channels
        data_freqs = to_dev(data_freqs)
        (freqs, y, c1, c2, c3) = [to_dev(a) for a in interp_container]
        freqs_shaped = freqs.reshape(num_bin_all, num_modes, -1)
        lo = freqs_shaped.reshape(num_bin_all, -1).min(dim=1).values
        hi = freqs_shaped.reshape(num_bin_all, -1).max(dim=1).values
        se = t.searchsorted(data_freqs, t.stack([lo, hi], dim=1).contiguous(), right=True)
        se_h = to_np(se).astype(np.int64)
        inds = []
        for i, (st, et) in enumerate(se_h):
            v = data_freqs[st:et].reshape(1, -1).expand(num_modes, -1).contiguous()
            inds.append((t.searchsorted(freqs_shaped[i].contiguous(), v, right=True) - 1)
                        .to(t.int32).flatten().contiguous())
        self.lengths = lengths = np.asarray([len(x) // num_modes for x in inds], dtype=np.int32)
        self.start_inds = start_inds = se_h[:, 0].astype(np.int32).copy()
        ptrs = np.asarray([x.data_ptr() for x in inds], dtype=np.int64)
        self.template_carrier = [t.zeros(int(num_channels * L), dtype=t.complex128, device=device())
                                 for L in lengths]
        tptrs = np.asarray([x.data_ptr() for x in self.template_carrier], dtype=np.int64)
        ts = np.ascontiguousarray(to_np(t_start), dtype=np.float64)
        te = np.ascontiguousarray(to_np(t_end), dtype=np.float64)
        self._inds = inds
        _lib.call("bbhx_InterpTDI", _lib.hptr(tptrs), _lib.dptr(data_freqs), _lib.dptr(freqs),
                  _lib.dptr(y), _lib.dptr(c1), _lib.dptr(c2), _lib.dptr(c3), _lib.hptr(ts),
                  _lib.hptr(te), length, self.data_length, num_bin_all, num_modes, _lib.hptr(ptrs),
                  _lib.hptr(start_inds), _lib.hptr(lengths), _lib.stream())
        return self.template_channels


class BBHWaveformFD:
    """PhenomHM + fast LISA response, interpolated or direct (waveformbuild.py:242-700)."""

    def __init__(self, amp_phase_kwargs=None, response_kwargs=None, interp_kwargs=None,
                 force_backend=None):
        amp_phase_kwargs = amp_phase_kwargs or {}
        response_kwargs = response_kwargs or {}
        interp_kwargs = interp_kwargs or {}
        self.force_backend = force_backend
        self.amp_phase_gen = PhenomHMAmpPhase(**amp_phase_kwargs)
        self.response_gen = LISATDIResponse(**response_kwargs)
        self.num_interp_params = 9
        self.interp_response = TemplateInterpFD(**interp_kwargs)

    @property
    def xp(self):
        return torch()

    # ------------------------------------------------------------------ helpers
    def _sparse_buffer(self, params, t_obs_start, t_obs_end, freqs, length, modes, direct,
                       flags=None):
        """Fill the [9, B, M, L] sparse buffer (amp, phase, t(f), 6 transfer slots).

        Non-direct: default grid -> t(f) -> window regrid -> fused waveform + response.
        Direct: waveform + response at the given frequencies.  When ``flags`` (device int32
        [2]) is given, the window-search failure and the orbit-coverage violation are
        recorded there instead of raising, so the caller can defer the host sync."""
        t = torch()
        (m1, m2, chi1z, chi2z, distance, phi_ref, f_ref, inc, lam, beta, psi, t_ref) = params
        if freqs is None and length is None:
            raise ValueError("Must input freqs or length.")
        ap = self.amp_phase_gen
        if direct:
            length = freqs.shape[-1] if freqs is not None else length
        M = len(modes) if modes is not None else len(ap.allowable_modes)
        # mass ordering, spin check, SSB observation limits and per-row spans in one kernel
        pars, t_start, t_end, tobs_rows = step_front(m1, m2, chi1z, chi2z, lam, beta, M,
                                                     (t_obs_start, t_obs_end), flags=flags)
        B = pars.shape[1]
        # every slot of every (binary, mode, frequency) is written by the fused waveform +
        # response kernel below, so the buffer is not cleared first
        out_buffer = t.empty(9 * length * M * B, dtype=t.float64, device=device())
        ap._prepare(m1, m2, chi1z, chi2z, distance, None, f_ref, t_ref, length,
                    freqs if direct else None, out_buffer, modes, flags=flags, front=pars)
        M = ap.num_modes
        if not direct:
            n = ap.num_per_param
            tf0 = t.empty(n, dtype=t.float64, device=device())
            _lib.call("bbhx_phenomhm_tf", _lib.dptr(tf0), _lib.dptr(ap._freqs), _lib.dptr(ap._coeffs),
                      _lib.dptr(ap.t_ref_dev), M, length, B, _lib.stream())
            rows = B * M
            new_f = t.empty(n, dtype=t.float64, device=device())
            fminmax = t.empty(2 * rows, dtype=t.float64, device=device())
            err = flags if flags is not None else t.zeros(2, dtype=t.int32, device=device())
            _lib.call("bbhx_tf_window_regrid", _lib.dptr(new_f), _lib.dptr(fminmax),
                      _lib.dptr(ap._freqs), _lib.dptr(tf0), _lib.dptr(tobs_rows), length, rows,
                      _lib.dptr(err), _lib.stream())
            if flags is None:
                e = int(err[0].item())
                if e:
                    raise ValueError("The search for a window at x_%s did not run correctly."
                                     % ("min" if e == 1 else "max"))
            # what the regrid read, for the knots' derivative in direct_grad
            self._regrid_inputs = (ap._freqs, tf0)
            ap._freqs = new_f
        rg = self.response_gen
        inc_d, lam_d, beta_d, psi_d, phi_d = (to_dev(atleast_1d(v)) for v in (inc, lam, beta, psi, phi_ref))
        _lib.call("bbhx_waveform_response_fused", rg.orbit_handle.ptr, _lib.dptr(out_buffer),
                  _lib.dptr(ap._freqs), _lib.dptr(ap._coeffs), _lib.dptr(ap.ells), _lib.dptr(ap.mms),
                  _lib.dptr(phi_d), _lib.dptr(inc_d), _lib.dptr(lam_d), _lib.dptr(beta_d),
                  _lib.dptr(psi_d), _lib.dptr(ap.t_ref_dev), float(ap.initial_t_val),
                  rg.TDItag_int, int(rg.rescaled), int(rg.tdi2), M, length, B, _lib.stream())
        if not direct:
            tfs = out_buffer[2 * B * M * length:3 * B * M * length]
            tmin, tmax = float(rg.orbits.t_base.min()), float(rg.orbits.t_base.max())
            if flags is not None:
                _lib.call("bbhx_tf_range_check", _lib.dptr(tfs), tfs.numel(), tmin, tmax,
                          _lib._VP(flags.data_ptr() + 4), _lib.stream())
            else:
                lo, hi = float(tfs.min()), float(tfs.max())
                if lo < tmin or hi > tmax:
                    raise ValueError(
                        f"Orbital information does not cover minimum ({lo}) and maximum ({hi}) tf. "
                        f"Orbital information begins at {tmin} and ends at {tmax}.")
        # expose the reference's views
        ap.waveform_carrier = out_buffer
        rg.response_carrier = out_buffer
        rg.includes_amps = 1
        rg.num_bin_all, rg.num_modes, rg.length = B, M, length
        rg.num_per_param = B * M * length
        self.num_bin_all, self.num_modes, self.length = B, M, length
        self.out_buffer_final = out_buffer.reshape(9, B, M, length)
        return out_buffer, t_start, t_end

    # ------------------------------------------------------------------ public API
    def __call__(self, m1, m2, chi1z, chi2z, distance, phi_ref, f_ref, inc, lam, beta, psi, t_ref,
                 t_obs_start=0.0, t_obs_end=1.0, freqs=None, length=None, modes=None,
                 shift_t_limits=True, direct=False, compress=True, squeeze=False, fill=False,
                 combine=False):
        t = torch()
        if shift_t_limits is False:
            warnings.warn("Deprecated: shift_t_limits. The option is permanently True.")
        if modes is not None and not isinstance(modes, list):
            raise ValueError("modes must be a list.")
        params = (m1, m2, chi1z, chi2z, distance, phi_ref, f_ref, inc, lam, beta, psi, t_ref)
        if freqs is None and length is None:
            raise ValueError("Must input freqs or length.")
        if not direct:
            if length is None:
                raise ValueError("If direct is False, length parameter must be given.")
            self.data_length = len(freqs)
        buf, t_start, t_end = self._sparse_buffer(params, t_obs_start, t_obs_end, freqs, length,
                                                  modes, direct)
        B, M, L = self.num_bin_all, self.num_modes, self.length
        t_start_d, t_end_d = to_dev(t_start), to_dev(t_end)
        if direct and compress:
            tc = t.zeros(B * 3 * L, dtype=t.complex128, device=device())
            _lib.call("bbhx_direct_sum", _lib.dptr(tc), _lib.dptr(buf), B, L, 3, M,
                      _lib.dptr(t_start_d), _lib.dptr(t_end_d), _lib.stream())
            out = tc.reshape(B, 3, L)
            return out.squeeze() if squeeze else out
        if direct:
            out = t.zeros((B, 3, M, L), dtype=t.complex128, device=device())
            for mode_i in range(M):
                tc = t.zeros(B * 3 * L, dtype=t.complex128, device=device())
                bm = self.out_buffer_final[:, :, mode_i, :].contiguous().flatten()
                _lib.call("bbhx_direct_sum", _lib.dptr(tc), _lib.dptr(bm), B, L, 3, 1,
                          _lib.dptr(t_start_d), _lib.dptr(t_end_d), _lib.stream())
                out[:, :, mode_i, :] += tc.reshape(B, 3, L)
            return out.squeeze() if squeeze else out
        spline = CubicSplineInterpolant(self.amp_phase_gen.freqs, buf, length=L,
                                        num_interp_params=9, num_modes=M, num_bin_all=B)
        template_channels = self.interp_response(freqs, spline.container, t_start, t_end, L, M, 3)
        if fill:
            # placement on the full grid in one kernel (waveformbuild.py:663-693 loops over
            # binaries): combined into [3, N] in binary order, or one row per binary
            nf = len(freqs)
            ir = self.interp_response
            tptrs = np.asarray([x.data_ptr() for x in ir.template_carrier], dtype=np.int64)
            starts = np.ascontiguousarray(ir.start_inds, dtype=np.int32)
            lengths = np.ascontiguousarray(ir.lengths, dtype=np.int32)
            shape = (3, nf) if combine else (B, 3, nf)
            data_out = t.zeros(shape, dtype=t.complex128, device=device())
            _lib.call("bbhx_fill_templates", _lib.dptr(data_out), _lib.hptr(tptrs),
                      _lib.hptr(starts), _lib.hptr(lengths), B, nf, int(bool(combine)),
                      _lib.stream())
            if combine:
                return data_out.squeeze() if squeeze else data_out
            return data_out
        return (template_channels, self.interp_response.start_inds, self.interp_response.lengths)

    def heterodyne_setup(self, params, freqs, h0, constants, t_obs_start=0.0, t_obs_end=1.0,
                         modes=None, flags=None):
        """Everything a fused heterodyned evaluation of the walkers ``params`` reads, without
        the evaluation: per-walker model records, observation limits and the output tensors.
        Returns the arguments of ``bbhx_hdyn_fused`` (after ``orbits``, before ``precision``)
        by name; the tensors stay referenced by the returned dict."""
        t = torch()
        (m1, m2, chi1z, chi2z, distance, phi_ref, f_ref, inc, lam, beta, psi, t_ref) = params
        ap = self.amp_phase_gen
        pars, ts_d, te_d, _ = step_front(m1, m2, chi1z, chi2z, lam, beta, 1,
                                         (t_obs_start, t_obs_end), flags=flags)
        ap._setup_records(m1, m2, chi1z, chi2z, distance, t_ref, modes, flags=flags, front=pars)
        B, M, L = ap.num_bin_all, ap.num_modes, int(freqs.numel())
        rg = self.response_gen
        inc_d, lam_d, beta_d, psi_d, phi_d = (to_dev(atleast_1d(v)) for v in (inc, lam, beta, psi, phi_ref))
        return dict(d_h=t.empty(B, dtype=t.complex128, device=device()),
                    h_h=t.empty(B, dtype=t.complex128, device=device()),
                    coeffs=ap._coeffs, ells=ap.ells, mms=ap.mms, phi_ref=phi_d, inc=inc_d,
                    lam=lam_d, beta=beta_d, psi=psi_d, t_ref=ap.t_ref_dev,
                    t_init=float(ap.initial_t_val), t_start=ts_d, t_end=te_d, freqs=freqs, h0=h0,
                    consts=constants, TDItag=rg.TDItag_int, rescaled=int(rg.rescaled),
                    tdi2=int(rg.tdi2), num_modes=M, length=L, num_bin_all=B)

    HDYN_ARGS = ("d_h", "h_h", "coeffs", "ells", "mms", "phi_ref", "inc", "lam", "beta", "psi",
                 "t_ref", "t_init", "t_start", "t_end", "freqs", "h0", "consts", "TDItag",
                 "rescaled", "tdi2", "num_modes", "length", "num_bin_all")

    def heterodyne_sums(self, params, freqs, h0, constants, t_obs_start=0.0, t_obs_end=1.0,
                        modes=None, precision="fp64", flags=None, **unused):
        """Relative-binning sums d_h, h_h (device complex128 [B] each) of the walkers
        ``params`` in one fused kernel: waveform + response at the sparse grid ``freqs``
        [L], mode sum, r = h / h0 (``h0`` [3, L]) and the bin terms with ``constants``
        [4, 3, L] (likelihood.py:550-648, Likelihood.cu:20-123)."""
        a = self.heterodyne_setup(params, freqs, h0, constants, t_obs_start, t_obs_end, modes,
                                  flags)
        vals = [a[k] if isinstance(a[k], (int, float)) else _lib.dptr(a[k]) for k in self.HDYN_ARGS]
        _lib.call("bbhx_hdyn_fused", self.response_gen.orbit_handle.ptr, *vals,
                  PRECISIONS[precision], _lib.stream())
        return a["d_h"], a["h_h"]

    def heterodyne_grad(self, params, freqs, h0, constants, t_obs_start=0.0, t_obs_end=1.0,
                        modes=None, **unused):
        """Relative-binning sums d_h, h_h [B] and d lnL / d theta [B, 11] of the walkers
        ``params`` (device tensor [12, B]); theta = rows (0, 1, 2, 3, 4, 5, 7, 8, 9, 10, 11)
        of ``params`` (f_ref, row 6, does not enter the model)."""
        t = torch()
        P = params.to(device=device(), dtype=t.float64).contiguous()
        rows = tuple(P[k] for k in range(12))
        m1, m2, chi1z, chi2z, distance, phi_ref, f_ref, inc, lam, beta, psi, t_ref = rows
        pars, t_start, t_end, _ = step_front(m1, m2, chi1z, chi2z, lam, beta, 1,
                                             (t_obs_start, t_obs_end))
        ap = self.amp_phase_gen
        ap._setup_records(m1, m2, chi1z, chi2z, distance, t_ref, modes, front=pars)
        B, M, L = ap.num_bin_all, ap.num_modes, int(freqs.numel())
        rg = self.response_gen
        d_h = t.empty(B, dtype=t.complex128, device=device())
        h_h = t.empty(B, dtype=t.complex128, device=device())
        grad = t.empty((B, 11), dtype=t.float64, device=device())
        tab = ap.qnm_table
        from .waveforms.ringdownphenomd import dspin
        _lib.call("bbhx_hdyn_grad", rg.orbit_handle.ptr, _lib.dptr(d_h), _lib.dptr(h_h),
                  _lib.dptr(grad), _lib.dptr(ap._coeffs), _lib.dptr(P), _lib.dptr(ap.ells),
                  _lib.dptr(ap.mms), _lib.dptr(tab), int(tab.shape[1]), float(dspin),
                  float(ap.initial_t_val), _lib.dptr(t_start), _lib.dptr(t_end), _lib.dptr(freqs),
                  _lib.dptr(h0), _lib.dptr(constants), rg.TDItag_int, int(rg.rescaled),
                  int(rg.tdi2), int(ap.run_phenomd), M, L, B, _lib.stream())
        return d_h, h_h, grad

    def direct_grad(self, params, data_freqs, data_weighted, noise_factors, t_obs_start=0.0,
                    t_obs_end=1.0, length=1024, modes=None, **unused):
        """<d|h>, <h|h> [B] and d lnL / d theta [B, 11] for a [12, B] device parameter tensor
        (theta: rows 0-5, 7-11).  Forward as inner_products (FP64), then the gradient chain."""
        t = torch()
        P = params.to(device=device(), dtype=t.float64).contiguous()
        rows = tuple(P[k] for k in range(12))
        buf, c1, c2, c3, x, ts, te = self._spline_set(rows, t_obs_start, t_obs_end, length, modes)
        f_default, tf_default = self._regrid_inputs
        ap, rg = self.amp_phase_gen, self.response_gen
        B, M, L = self.num_bin_all, self.num_modes, self.length
        grad = t.empty((B, 11), dtype=t.float64, device=device())
        d_h = t.empty(B, dtype=t.complex128, device=device())
        h_h = t.empty(B, dtype=t.complex128, device=device())
        tab = ap.qnm_table
        from .waveforms.ringdownphenomd import dspin
        _lib.call("bbhx_direct_like_grad", rg.orbit_handle.ptr, _lib.dptr(d_h), _lib.dptr(h_h),
                  _lib.dptr(grad), _lib.dptr(P),
                  _lib.dptr(ap.ells), _lib.dptr(ap.mms), _lib.dptr(tab), int(tab.shape[1]),
                  float(dspin), float(ap.initial_t_val), _lib.dptr(data_freqs),
                  _lib.dptr(data_weighted), _lib.dptr(noise_factors), int(data_freqs.numel()),
                  _lib.dptr(x), _lib.dptr(buf), _lib.dptr(c1), _lib.dptr(c2), _lib.dptr(c3),
                  _lib.dptr(ts), _lib.dptr(te), _lib.dptr(f_default), _lib.dptr(tf_default),
                  float(t_obs_start * YRSID_SI), float(t_obs_end * YRSID_SI), rg.TDItag_int,
                  int(rg.rescaled), int(rg.tdi2), int(ap.run_phenomd), M, L, B, _lib.stream())
        return d_h, h_h, grad

    def _spline_set(self, params, t_obs_start, t_obs_end, length, modes, flags=None,
                    timing=None):
        """Sparse buffer [9, B, M, L], its spline coefficients c1..c3, the knots and the
        per-binary observation limits (device), as the fused likelihood consumes them.
        ``timing``: optional dict that receives CUDA events around the spline build."""
        t = torch()
        buf, t_start, t_end = self._sparse_buffer(params, t_obs_start, t_obs_end, None, length,
                                                  modes, False, flags=flags)
        B, M, L = self.num_bin_all, self.num_modes, self.length
        x = self.amp_phase_gen.freqs
        c1 = t.empty_like(buf)
        c2 = t.empty_like(buf)
        c3 = t.empty_like(buf)
        if timing is not None:
            ev0 = t.cuda.Event(enable_timing=True)
            ev1 = t.cuda.Event(enable_timing=True)
            ev0.record()
        _lib.call("bbhx_interpolate", _lib.dptr(x), _lib.dptr(buf), _lib._VP(0),
                  _lib.dptr(c1), _lib.dptr(c2), _lib.dptr(c3), L, 9, M, B, _lib.stream())
        if timing is not None:
            ev1.record()
            timing.setdefault("spline", []).append((ev0, ev1))
        return buf, c1, c2, c3, x, to_dev(t_start), to_dev(t_end)

    def inner_products(self, params, data_freqs, data_weighted, noise_factors, t_obs_start=0.0,
                       t_obs_end=1.0, length=1024, modes=None, flags=None, timing=None,
                       precision="fp64", data32=None, **unused):
        """Fused <d|h>, <h|h> for every binary (device complex128 [B] each).

        ``data_weighted`` [3, N] complex = data * sqrt(df / S); ``noise_factors`` [3, N] =
        sqrt(df / S) (the reference's Likelihood attributes, likelihood.py:99-112).
        ``data32``: optional (complex64, float32) copies of the two, read by the mixed form."""
        t = torch()
        # ts_d / te_d stay referenced across the call: a temporary freed inside the argument
        # list can be handed back by the caching allocator to the next one
        buf, c1, c2, c3, x, ts_d, te_d = self._spline_set(params, t_obs_start, t_obs_end, length,
                                                          modes, flags=flags, timing=timing)
        B, M, L = self.num_bin_all, self.num_modes, self.length
        d_h = t.empty(B, dtype=t.complex128, device=device())
        h_h = t.empty(B, dtype=t.complex128, device=device())
        if timing is not None:  # optional CUDA events around the fused kernel (benchmarks)
            ev0 = t.cuda.Event(enable_timing=True)
            ev1 = t.cuda.Event(enable_timing=True)
            ev0.record()
        _lib.call("bbhx_direct_like_fused", _lib.dptr(d_h), _lib.dptr(h_h), _lib.dptr(data_freqs),
                  _lib.dptr(data_weighted), _lib.dptr(noise_factors), int(data_freqs.numel()),
                  _lib.dptr(x), _lib.dptr(buf), _lib.dptr(c1), _lib.dptr(c2), _lib.dptr(c3),
                  _lib.dptr(ts_d), _lib.dptr(te_d), M, L, B, PRECISIONS[precision],
                  _lib.dptr(data32[0]) if data32 is not None else _lib._VP(0),
                  _lib.dptr(data32[1]) if data32 is not None else _lib._VP(0), _lib.stream())
        if timing is not None:
            ev1.record()
            timing.setdefault("fused", []).append((ev0, ev1))
            self._last_x = x
        return d_h, h_h
