"""Direct and heterodyned log-likelihoods on the GPU.

Drop-ins for the reference's ``Likelihood`` and ``HeterodynedLikelihood``
(src/bbhx/likelihood.py:26-648): same constructors, attributes (``d_d``, ``noise_factors``,
``data_channels``, ``reference_d_d``, ``data_constants``, ``freqs``, ...) and ``get_ll``
keywords (``return_extracted_snr``, ``phase_marginalize``, waveform keywords); results come
back as numpy arrays, as in the reference.

``Likelihood.get_ll`` runs the fused device path (``BBHWaveformFD.inner_products``): no
per-binary templates are materialised and the single host synchronisation is the copy of
the results (together with the deferred error flags).
"""
import numpy as np

from . import _lib
from .sensitivity import AET1SensitivityMatrix, SensitivityMatrix
from .utils.arrays import device, to_dev, to_np, torch
from .waveformbuild import PRECISIONS
from .waveforms.phenomhm import raise_chi_flag


def pack_lnl(d_h, h_h, d_d, out=None):
    """lnL = -(d_d + Re h_h - 2 Re d_h) / 2 of complex [B] device sums, by the library's packing
    kernel (bbhx_pack_lnl); ``out``: optional preallocated float64 [3 B] buffer (fixed address,
    e.g. under CUDA graph capture).  Returns the lnL view [B]."""
    B = d_h.numel()
    if out is None:
        out = torch().empty(3 * B, dtype=torch().float64, device=device())
    _lib.call("bbhx_pack_lnl", _lib.dptr(out), _lib.dptr(d_h), _lib.dptr(h_h), float(d_d), B, 0,
              _lib._VP(0), 0, _lib.stream())
    return out[:B]


class Likelihood:
    """Direct log-likelihood.  ``precision`` selects the arithmetic of the fused kernel:
    "fp64" (default, the parity form) or "mixed" (FP64 phase / t(f) / accumulations, FP32
    amplitudes, transfer functions and per-bin products)."""

    def __init__(self, template_gen, data_freqs, data_channels, psd, force_backend=None,
                 precision="fp64"):
        t = torch()
        self.precision = precision
        self.data_freqs = to_dev(data_freqs)
        data_freqs_cpu = to_np(data_freqs).astype(np.float64)
        self.psd = np.asarray(to_np(psd), dtype=np.float64)
        self.delta_f = np.zeros_like(self.psd)
        self.delta_f[:, 1:] = np.diff(data_freqs_cpu)
        self.delta_f[:, 0] = self.delta_f[:, 1]
        self.noise_factors = to_dev(np.sqrt(1.0 / self.psd * self.delta_f).flatten())
        self.data_channels = (self.noise_factors * to_dev(data_channels, t.complex128).flatten()).contiguous()
        self.waveform_gen = template_gen
        self.data_stream_length = len(data_freqs_cpu)
        self.d_d = float((4 * (self.data_channels.conj() * self.data_channels).sum()).real.item())
        self._fp32 = None

    def fp32_data(self):
        """FP32 copies of the weighted data and the weights (complex64 / float32 [3 N]) that the
        mixed form reads; made once, on first use."""
        if self._fp32 is None:
            t = torch()
            self._fp32 = (self.data_channels.to(t.complex64).contiguous(),
                          self.noise_factors.to(t.float32).contiguous())
        return self._fp32

    @property
    def xp(self):
        return torch()

    @property
    def precision(self):
        return self._precision

    @precision.setter
    def precision(self, value):
        if value not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}, got {value!r}")
        self._precision = value

    def get_ll(self, params, return_extracted_snr=False, phase_marginalize=False,
               **waveform_kwargs):
        """log-likelihood for params of shape (12,) or (12, B) (likelihood.py:140-225)."""
        t = torch()
        self.phase_marginalize = phase_marginalize
        self.return_extracted_snr = return_extracted_snr
        if isinstance(params, t.Tensor):
            # (pinned) host or device tensor: one asynchronous copy, parameters stay on the GPU
            params = params.to(device=device(), dtype=t.float64, non_blocking=True)
            if params.ndim == 1:
                params = params.reshape(-1, 1)
            params = tuple(params[k].contiguous() for k in range(params.shape[0]))
        else:
            params = np.atleast_2d(np.asarray(params, dtype=np.float64))
            if params.shape[0] != 12 and params.shape[1] == 12:
                params = params.T
            params = tuple(params)
        kw = dict(waveform_kwargs)
        for k in ("freqs", "fill", "direct", "compress", "squeeze", "combine"):
            kw.pop(k, None)
        flags = t.empty(3, dtype=t.int32, device=device())  # cleared by the step's front end
        if self.precision == "mixed":
            kw["data32"] = self.fp32_data()
        d_h, h_h = self.waveform_gen.inner_products(params, self.data_freqs,
                                                    self.data_channels, self.noise_factors,
                                                    flags=flags, precision=self.precision, **kw)
        self.d_h, self.h_h = d_h, h_h
        # lnL, Re <d|h> (|<d|h>| when phase-marginalised), Re <h|h> and the status flags in one
        # device buffer, one copy to the host (likelihood.py:204-225)
        B = d_h.numel()
        packed_d = t.empty(3 * B + 3, dtype=t.float64, device=device())
        _lib.call("bbhx_pack_lnl", _lib.dptr(packed_d), _lib.dptr(d_h), _lib.dptr(h_h),
                  float(self.d_d), B, int(bool(phase_marginalize)), _lib.dptr(flags), 3,
                  _lib.stream())
        packed = packed_d.cpu().numpy()
        fl = packed[3 * B:]
        if fl[0] == 1:
            raise ValueError("The search for a window at x_min did not run correctly. If t_ref is "
                             "close to zero, the time-frequency correspondence may be crossing zero twice.")
        if fl[0] == 2:
            raise ValueError("The search for a window at x_max did not run correctly. If t_ref is "
                             "close to the observation time, the time-frequency correspondence may be "
                             "crossing zero twice.")
        if fl[1] != 0:
            raise ValueError("Orbital information does not cover the t(f) range of the templates.")
        raise_chi_flag(int(fl[2]))
        ll = packed[:B]
        if return_extracted_snr:
            return np.array([ll, packed[B:2 * B] / np.sqrt(packed[2 * B:3 * B])]).T
        return ll


    # ------------------------------------------------------------------ gradients
    def _device_ll(self, params, kw):
        rows = tuple(params[k].contiguous() for k in range(12))
        kw = {k: v for k, v in kw.items() if k in ("t_obs_start", "t_obs_end", "length", "modes")}
        d_h, h_h = self.waveform_gen.inner_products(rows, self.data_freqs, self.data_channels,
                                                    self.noise_factors, precision="fp64", **kw)
        return pack_lnl(d_h, h_h, self.d_d)

    def get_ll_and_grad(self, params, **waveform_kwargs):
        """lnL [B] and d lnL / d theta [B, 11] (device tensors); theta = (m1, m2, chi1z,
        chi2z, distance, phi_ref, inc, lam, beta, psi, t_ref).  FP64, plain lnL; the
        derivative follows the sparse knots as the observation-window regrid moves them."""
        from .autodiff import as_param_tensor

        P = as_param_tensor(params)
        kw = {k: v for k, v in waveform_kwargs.items()
              if k in ("t_obs_start", "t_obs_end", "length", "modes")}
        d_h, h_h, grad = self.waveform_gen.direct_grad(P, self.data_freqs, self.data_channels,
                                                       self.noise_factors, **kw)
        return pack_lnl(d_h, h_h, self.d_d), grad

    def loglike_torch(self, params, **waveform_kwargs):
        """Differentiable lnL [B] tensor; the backward pass runs the gradient kernels."""
        from .autodiff import as_param_tensor, function

        P = params if (hasattr(params, "requires_grad") and params.requires_grad) else as_param_tensor(params)
        return function("direct").apply(P, self, dict(waveform_kwargs))


class HeterodynedLikelihood:
    """Heterodyned (relative-binning) log-likelihood.  ``precision`` selects the fused kernel
    that evaluates the walkers: "fp64" (default) or "mixed" (FP64 phase, t(f), Roemer delay,
    ratio and sums; FP32 amplitude, transfer functions and channel products).  ``None``
    runs the reference's step-by-step chain (sparse templates, ratio, hdyn), which also
    materialises ``h_sparse``; with a fused precision ``h_sparse`` is produced on first
    access from the last walkers."""

    def __init__(self, template_gen, data_freqs, data_channels, reference_template_params,
                 length_f_het, template_gen_kwargs=None, reference_gen_kwargs=None, sens_mat=None,
                 force_backend=None, precision="fp64"):
        template_gen_kwargs = {} if template_gen_kwargs is None else template_gen_kwargs
        reference_gen_kwargs = {} if reference_gen_kwargs is None else reference_gen_kwargs
        self.precision = precision
        self._h_sparse = None
        self._last = None
        self.template_gen = template_gen
        self.f_dense = to_dev(data_freqs)
        self.d = to_dev(data_channels, torch().complex128)
        self.length_f_het = length_f_het
        self.sens_mat = sens_mat
        self.init_heterodyne_info(reference_template_params,
                                  template_gen_kwargs=template_gen_kwargs,
                                  reference_gen_kwargs=reference_gen_kwargs)

    @property
    def xp(self):
        return torch()

    @property
    def precision(self):
        return self._precision

    @precision.setter
    def precision(self, value):
        if value is not None and value not in PRECISIONS:
            raise ValueError(f"precision must be None or one of {sorted(PRECISIONS)}, got {value!r}")
        self._precision = value

    @property
    def sens_mat(self):
        return self._sens_mat

    @sens_mat.setter
    def sens_mat(self, sens_mat):
        if sens_mat is None:
            sens_mat = AET1SensitivityMatrix(np.logspace(-5, -1, 1000))
        assert isinstance(sens_mat, SensitivityMatrix)
        self._sens_mat = sens_mat

    def init_heterodyne_info(self, reference_template_params, template_gen_kwargs=None,
                             reference_gen_kwargs=None):
        """Reference template, sparse grid and relative-binning constants
        (likelihood.py:380-548)."""
        t = torch()
        template_gen_kwargs = dict(template_gen_kwargs or {})
        reference_gen_kwargs = dict(reference_gen_kwargs or {})
        template_gen_kwargs["squeeze"] = True
        template_gen_kwargs["compress"] = True
        template_gen_kwargs["direct"] = True
        fd = to_np(self.f_dense)
        # a probe grid just wider than the data, then narrowed (likelihood.py:424-462)
        f_lo = fd.min() * 0.999999999999
        f_hi = fd.max() * 1.000000000001
        if f_lo == 0.0:
            f_lo = 1e-6
        reference_gen_kwargs["squeeze"] = True
        reference_gen_kwargs["compress"] = True
        reference_gen_kwargs["fill"] = True
        if not ("direct" in reference_gen_kwargs and reference_gen_kwargs["direct"] is True):
            reference_gen_kwargs["direct"] = False
            if "length" not in reference_gen_kwargs:
                reference_gen_kwargs["length"] = 8096
        probe = np.logspace(np.log10(f_lo), np.log10(f_hi), self.length_f_het)
        p = [np.atleast_1d(v) for v in reference_template_params]
        h0 = self.template_gen(*p, freqs=self.f_dense, **reference_gen_kwargs)[0]
        # the sparse grid spans the probe points where the reference template is non-zero
        nonzero = to_np(self.template_gen(*p, freqs=probe, **template_gen_kwargs)[0].abs() != 0.0)
        band = probe[nonzero]
        freqs = np.logspace(np.log10(band[0]), np.log10(band[-1]), self.length_f_het)
        self.h0_sparse = self.template_gen(*p, freqs=freqs, **template_gen_kwargs)[None, :, :]
        self._h0_flat = self.h0_sparse[0].contiguous()
        # the band the reference keeps, (f >= freqs[0]) & (f <= freqs[-1]), is a contiguous run
        # of the sorted dense grid: [i0, i1)
        fd_all = to_np(self.f_dense)
        i0 = int(np.searchsorted(fd_all, freqs[0], "left"))
        i1 = int(np.searchsorted(fd_all, freqs[-1], "right"))
        n = i1 - i0
        f_dense_h = fd_all[i0:i1]
        df = f_dense_h[1] - f_dense_h[0]
        self.sens_mat.update_frequency_arr(f_dense_h)
        S_n = to_dev(np.ascontiguousarray([self.sens_mat[0], self.sens_mat[1], self.sens_mat[2]]))
        h0 = h0.contiguous()
        d_full = self.d.contiguous()
        N_all = d_full.shape[1]
        L = self.length_f_het
        freqs_d = to_dev(freqs)
        consts = t.empty(4 * 3 * L, dtype=t.complex128, device=device())
        ref = t.empty(3, dtype=t.float64, device=device())
        # per-bin A0, A1, B0, B1 sums into slot j + 1 and the band's reference sums on the device
        # (likelihood.py:480-530): bbhx_hdyn_constants reads the band in place
        _lib.call("bbhx_hdyn_constants", _lib.dptr(consts), _lib.dptr(ref),
                  _lib._VP(self.f_dense.data_ptr() + 8 * i0),
                  _lib._VP(d_full.data_ptr() + 16 * i0), N_all,
                  _lib._VP(h0.data_ptr() + 16 * i0), int(h0.shape[1]), _lib.dptr(S_n), n, n,
                  _lib.dptr(freqs_d), L, float(df), _lib.stream())
        self.f_dense = self.f_dense[i0:i1]
        self.d = d_full[:, i0:i1]
        self.data_constants = consts
        self.reference_d_d, self.reference_h_h, self.reference_d_h = (float(v) for v in ref.cpu())
        self.reference_ll = -1 / 2 * (self.reference_d_d + self.reference_h_h - 2 * self.reference_d_h)
        self.freqs = freqs_d
        self.f_m = (freqs[1:] + freqs[:-1]) / 2
        template_gen_kwargs["squeeze"] = False
        self.template_gen_kwargs = template_gen_kwargs

    # ------------------------------------------------------------------ gradients
    def _fused_ll(self, params, kw, precision, flags=None):
        """lnL [B] (device) and the raw sums for a [12, B] device parameter tensor; with a
        device ``flags`` tensor the spin check is recorded there (no host synchronisation)."""
        rows = tuple(params[k].contiguous() for k in range(12))
        kw = {k: v for k, v in kw.items() if k in ("t_obs_start", "t_obs_end", "modes")}
        d_h, h_h = self.template_gen.heterodyne_sums(rows, self.freqs, self._h0_flat,
                                                     self.data_constants, precision=precision,
                                                     flags=flags, **kw)
        return pack_lnl(d_h, h_h, self.reference_d_d), (d_h, h_h)

    def get_ll_and_grad(self, params, **waveform_kwargs):
        """lnL [B] and d lnL / d theta [B, 11] (device tensors) for walkers ``params``
        ([12, B]); theta = (m1, m2, chi1z, chi2z, distance, phi_ref, inc, lam, beta, psi,
        t_ref).  FP64; the gradient of the plain (not phase-marginalised) lnL."""
        from .autodiff import as_param_tensor

        P = as_param_tensor(params)
        kw = dict(self.template_gen_kwargs)
        kw.update(waveform_kwargs)
        kw = {k: v for k, v in kw.items() if k in ("t_obs_start", "t_obs_end", "modes")}
        d_h, h_h, grad = self.template_gen.heterodyne_grad(P, self.freqs, self._h0_flat,
                                                           self.data_constants, **kw)
        return pack_lnl(d_h, h_h, self.reference_d_d), grad

    def loglike_torch(self, params, **waveform_kwargs):
        """Differentiable lnL: a [B] tensor whose backward pass runs the gradient kernels
        (the waveform is recomputed there, nothing is stored)."""
        from .autodiff import as_param_tensor, function

        kw = dict(self.template_gen_kwargs)
        kw.update(waveform_kwargs)
        P = params if (hasattr(params, "requires_grad") and params.requires_grad) else as_param_tensor(params)
        return function("heterodyned").apply(P, self, kw)

    @property
    def h_sparse(self):
        """Sparse templates [B, 3, L] of the last walkers (likelihood.py:612)."""
        if self._h_sparse is None and self._last is not None:
            params, kw = self._last
            self._h_sparse = self.template_gen(*params, **kw)
        return self._h_sparse

    def get_ll(self, params, return_extracted_snr=False, phase_marginalize=False,
               **waveform_kwargs):
        """Heterodyned log-likelihood (likelihood.py:550-648)."""
        t = torch()
        self.phase_marginalize = phase_marginalize
        self.return_extracted_snr = return_extracted_snr
        keys = set(waveform_kwargs) | set(self.template_gen_kwargs)
        for key in keys:
            if key in ["direct", "compress", "squeeze"]:
                waveform_kwargs[key] = self.template_gen_kwargs[key]
            elif key in self.template_gen_kwargs:
                waveform_kwargs[key] = waveform_kwargs.get(key, self.template_gen_kwargs[key])
        waveform_kwargs["freqs"] = self.freqs
        if isinstance(params, t.Tensor):
            params = params.to(device=device(), dtype=t.float64, non_blocking=True)
            if params.ndim == 1:
                params = params.reshape(-1, 1)
            params = tuple(params[k].contiguous() for k in range(params.shape[0]))
        else:
            params = tuple(np.atleast_2d(np.asarray(params, dtype=np.float64)))
        if self.precision is not None:
            kw = {k: v for k, v in waveform_kwargs.items()
                  if k in ("t_obs_start", "t_obs_end", "modes")}
            self._last = (params, dict(waveform_kwargs))
            self._h_sparse = None
            self.hdyn_d_h, self.hdyn_h_h = self.template_gen.heterodyne_sums(
                params, self.freqs, self._h0_flat, self.data_constants,
                precision=self.precision, **kw)
        else:
            self._h_sparse = self.template_gen(*params, **waveform_kwargs)
            r = self._h_sparse / self.h0_sparse
            B = r.shape[0]
            residuals = r.permute(2, 1, 0).contiguous().flatten()
            self.hdyn_d_h = t.zeros(B, dtype=t.complex128, device=device())
            self.hdyn_h_h = t.zeros(B, dtype=t.complex128, device=device())
            _lib.call("bbhx_hdyn", _lib.dptr(self.hdyn_d_h), _lib.dptr(self.hdyn_h_h),
                      _lib.dptr(residuals), _lib.dptr(self.data_constants), _lib.dptr(self.freqs),
                      B, len(self.freqs), 3, _lib.stream())
        B = self.hdyn_d_h.numel()
        packed_d = t.empty(3 * B, dtype=t.float64, device=device())
        _lib.call("bbhx_pack_lnl", _lib.dptr(packed_d), _lib.dptr(self.hdyn_d_h),
                  _lib.dptr(self.hdyn_h_h), float(self.reference_d_d), B,
                  int(bool(phase_marginalize)), _lib._VP(0), 0, _lib.stream())
        packed = packed_d.cpu().numpy()
        out = packed[:B]
        if return_extracted_snr:
            return np.array([out, packed[B:2 * B] / np.sqrt(packed[2 * B:3 * B])]).T
        return out
