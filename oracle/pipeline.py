"""Oracle (test infrastructure only): CPU restatement of the reference's Python driver
path, with the compute kernels delegated to a selectable backend.

Backends (same argument order as the reference's compiled-extension functions):
  * "ref": the reference's own C++ compiled for CPU (``oracle/_ref/libbbhx_ref.so``,
    ctypes bindings in ``oracle/refenv/bbhx_backend_cpu``);
  * "np":  the numpy restatement in ``oracle/kernels_np.py``.

Driver steps restated here (each function names the reference lines it follows):
  PhenomHMAmpPhase.run_wave / __call__   src/bbhx/waveforms/phenomhm.py:270-614
  LISATDIResponse.__call__                src/bbhx/response/fastfdresponse.py:278-531
  BBHWaveformFD.__call__                  src/bbhx/waveformbuild.py:338-700
  TemplateInterpFD.__call__               src/bbhx/waveformbuild.py:89-239
  Likelihood.__init__ / get_ll            src/bbhx/likelihood.py:75-225
  HeterodynedLikelihood                   src/bbhx/likelihood.py:380-648

Nothing in bbhx_b200/ imports this module; tests and bench.py use it as the checker and
as the CPU baseline.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "refenv"))
sys.path.insert(0, os.path.dirname(HERE))

from bbhx_b200.orbits import EqualArmlengthOrbits  # noqa: E402
from bbhx_b200.utils.constants import MSUN_SI, YRSID_SI  # noqa: E402
from bbhx_b200.utils.transform import tSSBfromLframe  # noqa: E402
from bbhx_b200.waveforms.ringdownphenomd import (QNMData_a, QNMData_fdamp,  # noqa: E402
                                                  QNMData_fring, dspin)

DEFAULT_MODES = [(2, 2), (3, 3), (4, 4), (2, 1), (3, 2), (4, 3)]


def qnm_spline_coeffs():
    """c1, c2, c3 of the not-a-knot spline through the QNM table (phenomhm.py:148-163)."""
    from scipy.interpolate import CubicSpline

    out = []
    for y in (QNMData_fring, QNMData_fdamp):
        s = CubicSpline(QNMData_a, y)
        out.append((np.asarray(y).copy(), s.c[-2].copy(), s.c[-3].copy(), s.c[-4].copy()))
    return out


class Kernels:
    """Backend dispatch for the nine reference kernels."""

    def __init__(self, backend="ref"):
        self.name = backend
        if backend == "ref":
            from oracle.build_ref import OUT, build, reference_available

            if reference_available():
                build()
            if not os.path.isfile(OUT):
                raise FileNotFoundError(OUT)
            import bbhx_backend_cpu.interp as I
            import bbhx_backend_cpu.likelihood as LK
            import bbhx_backend_cpu.phenomhm as PH
            import bbhx_backend_cpu.response as R
            import bbhx_backend_cpu.waveformbuild as W

            self.waveform_amp_phase = PH.waveform_amp_phase_wrap
            self.ringdown_hm = PH.get_phenomhm_ringdown_frequencies
            self.ringdown_d = PH.get_phenomd_ringdown_frequencies
            self.Response = R.pyFastLISAResponse
            self.interpolate = I.interpolate_wrap
            self.InterpTDI = W.InterpTDI_wrap
            self.direct_sum = W.direct_sum_wrap
            self.direct_like = LK.direct_like_wrap
            self.hdyn = LK.hdyn_wrap
        elif backend == "np":
            from oracle import kernels_np as K

            self.waveform_amp_phase = K.waveform_amp_phase
            self.ringdown_hm = K.get_phenomhm_ringdown_frequencies
            self.ringdown_d = K.get_phenomd_ringdown_frequencies
            self.Response = K.FastLISAResponse
            self.interpolate = K.interpolate
            self.InterpTDI = K.InterpTDI
            self.direct_sum = K.direct_sum
            self.direct_like = K.direct_like
            self.hdyn = K.hdyn
        else:
            raise ValueError(backend)


class RefPipeline:
    """The reference's driver logic on numpy arrays with the chosen kernel backend."""

    def __init__(self, backend="ref", orbits=None, TDItag="AET", tdi2=True, rescaled=False,
                 run_phenomd=False, mf_min=1e-4, mf_max=0.6, initial_t_val=0.0):
        self.K = Kernels(backend)
        self.orbits = orbits if orbits is not None else EqualArmlengthOrbits()
        self.resp = self.K.Response()
        self.resp.add_orbit_information(*self.orbits.pycppdetector_args)
        self.TDItag_int = 1 if TDItag == "XYZ" else 2
        self.tdi2 = tdi2
        self.rescaled = rescaled
        self.run_phenomd = run_phenomd
        self.mf_min, self.mf_max = mf_min, mf_max
        self.initial_t_val = initial_t_val
        self.qnm = qnm_spline_coeffs()

    # ------------------------------------------------------------ phenomhm.py:270-507
    def run_wave(self, m1, m2, chi1z, chi2z, distance, f_ref, t_ref, length, freqs, modes, out):
        m1, m2, chi1z, chi2z = (np.array(v, dtype=np.float64) for v in (m1, m2, chi1z, chi2z))
        sw = m1 < m2
        m1[sw], m2[sw] = m2[sw].copy(), m1[sw].copy()
        chi1z[sw], chi2z[sw] = chi2z[sw].copy(), chi1z[sw].copy()
        if self.run_phenomd:
            modes = [(2, 2)]
        ells = np.asarray([l for l, m in modes], dtype=np.int32)
        mms = np.asarray([m for l, m in modes], dtype=np.int32)
        B, M, L = len(m1), len(modes), length
        if freqs is None:
            Msec = (m1 + m2) * 4.925491025873693e-06
            base = np.logspace(np.log10(self.mf_min), np.log10(self.mf_max), L)
            freqs = (base[None, None, :] / Msec[:, None, None] * mms[None, :, None] / 2).flatten()
        elif freqs.ndim == 1:
            freqs = np.tile(freqs, (B, M, 1)).flatten()
        else:
            freqs = np.ascontiguousarray(freqs, dtype=np.float64).flatten()
        fring = np.zeros(M * B)
        fdamp = np.zeros(M * B)
        (yr, c1r, c2r, c3r), (yd, c1d, c2d, c3d) = self.qnm
        self.K.ringdown_d(fring, fdamp, m1, m2, chi1z, chi2z, B, yr, c1r, c2r, c3r, yd, c1d, c2d,
                          c3d, dspin)
        if not self.run_phenomd:
            pd_r = fring[:B].copy()
            pd_d = fdamp[:B].copy()
            self.K.ringdown_hm(fring, fdamp, m1, m2, chi1z, chi2z, ells, mms, M, B)
            fring = np.concatenate([fring.reshape(-1, M), pd_r[:, None]], axis=1).flatten().copy()
            fdamp = np.concatenate([fdamp.reshape(-1, M), pd_d[:, None]], axis=1).flatten().copy()
        self.K.waveform_amp_phase(out, ells, mms, freqs, m1 * MSUN_SI, m2 * MSUN_SI, chi1z, chi2z,
                                  np.asarray(distance, dtype=np.float64), np.asarray(f_ref, dtype=np.float64),
                                  M, L, B, fring, fdamp, int(self.run_phenomd))
        n = B * M * L
        out[n:2 * n] += (freqs.reshape(B, M, L) * (np.asarray(t_ref)[:, None, None] - self.initial_t_val)
                         * 2 * np.pi).flatten()
        out[2 * n:3 * n] += np.tile(np.asarray(t_ref)[:, None, None], (1, M, L)).flatten()
        return freqs, ells, mms

    @staticmethod
    def window(freqs, tf, Tobs):
        """f_min / f_max from the t(f) crossings and the log-spaced regrid (phenomhm.py:520-610)."""
        f_min = freqs.min(axis=-1)
        fix = tf.min(axis=-1) < 0.0
        if np.any(fix):
            w = np.argwhere((0.0 < tf[fix, 1:]) & (0.0 > tf[fix, :-1]))
            if w.shape[0] != fix.sum():
                raise ValueError("The search for a window at x_min did not run correctly.")
            s = w[:, 1]
            y1 = np.take_along_axis(freqs[fix], s[:, None], -1)[:, 0]
            y2 = np.take_along_axis(freqs[fix], s[:, None] + 1, -1)[:, 0]
            x1 = np.take_along_axis(tf[fix], s[:, None], -1)[:, 0]
            x2 = np.take_along_axis(tf[fix], s[:, None] + 1, -1)[:, 0]
            f_min[fix] = (y2 - y1) / (x2 - x1) * (0.0 - x1) + y1
        f_max = freqs.max(axis=-1)
        fix = tf.max(axis=-1) > Tobs
        if np.any(fix):
            w = np.argwhere((Tobs[fix][:, None] < tf[fix, 1:]) & (Tobs[fix][:, None] > tf[fix, :-1]))
            if w.shape[0] != fix.sum():
                raise ValueError("The search for a window at x_max did not run correctly.")
            s = w[:, 1]
            y1 = np.take_along_axis(freqs[fix], s[:, None], -1)[:, 0]
            y2 = np.take_along_axis(freqs[fix], s[:, None] + 1, -1)[:, 0]
            x1 = np.take_along_axis(tf[fix], s[:, None], -1)[:, 0]
            x2 = np.take_along_axis(tf[fix], s[:, None] + 1, -1)[:, 0]
            f_max[fix] = (y2 - y1) / (x2 - x1) * (Tobs[fix] - x1) + y1
        return np.logspace(np.log10(f_min), np.log10(f_max), freqs.shape[-1], axis=-1)

    # ------------------------------------------------------------ waveformbuild.py:338-600
    def sparse_buffer(self, params, t_obs_start=0.0, t_obs_end=1.0, length=1024, modes=None,
                      freqs=None, direct=False):
        (m1, m2, c1, c2, dist, phi_ref, f_ref, inc, lam, beta, psi, t_ref) = [
            np.atleast_1d(np.asarray(p, dtype=np.float64)) for p in params]
        modes = list(DEFAULT_MODES) if modes is None else list(modes)
        if self.run_phenomd:
            modes = [(2, 2)]
        B, M = len(m1), len(modes)
        t_start = np.atleast_1d(tSSBfromLframe(t_obs_start * YRSID_SI, lam, beta, 0.0))
        t_end = np.atleast_1d(tSSBfromLframe(t_obs_end * YRSID_SI, lam, beta, 0.0))
        if direct:
            length = freqs.shape[-1]
        L = length
        out = np.zeros(9 * L * M * B)
        f, ells, mms = self.run_wave(m1, m2, c1, c2, dist, f_ref, t_ref, L, freqs if direct else None,
                                     modes, out)
        if not direct:
            n = B * M * L
            tf = out[2 * n:3 * n].reshape(B, M, L)
            Tobs = np.repeat((t_end - t_start)[:, None], M, axis=-1)
            newf = self.window(f.reshape(B, M, L), tf, Tobs)
            out[:] = 0.0
            f, ells, mms = self.run_wave(m1, m2, c1, c2, dist, f_ref, t_ref, L, newf, modes, out)
            tfs = out[2 * n:3 * n]
            if tfs.min() < self.orbits.t_base.min() or tfs.max() > self.orbits.t_base.max():
                raise ValueError("Orbital information does not cover the t(f) range.")
        self.resp.LISA_response_wrap(out, ells, mms, f, phi_ref, inc, lam, beta, psi, self.TDItag_int,
                                     self.rescaled, self.tdi2, 0, M, L, B, 1)
        return out, f, t_start, t_end, (B, M, L)

    # ------------------------------------------------------------ spline + TemplateInterpFD
    def templates(self, params, data_freqs, t_obs_start=0.0, t_obs_end=1.0, length=1024, modes=None):
        buf, f, t_start, t_end, (B, M, L) = self.sparse_buffer(params, t_obs_start, t_obs_end, length,
                                                               modes)
        Bsl = np.zeros(9 * B * M * L)
        c1 = np.zeros_like(Bsl)
        c2 = np.zeros_like(Bsl)
        c3 = np.zeros_like(Bsl)
        self.K.interpolate(f, buf, Bsl, c1, c2, c3, L, 9, M, B)
        fs = f.reshape(B, M, L)
        se = np.asarray([np.searchsorted(data_freqs, v, side="right")
                         for v in np.array([fs.min(axis=(1, 2)), fs.max(axis=(1, 2))]).T])
        inds = [np.concatenate([np.searchsorted(fs[i, j], data_freqs[st:et], side="right") - 1
                                for j in range(M)]).astype(np.int32) for i, (st, et) in enumerate(se)]
        lengths = np.asarray([len(x) // M for x in inds], dtype=np.int32)
        starts = se[:, 0].astype(np.int32)
        ptrs = np.asarray([x.__array_interface__["data"][0] for x in inds], dtype=np.int64)
        tmpl = [np.zeros(3 * n, dtype=np.complex128) for n in lengths]
        tptrs = np.asarray([x.__array_interface__["data"][0] for x in tmpl], dtype=np.int64)
        self.K.InterpTDI(tptrs, data_freqs, f, buf, c1, c2, c3, t_start, t_end, L, len(data_freqs), B,
                         M, ptrs, starts, lengths)
        self._keep = (inds,)
        return tmpl, starts, lengths

    # ------------------------------------------------------------ likelihood.py:75-225
    def direct_lnl(self, params, data_freqs, data, psd, **kw):
        df = np.zeros_like(psd)
        df[:, 1:] = np.diff(data_freqs)
        df[:, 0] = df[:, 1]
        nf = np.sqrt(1.0 / psd * df).flatten()
        dw = nf * np.asarray(data, dtype=np.complex128).flatten()
        d_d = (4 * np.sum(dw.conj() * dw)).real
        tmpl, starts, lengths = self.templates(params, data_freqs, **kw)
        B = len(tmpl)
        ptrs = np.asarray([x.__array_interface__["data"][0] for x in tmpl], dtype=np.int64)
        d_h = np.zeros(B, dtype=np.complex128)
        h_h = np.zeros(B, dtype=np.complex128)
        self.K.direct_like(d_h, h_h, dw, nf, ptrs, starts, lengths, len(data_freqs), B)
        return -0.5 * (d_d + h_h - 2 * d_h).real, d_h, h_h, d_d
