"""Generate tests/golden/reftest_golden.npz: the reference's own tests (tests/test_bbhx.py:
47-95 test_full_waveform, :97-119 test_phenom_hm, :121-162 test_fast_fd_response, :164-256
test_direct_likelihood and :258-373 test_het_likelihood) run by the REFERENCE implementation,
with their numbers kept instead of only checked for NaN.

Waveform tests: the binary below on 10,000 log-spaced frequencies over 1e-4..1 Hz (fill=True,
squeeze=True, sparse length 1024), PhenomHM at the default grid of 1024 points, and the TDI
response of that PhenomHM output at inc pi/4, lambda pi/6, beta pi/5, psi pi/7.

Configuration of those tests: one binary (m1 = 1e6, m2 = 5e5 Msun, spins 0.2 / 0.4, 18 Gpc,
inc pi/3, beta pi/4, lambda pi/5, psi pi/6, t_ref = 0.8 yr, phi_ref = f_ref = 0) injected with
no noise on the grid rfftfreq(int(1.2 yr / 10 s), 10 s)[1:] (1.89e6 bins up to 0.05 Hz); the
six PhenomHM modes on sparse grids of 1024 points (fill=True, squeeze=True); PSD from the A/E/T
first-generation sensitivities; ten binaries with relative 1e-4 jitter on m1 (numpy's global
generator seeded 111222, as the reference test module does); the heterodyned likelihood around
the best of the ten with 128 bins, sensitivity matrix and generator settings left at their
defaults.  The reference's Python classes run unmodified on the reference's C++ compiled for
CPU (oracle/_ref), with oracle/refenv standing in for gpubackendtools / lisatools, as in
make_golden.py.

Usage:  python tests/golden/make_reftest_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, REPO)
from oracle.build_ref import REF_ROOT  # noqa: E402

sys.path.insert(0, os.path.join(REPO, "oracle", "refenv"))
sys.path.insert(0, os.path.join(REF_ROOT, "src"))

from oracle.build_ref import build as build_ref  # noqa: E402

build_ref()

import warnings  # noqa: E402

warnings.filterwarnings("ignore")
from bbhx.likelihood import HeterodynedLikelihood, Likelihood  # noqa: E402
from bbhx.response.fastfdresponse import LISATDIResponse  # noqa: E402
from bbhx.utils.constants import PC_SI, YRSID_SI  # noqa: E402
from bbhx.waveformbuild import BBHWaveformFD  # noqa: E402
from bbhx.waveforms.phenomhm import PhenomHMAmpPhase  # noqa: E402
from lisatools.detector import EqualArmlengthOrbits  # noqa: E402
from lisatools.sensitivity import get_sensitivity  # noqa: E402

MODES = [(2, 2), (2, 1), (3, 3), (3, 2), (4, 4), (4, 3)]
T_OBS_DATA = 1.2  # yr
DT = 10.0  # s
NUM_BINS = 10
LENGTH_F_HET = 128


def injection_params():
    """(m1, m2, a1, a2, dist, phi_ref, f_ref, inc, lam, beta, psi, t_ref) of the injection."""
    return np.array([1e6, 5e5, 0.2, 0.4, 18e3 * PC_SI * 1e6, 0.0, 0.0, np.pi / 3.0, np.pi / 5.0,
                     np.pi / 4.0, np.pi / 6.0, 0.8 * YRSID_SI])


def data_freqs():
    n = int(T_OBS_DATA * YRSID_SI / DT)
    return np.fft.rfftfreq(n, DT)[1:]


def waveform_tests(orbits, wave_gen):
    inj = injection_params()
    m1, m2, a1, a2, dist, phi_ref, f_ref = inj[:7]
    t_ref = inj[11]
    full = wave_gen(*inj, freqs=np.logspace(-4, 0, 10000), modes=MODES, direct=False, fill=True,
                    squeeze=True, length=1024)[0]
    phm = PhenomHMAmpPhase(run_phenomd=False)
    phm(m1, m2, a1, a2, dist, phi_ref, f_ref, t_ref, 1024)
    out = dict(full_wave=np.asarray(full), phm_freqs=phm.freqs_shaped.copy(),
               phm_amp=phm.amp.copy(), phm_phase=phm.phase.copy(), phm_tf=phm.tf.copy())
    freqs, phase, tf = phm.freqs.copy(), phm.phase.copy(), phm.tf.copy()
    resp = LISATDIResponse(orbits=orbits)
    resp(freqs, np.pi / 4, np.pi / 6, np.pi / 5, np.pi / 7, 0.0, phm.freqs_shaped.shape[-1],
         phase=phase, tf=tf, modes=phm.modes)
    out.update(resp_L1=resp.transferL1.copy(), resp_L2=resp.transferL2.copy(),
               resp_L3=resp.transferL3.copy(), resp_phase=resp.phase.copy(),
               resp_tf=resp.tf.copy())
    return out


def main():
    np.random.seed(111222)
    orbits = EqualArmlengthOrbits()
    orbits.configure(linear_interp_setup=True)
    wave_gen = BBHWaveformFD(amp_phase_kwargs=dict(run_phenomd=False),
                             response_kwargs=dict(orbits=orbits))
    waves = waveform_tests(orbits, wave_gen)
    f = data_freqs()
    waveform_kwargs = dict(modes=MODES, direct=False, fill=True, squeeze=True, length=1024)
    inj = injection_params()
    data = wave_gen(*inj, freqs=f, **waveform_kwargs)[0]
    psd = np.asarray([get_sensitivity(f, sens_fn=s) for s in ("A1TDISens", "E1TDISens",
                                                              "T1TDISens")])
    like = Likelihood(wave_gen, f, data, psd)
    params_in = np.tile(inj, (NUM_BINS, 1))
    params_in[:, 0] *= 1 + 1e-4 * np.random.randn(NUM_BINS)
    ll = like.get_ll(params_in.T, **waveform_kwargs)
    ref_index = int(ll.argmax())
    het = HeterodynedLikelihood(wave_gen, f, data, params_in[ref_index], LENGTH_F_HET)
    ll_het = het.get_ll(params_in.T, **waveform_kwargs)
    out = dict(params=params_in.T.copy(), lnl=np.asarray(ll), lnl_het=np.asarray(ll_het),
               d_d=np.array(like.d_d), ref_index=np.array(ref_index),
               het_reference_d_d=np.array(het.reference_d_d), data_abs_sum=np.abs(data).sum(axis=-1),
               **waves)
    path = os.path.join(HERE, "reftest_golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, "lnl", ll, "lnl_het", ll_het)


if __name__ == "__main__":
    main()
