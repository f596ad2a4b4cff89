"""BBHx's own tests (tests/test_bbhx.py:47-95 test_full_waveform, :97-119 test_phenom_hm,
:121-162 test_fast_fd_response, :164-256 test_direct_likelihood and :258-373
test_het_likelihood) at their configuration, with the numbers of the reference implementation
(tests/golden/reftest_golden.npz, written by tests/golden/make_reftest_golden.py) instead of
the reference test's NaN checks.  Waveform tests: PhenomHM amplitude, phase, t(f) and the TDI
response at row-relative 1e-10 (the tolerance of the other golden parity tests), the full
filled waveform on 10,000 log-spaced frequencies at row-relative 4e-9 (its phases reach
2.6e7 rad, whose FP64 spacing is 3.7e-9 rad; measured 1.5e-9).  Likelihood tests: one injected binary without noise on the 10-s, 1.2-yr rfft
grid (1.89e6 bins), the six modes, ten binaries with 1e-4 jitter on m1 (lnL between -0.4 and
-23), and the heterodyned likelihood with 128 bins around the best of them.  The injection is
loud (<d|d> = 1.8e6, SNR 1340) and lnL = -(<d|d> + <h|h> - 2 <d|h>) / 2 cancels three sums of
5.7e6 terms of that size; each side's FP64 rounding of those sums is ~1e-12 of them, so the
direct tolerance is |dlnL| <= 1e-6 + 1e-12 (<d|d> + <h|h>) (measured 1.3e-6; the injections of
the two sides differ by 5e-12 relative, which the near-injection lnL cancels to first order).
The heterodyned sums run over 127 bins only: |dlnL| <= 1e-6 absolute.  <d|d> agrees to 1e-10
relative."""
import numpy as np
import pytest

from conftest import REPO

pytestmark = pytest.mark.gpu

MODES = [(2, 2), (2, 1), (3, 3), (3, 2), (4, 4), (4, 3)]


@pytest.fixture(scope="module")
def reftest():
    import os

    from bbhx_b200 import BBHWaveformFD, EqualArmlengthOrbits, Likelihood
    from bbhx_b200.sensitivity import aet_psd
    from bbhx_b200.utils.constants import PC_SI, YRSID_SI

    g = np.load(os.path.join(REPO, "tests", "golden", "reftest_golden.npz"))
    orbits = EqualArmlengthOrbits()
    wave = BBHWaveformFD(amp_phase_kwargs=dict(run_phenomd=False), response_kwargs=dict(orbits=orbits))
    n = int(1.2 * YRSID_SI / 10.0)
    f = np.fft.rfftfreq(n, 10.0)[1:]
    inj = np.array([1e6, 5e5, 0.2, 0.4, 18e3 * PC_SI * 1e6, 0.0, 0.0, np.pi / 3.0, np.pi / 5.0,
                    np.pi / 4.0, np.pi / 6.0, 0.8 * YRSID_SI])
    kw = dict(modes=MODES, direct=False, fill=True, squeeze=True, length=1024)
    data = wave(*inj, freqs=f, **kw)[0]
    psd = np.asarray([aet_psd(f, c) for c in "AET"])
    like = Likelihood(wave, f, data, psd)
    return g, wave, f, data, like, kw


def test_reference_direct_likelihood_test_numbers(reftest):
    g, wave, f, data, like, kw = reftest
    assert len(f) == 1893488
    assert abs(like.d_d - float(g["d_d"])) <= 1e-10 * abs(float(g["d_d"]))
    ll = like.get_ll(g["params"], **kw)
    hh = like.h_h.real.cpu().numpy()
    d = np.abs(ll - g["lnl"])
    print("direct |dlnL|", d)
    assert np.all(d <= 1e-6 + 1e-12 * (like.d_d + hh)), d
    assert int(ll.argmax()) == int(g["ref_index"])


def test_reference_het_likelihood_test_numbers(reftest):
    from bbhx_b200 import HeterodynedLikelihood

    g, wave, f, data, like, kw = reftest
    het = HeterodynedLikelihood(wave, f, data, g["params"][:, int(g["ref_index"])], 128)
    assert abs(het.reference_d_d - float(g["het_reference_d_d"])) <= 1e-10 * abs(
        float(g["het_reference_d_d"]))
    ll = het.get_ll(g["params"], **kw)
    d = np.abs(ll - g["lnl_het"])
    print("heterodyned |dlnL|", d)
    assert np.all(d <= 1e-6), d


def test_reference_phenom_hm_and_response_test_numbers(reftest):
    from test_gpu_parity import rowclose

    from bbhx_b200 import EqualArmlengthOrbits, LISATDIResponse, PhenomHMAmpPhase
    from bbhx_b200.utils.constants import PC_SI, YRSID_SI

    g = reftest[0]
    phm = PhenomHMAmpPhase(run_phenomd=False)
    phm(1e6, 5e5, 0.2, 0.4, 18e3 * PC_SI * 1e6, 0.0, 0.0, 0.8 * YRSID_SI, 1024)
    rowclose(phm.freqs_shaped.cpu().numpy(), g["phm_freqs"])
    rowclose(phm.amp.cpu().numpy(), g["phm_amp"])
    rowclose(phm.phase.cpu().numpy(), g["phm_phase"])
    rowclose(phm.tf.cpu().numpy(), g["phm_tf"])
    resp = LISATDIResponse(orbits=EqualArmlengthOrbits())
    resp(phm.freqs.clone(), np.pi / 4, np.pi / 6, np.pi / 5, np.pi / 7, 0.0,
         phm.freqs_shaped.shape[-1], phase=phm.phase.clone(), tf=phm.tf.clone(), modes=phm.modes)
    for name, ref in (("transferL1", "resp_L1"), ("transferL2", "resp_L2"),
                      ("transferL3", "resp_L3"), ("phase", "resp_phase"), ("tf", "resp_tf")):
        got = getattr(resp, name).cpu().numpy().reshape(g[ref].shape)
        if np.iscomplexobj(g[ref]):
            rowclose(got.real, g[ref].real)
            rowclose(got.imag, g[ref].imag)
        else:
            rowclose(got, g[ref])


def test_reference_full_waveform_test_numbers(reftest):
    from test_gpu_parity import rowclose

    g, wave = reftest[0], reftest[1]
    from bbhx_b200.utils.constants import PC_SI, YRSID_SI

    inj = np.array([1e6, 5e5, 0.2, 0.4, 18e3 * PC_SI * 1e6, 0.0, 0.0, np.pi / 3.0, np.pi / 5.0,
                    np.pi / 4.0, np.pi / 6.0, 0.8 * YRSID_SI])
    full = wave(*inj, freqs=np.logspace(-4, 0, 10000), modes=MODES, direct=False, fill=True,
                squeeze=True, length=1024)[0]
    full = full.cpu().numpy() if hasattr(full, "cpu") else np.asarray(full)
    rowclose(full.real, g["full_wave"].real, rtol=4e-9)
    rowclose(full.imag, g["full_wave"].imag, rtol=4e-9)
