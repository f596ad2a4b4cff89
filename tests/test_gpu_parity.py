"""GPU parity of the CUDA path against the reference golden fixtures.

The fixtures (tests/golden/reference_golden.npz) were produced by the reference's own
Python classes on the reference's own C++ compiled for CPU (tests/golden/make_golden.py).
Tolerances (plain FP64 path):
  * waveform / response / spline arrays: |a - b| <= 1e-10 * max|b| over each
    (binary, mode) row, i.e. relative 1e-10 on the row scale (entries that pass through
    zero, like phases and transfer functions, make a pointwise relative test meaningless);
  * log-likelihoods: |dlnL| <= 1e-6 + 1e-11 |lnL| (the golden lnL reach 1e10 with pure-noise
    data, where 1e-6 absolute is below FP64 resolution of the sum).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def rowclose(a, b, rtol=RTOL, axis=-1):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, (a.shape, b.shape)
    scale = np.max(np.abs(b), axis=axis, keepdims=True)
    scale = np.where(scale == 0, 1.0, scale)
    err = np.abs(a - b) / scale
    worst = float(np.nanmax(err)) if err.size else 0.0
    assert np.all(np.isfinite(a) == np.isfinite(b))
    assert worst <= rtol, f"max row-relative error {worst:.3e} > {rtol:.1e}"
    return worst


def lnl_close(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    tol = 1e-6 + 1e-11 * np.abs(b)
    d = np.abs(a - b)
    assert np.all(d <= tol), f"|dlnL| {d} vs tol {tol}"


def _phm(prm, length, tobs=None, direct=False, run_phenomd=False, freqs=None):
    from bbhx_b200 import PhenomHMAmpPhase
    from bbhx_b200.utils.constants import YRSID_SI

    w = PhenomHMAmpPhase(run_phenomd=run_phenomd)
    B = prm.shape[1]
    args = (prm[0], prm[1], prm[2], prm[3], prm[4], np.zeros(B), prm[6], prm[11], length)
    if direct:
        w(*args, freqs=freqs, direct=True)
    else:
        w(*args, Tobs=np.full(B, tobs * YRSID_SI))
    return w


@pytest.mark.parametrize("tag", ["main", "edge"])
def test_phenomhm_regrid_matches_reference(golden, tag):
    prm = golden["params"] if tag == "main" else golden["edge_params"]
    w = _phm(prm, 256, tobs=float(golden["meta"][0]))
    f = w.freqs_shaped.cpu().numpy()
    rowclose(f, golden[f"phm_{tag}_freqs"])
    rowclose(w.amp.cpu().numpy(), golden[f"phm_{tag}_amp"])
    rowclose(w.phase.cpu().numpy(), golden[f"phm_{tag}_phase"])
    rowclose(w.tf.cpu().numpy(), golden[f"phm_{tag}_tf"])


def test_phenomhm_direct_and_ringdown(golden):
    w = _phm(golden["params"], 128, direct=True, freqs=np.logspace(-4, -1, 128))
    rowclose(w.amp.cpu().numpy(), golden["phm_direct_amp"])
    rowclose(w.phase.cpu().numpy(), golden["phm_direct_phase"])
    rowclose(w.tf.cpu().numpy(), golden["phm_direct_tf"])
    np.testing.assert_allclose(w.fringdown.cpu().numpy(), golden["phm_direct_fring"], rtol=1e-12)
    np.testing.assert_allclose(w.fdamp.cpu().numpy(), golden["phm_direct_fdamp"], rtol=1e-12)


def test_phenomd_matches_reference(golden):
    w = _phm(golden["params"], 128, tobs=float(golden["meta"][0]), run_phenomd=True)
    rowclose(w.freqs_shaped.cpu().numpy(), golden["phd_freqs"])
    rowclose(w.amp.cpu().numpy(), golden["phd_amp"])
    rowclose(w.phase.cpu().numpy(), golden["phd_phase"])
    rowclose(w.tf.cpu().numpy(), golden["phd_tf"])


def _response(prm, wf_prefix, golden, tdi_tag="AET", tdi2=True, rescaled=False):
    import torch

    from bbhx_b200 import EqualArmlengthOrbits, LISATDIResponse

    amp = golden[f"{wf_prefix}_amp"]
    B, M, L = amp.shape
    buf = np.zeros((9, B, M, L))
    buf[0], buf[1], buf[2] = amp, golden[f"{wf_prefix}_phase"], golden[f"{wf_prefix}_tf"]
    buf_d = torch.as_tensor(buf.ravel(), device="cuda")
    r = LISATDIResponse(TDItag=tdi_tag, tdi2=tdi2, rescaled=rescaled, orbits=EqualArmlengthOrbits())
    r(golden[f"{wf_prefix}_freqs"].ravel(), prm[7], prm[8], prm[9], prm[10], prm[5], L,
      out_buffer=buf_d, direct=True)
    return buf_d.cpu().numpy().reshape(9, B, M, L)


@pytest.mark.parametrize("tag", ["main", "edge"])
def test_response_aet_tdi2_matches_reference(golden, tag):
    prm = golden["params"] if tag == "main" else golden["edge_params"]
    out = _response(prm, f"phm_{tag}", golden)
    ref = golden[f"resp_{tag}_aet2"]
    for k in range(1, 9):
        rowclose(out[k], ref[k])


def test_response_xyz_and_rescaled_match_reference(golden):
    prm = golden["params"]
    out = _response(prm, "phm_direct", golden, tdi_tag="XYZ", tdi2=False)
    ref = golden["resp_direct_xyz"]
    for k in range(1, 9):
        rowclose(out[k], ref[k])
    out = _response(prm, "phm_direct", golden, tdi2=False, rescaled=True)
    ref = golden["resp_direct_aet1_rescaled"]
    for k in range(1, 9):
        rowclose(out[k], ref[k])


def test_spline_matches_reference(golden):
    from bbhx_b200 import CubicSplineInterpolant

    s = CubicSplineInterpolant(golden["spl_x"], golden["spl_y"])
    for c in ("c1", "c2", "c3"):
        got = getattr(s, f"{c}_shaped").cpu().numpy()[..., :-1]
        ref = golden[f"spl_{c}"][..., :-1]
        worst = rowclose(got, ref, rtol=1e-10)
        print(c, worst)


def _waveform_gen():
    from bbhx_b200 import BBHWaveformFD, EqualArmlengthOrbits

    return BBHWaveformFD(amp_phase_kwargs=dict(run_phenomd=False),
                         response_kwargs=dict(orbits=EqualArmlengthOrbits(), TDItag="AET", tdi2=True))


def test_direct_likelihood_matches_reference(golden, golden_data):
    from bbhx_b200 import Likelihood

    wave = _waveform_gen()
    like = Likelihood(wave, golden_data["f"], golden_data["data"], golden_data["psd"])
    assert abs(like.d_d - float(golden["dl_d_d"])) <= 1e-9 * abs(float(golden["dl_d_d"]))
    ll = like.get_ll(golden["params"], length=1024, t_obs_start=0.0, t_obs_end=golden_data["tobs"])
    lnl_close(ll, golden["dl_lnl"])
    np.testing.assert_allclose(like.d_h.cpu().numpy(), golden["dl_d_h"], rtol=1e-9,
                               atol=1e-9 * np.abs(golden["dl_h_h"]).max() ** 0.5)
    np.testing.assert_allclose(like.h_h.cpu().numpy().real, golden["dl_h_h"].real, rtol=1e-11)


def test_interpolated_template_matches_reference(golden, golden_data):
    wave = _waveform_gen()
    prm = golden["params"]
    tmpl, starts, lengths = wave(*prm, freqs=golden_data["f"], length=1024, t_obs_start=0.0,
                                 t_obs_end=golden_data["tobs"], direct=False, fill=False)
    np.testing.assert_array_equal(np.asarray(starts), golden["dl_start_inds"])
    np.testing.assert_array_equal(np.asarray(lengths), golden["dl_lengths"])
    t0 = tmpl[0].cpu().numpy()[:, ::97]
    rowclose(t0, golden["dl_template0_decim"], rtol=1e-9)


def _hdyn_last_bin(golden):
    """The reference CPU hdyn stops one bin early (Likelihood.cu:150); the GPU form and
    this implementation include bin L-1.  Returns that bin's (d_h, h_h) contribution."""
    r = golden["het_h_sparse"] / golden["het_h0_sparse"]  # (B, 3, L)
    f = golden["het_freqs"]
    L = len(f)
    K = golden["het_data_constants"].reshape(4, 3, L)
    j = L - 1
    df = f[j] - f[j - 1]
    r1 = (r[:, :, j] - r[:, :, j - 1]) / df
    fm = (f[j] + f[j - 1]) / 2
    r0 = r[:, :, j] - r1 * (f[j] - fm)
    dh = (K[0, :, j] * np.conj(r0) + K[1, :, j] * np.conj(r1)).sum(axis=1)
    hh = (K[2, :, j] * np.abs(r0) ** 2 + 2 * K[3, :, j] * np.real(r0 * np.conj(r1))).sum(axis=1)
    return dh, hh


def test_heterodyned_likelihood_matches_reference(golden, golden_data):
    from bbhx_b200 import AET1SensitivityMatrix, HeterodynedLikelihood

    wave = _waveform_gen()
    kw = dict(t_obs_start=0.0, t_obs_end=golden_data["tobs"])
    het = HeterodynedLikelihood(wave, golden_data["f"], golden_data["data"], golden["params"][:, 0],
                                128, template_gen_kwargs=dict(kw),
                                reference_gen_kwargs=dict(kw, length=1024),
                                sens_mat=AET1SensitivityMatrix(golden_data["f"], tdi2=True))
    rowclose(het.freqs.cpu().numpy(), golden["het_freqs"])
    assert abs(het.reference_d_d - float(golden["het_reference_d_d"])) <= 1e-9 * abs(float(golden["het_reference_d_d"]))
    rowclose(het.data_constants.cpu().numpy().reshape(4, 3, -1),
             golden["het_data_constants"].reshape(4, 3, -1), rtol=1e-9)
    ll = het.get_ll(golden["het_walkers"], **kw)
    rowclose(het.h_sparse.cpu().numpy(), golden["het_h_sparse"], rtol=1e-9)
    dh_last, hh_last = _hdyn_last_bin(golden)
    d_h = het.hdyn_d_h.cpu().numpy() - dh_last
    h_h = het.hdyn_h_h.cpu().numpy() - hh_last
    np.testing.assert_allclose(d_h, golden["het_d_h"], rtol=1e-8, atol=1e-6)
    np.testing.assert_allclose(h_h.real, golden["het_h_h"].real, rtol=1e-9)
    ll_adj = -0.5 * (het.reference_d_d + h_h - 2 * d_h).real
    lnl_close(ll_adj, golden["het_lnl"])
    assert np.all(np.isfinite(ll))


def test_direct_likelihood_mixed_precision_error(golden, golden_data):
    """Mixed precision (FP32 amplitude / transfer / products, FP64 phase, t(f), sums) against
    the FP64 form on the golden case: |dlnL| <= 2e-6 * <h|h> (the FP32 relative error times
    the template norm squared; these pure-noise golden data have <h|h> up to 2.6e10)."""
    from bbhx_b200 import Likelihood

    wave = _waveform_gen()
    kw = dict(length=1024, t_obs_start=0.0, t_obs_end=golden_data["tobs"])
    like = Likelihood(wave, golden_data["f"], golden_data["data"], golden_data["psd"])
    ll64 = like.get_ll(golden["params"], **kw)
    hh = like.h_h.cpu().numpy().real
    like.precision = "mixed"
    llm = like.get_ll(golden["params"], **kw)
    d = np.abs(llm - ll64)
    print("mixed |dlnL|", d, "relative to h_h", d / hh)
    assert np.all(d <= 2e-6 * np.maximum(hh, 1.0))
