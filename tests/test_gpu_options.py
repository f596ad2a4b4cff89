"""API switches through the fused direct likelihood, against the numpy oracle pipeline
(oracle/pipeline.py with oracle/kernels_np.py) on the golden data: XYZ TDI (first
generation), rescaled first-generation AET, PhenomD only (run_phenomd) and a mode subset.
Tolerance: |dlnL| <= 1e-6 + 1e-10 |lnL| (both sides are FP64 restatements pinned to the
reference at <= 1e-12 on the waveform and transfer arrays)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = {
    "xyz_tdi1": dict(TDItag="XYZ", tdi2=False, rescaled=False, run_phenomd=False, modes=None),
    "aet1_rescaled": dict(TDItag="AET", tdi2=False, rescaled=True, run_phenomd=False, modes=None),
    "phenomd": dict(TDItag="AET", tdi2=True, rescaled=False, run_phenomd=True, modes=None),
    "modes_22_33": dict(TDItag="AET", tdi2=True, rescaled=False, run_phenomd=False,
                        modes=[(2, 2), (3, 3)]),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_direct_lnl_switches_match_oracle(golden, golden_data, case):
    from bbhx_b200 import BBHWaveformFD, EqualArmlengthOrbits, Likelihood
    from oracle.pipeline import RefPipeline

    c = CASES[case]
    wave = BBHWaveformFD(amp_phase_kwargs=dict(run_phenomd=c["run_phenomd"]),
                         response_kwargs=dict(orbits=EqualArmlengthOrbits(), TDItag=c["TDItag"],
                                              tdi2=c["tdi2"], rescaled=c["rescaled"]))
    like = Likelihood(wave, golden_data["f"], golden_data["data"], golden_data["psd"])
    P = golden["params"][:, :2]
    kw = dict(length=512, t_obs_start=0.0, t_obs_end=golden_data["tobs"])
    if c["modes"] is not None:
        kw["modes"] = c["modes"]
    ll = like.get_ll(P, **kw)
    pipe = RefPipeline("np", TDItag=c["TDItag"], tdi2=c["tdi2"], rescaled=c["rescaled"],
                       run_phenomd=c["run_phenomd"])
    ref, _, _, _ = pipe.direct_lnl(P, golden_data["f"], golden_data["data"], golden_data["psd"], **kw)
    d = np.abs(ll - ref)
    print(case, ll, ref, d)
    assert np.all(d <= 1e-6 + 1e-10 * np.abs(ref))


def test_heterodyned_fused_xyz_matches_chain(golden, golden_data):
    from bbhx_b200 import AET1SensitivityMatrix, BBHWaveformFD, EqualArmlengthOrbits, HeterodynedLikelihood

    kw = dict(t_obs_start=0.0, t_obs_end=golden_data["tobs"])
    out = {}
    for prec in (None, "fp64"):
        wave = BBHWaveformFD(response_kwargs=dict(orbits=EqualArmlengthOrbits(), TDItag="XYZ", tdi2=False))
        het = HeterodynedLikelihood(wave, golden_data["f"], golden_data["data"], golden["params"][:, 0], 96,
                                    template_gen_kwargs=dict(kw), reference_gen_kwargs=dict(kw, length=1024),
                                    sens_mat=AET1SensitivityMatrix(golden_data["f"], tdi2=False),
                                    precision=prec)
        out[prec] = het.get_ll(golden["het_walkers"], **kw)
    np.testing.assert_allclose(out["fp64"], out[None], rtol=1e-10, atol=1e-6)


def test_fill_and_per_mode_outputs_match_reference(golden, golden_data):
    """BBHWaveformFD's fill=True streams (combined [3, N] and one row per binary [B, 3, N],
    placed by the fill kernel; waveformbuild.py:663-693) and the direct=True, compress=False
    per-mode templates [B, 3, M, L] (waveformbuild.py:603-636) against the reference's own
    outputs (tests/golden, decimated every 97th bin plus exact per-row magnitude sums):
    row-relative 1e-9, the template bar of the InterpTDI parity test."""
    from bbhx_b200 import BBHWaveformFD, EqualArmlengthOrbits

    from test_gpu_parity import rowclose

    wave = BBHWaveformFD(amp_phase_kwargs=dict(run_phenomd=False),
                         response_kwargs=dict(orbits=EqualArmlengthOrbits(), TDItag="AET", tdi2=True))
    P = golden["params"][:, :3]
    f, tobs = golden_data["f"], golden_data["tobs"]
    kw = dict(length=1024, t_obs_start=0.0, t_obs_end=tobs)
    comb = wave(*P, freqs=f, direct=False, fill=True, combine=True, **kw).cpu().numpy()
    assert comb.shape == (3, len(f))
    rowclose(comb[:, ::97], golden["wf_combine_decim"], rtol=1e-9)
    np.testing.assert_allclose(np.abs(comb).sum(axis=-1), golden["wf_combine_abs_sum"], rtol=1e-9)
    each = wave(*P, freqs=f, direct=False, fill=True, combine=False, **kw).cpu().numpy()
    assert each.shape == (3, 3, len(f))
    rowclose(each[:, :, ::97], golden["wf_each_decim"], rtol=1e-9)
    np.testing.assert_allclose(np.abs(each).sum(axis=-1), golden["wf_each_abs_sum"], rtol=1e-9)
    # the combined stream is the sum of the rows (overlapping supports added in binary order)
    np.testing.assert_allclose(each.sum(axis=0), comb, rtol=0, atol=1e-12 * np.abs(comb).max())
    modes = wave(*P, freqs=golden["wf_modes_freqs"], direct=True, compress=False,
                 t_obs_start=0.0, t_obs_end=tobs).cpu().numpy()
    assert modes.shape == golden["wf_modes"].shape
    rowclose(modes, golden["wf_modes"], rtol=1e-9)
