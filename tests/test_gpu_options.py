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
