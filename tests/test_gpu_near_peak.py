"""Mixed precision near the likelihood peak, where a sampler spends its time: templates
within a few units of lnL of the injection (relative 5e-6 on masses, 5e-5 on spins and
angles, 0.05 s on t_ref).  There d - h is noise-level, so the FP32 amplitude / transfer error
enters lnL as ~1e-7 sqrt(<h|h>) rather than the ~1e-7 <h|h> of templates far from the data.
Bound: |lnL_mixed - lnL_FP64| <= 1e-2 for every template, direct and heterodyned.  As in the
benchmark workload, the PSD is notched around the equal-arm TDI noise zero at 30 mHz (zero
noise weight there; the golden noise stream with those bins zeroed)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(golden, golden_data, ci):
    from bbhx_b200 import BBHWaveformFD, EqualArmlengthOrbits
    from bbhx_b200.synthetic import notch_tdi_zeros

    wave = BBHWaveformFD(response_kwargs=dict(orbits=EqualArmlengthOrbits(), TDItag="AET", tdi2=True))
    kw = dict(t_obs_start=0.0, t_obs_end=golden_data["tobs"])
    center = golden["params"][:, ci].copy()
    inj = wave(*[np.atleast_1d(v) for v in center], freqs=golden_data["f"], length=1024, fill=True,
               direct=False, **kw)[0].cpu().numpy()
    psd = notch_tdi_zeros(golden_data["f"], golden_data["psd"])
    noise = np.where(np.isfinite(psd), golden_data["data"], 0.0)
    return wave, kw, center, inj + noise, psd


@pytest.mark.parametrize("ci", [0, 2])
def test_direct_mixed_near_peak(golden, golden_data, ci):
    from bbhx_b200 import Likelihood
    from bbhx_b200.synthetic import perturb_params

    wave, kw, center, data, psd = _setup(golden, golden_data, ci)
    like = Likelihood(wave, golden_data["f"], data, psd)
    P = perturb_params(center, 64, 13, rel_mass=5e-6, abs_spin_angle=5e-5, t_ref_s=0.05)
    ll64 = like.get_ll(P, length=1024, **kw)
    hh = float(np.median(like.h_h.real.cpu().numpy()))
    like.precision = "mixed"
    llm = like.get_ll(P, length=1024, **kw)
    d = np.abs(llm - ll64)
    print("direct", ci, "lnL spread", ll64.max() - ll64.min(), "<h|h>", hh, "max |dlnL|", d.max())
    assert np.all(d <= 1e-2)


@pytest.mark.parametrize("ci", [0, 2])
def test_heterodyned_mixed_near_peak(golden, golden_data, ci):
    from bbhx_b200 import AET1SensitivityMatrix, HeterodynedLikelihood
    from bbhx_b200.synthetic import perturb_params

    wave, kw, center, data, _ = _setup(golden, golden_data, ci)
    het = HeterodynedLikelihood(wave, golden_data["f"], data, center, 128,
                                template_gen_kwargs=dict(kw), reference_gen_kwargs=dict(kw, length=1024),
                                sens_mat=AET1SensitivityMatrix(golden_data["f"], tdi2=True, notch=True))
    W = perturb_params(center, 1024, 11, rel_mass=5e-6, abs_spin_angle=5e-5, t_ref_s=0.05)
    ll64 = het.get_ll(W, **kw)
    het.precision = "mixed"
    llm = het.get_ll(W, **kw)
    d = np.abs(llm - ll64)
    print("het", ci, "lnL spread", ll64.max() - ll64.min(), "<h|h>0", het.reference_h_h, "max |dlnL|", d.max())
    assert np.all(d <= 1e-2)
