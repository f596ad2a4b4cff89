"""Full-scale direct likelihood in the plain FP64 form against the reference's own CPU path on
the same inputs: 1-yr data stream, df = 1/Tobs over 1e-5..0.1 Hz (3.16e6 bins, A/E/T TDI2),
injection + Gaussian noise, 6 modes, sparse length 1024; 16 binaries from the benchmark's prior
through the reference's compiled C++ (oracle/_ref), or 1 through the numpy oracle when the
compiled reference is absent.  Tolerance |dlnL| <= 1e-6 + 2e-11 |lnL|: |lnL| ~ 1e7 here is the
difference of sums over 3.2e6 bins (d_d ~ 2e7), which the two sides accumulate in different
orders (per-tile partials vs one dot product per binary), so FP64 agreement stops near 1e-11 of
|lnL| (the golden-size bound is 1e-6 + 1e-11 |lnL| over 1.6e5 bins)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_fullscale_direct_lnl_matches_reference():
    from bbhx_b200 import BBHWaveformFD, EqualArmlengthOrbits, Likelihood
    from bbhx_b200.sensitivity import aet_psd
    from bbhx_b200.synthetic import data_grid, draw_params, gaussian_noise, notch_tdi_zeros
    from oracle.build_ref import OUT
    from oracle.pipeline import RefPipeline

    tobs = 1.0
    f = data_grid(tobs, 1e-5, 0.1)
    psd = notch_tdi_zeros(f, np.array([aet_psd(f, c, tdi2=True) for c in "AET"]))
    wave = BBHWaveformFD(response_kwargs=dict(orbits=EqualArmlengthOrbits(), TDItag="AET", tdi2=True))
    kw = dict(length=1024, t_obs_start=0.0, t_obs_end=tobs)
    inj = draw_params(1, tobs, 1241)
    h = wave(*inj, freqs=f, direct=False, fill=True, combine=True, **kw)
    data = gaussian_noise(psd, f[1] - f[0], 99) + h.cpu().numpy()
    have_ref = os.path.isfile(OUT)
    P = draw_params(16 if have_ref else 1, tobs, 1234)
    like = Likelihood(wave, f, data, psd)
    ll = like.get_ll(P, **kw)
    pipe = RefPipeline("ref" if have_ref else "np")
    ref = pipe.direct_lnl(P, f, data, psd, **kw)[0]
    d = np.abs(ll - ref)
    print(pipe.K.name, len(f), "max |dlnL|", d.max(), "max relative", np.max(d / np.abs(ref)))
    assert len(f) > 3_000_000
    assert np.all(d <= 1e-6 + 2e-11 * np.abs(ref))
