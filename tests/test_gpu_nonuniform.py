"""A non-uniform data grid (log-spaced, 4e4 bins over 0.1-50 mHz): the reference accepts any
sorted grid (its df comes from np.diff), and the fused kernels read the grid rather than
assuming a uniform spacing.  FP64 lnL against the reference's compiled CPU path (numpy oracle
when it is absent), 1e-6 + 1e-11 |lnL|; the gradient against central differences of the GPU
lnL with the bound of tests/test_gpu_gradient.py."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(golden):
    from bbhx_b200 import BBHWaveformFD, EqualArmlengthOrbits, Likelihood
    from bbhx_b200.sensitivity import aet_psd

    tobs = 0.1
    f = np.geomspace(1e-4, 5e-2, 40000)
    psd = np.array([aet_psd(f, c, tdi2=True) for c in "AET"])
    rng = np.random.default_rng(5)
    noise = np.sqrt(psd / 4.0 / np.gradient(f)) * (rng.standard_normal(psd.shape)
                                                    + 1j * rng.standard_normal(psd.shape))
    wave = BBHWaveformFD(response_kwargs=dict(orbits=EqualArmlengthOrbits(), TDItag="AET", tdi2=True))
    kw = dict(t_obs_start=0.0, t_obs_end=tobs, length=1024)
    center = golden["params"][:, 2].copy()
    inj = wave(*[np.atleast_1d(v) for v in center], freqs=f, fill=True, direct=False, **kw)[0]
    data = inj.cpu().numpy() + noise
    return Likelihood(wave, f, data, psd), f, data, psd, kw, center


def test_nonuniform_grid_lnl_matches_reference(golden):
    from oracle.build_ref import OUT
    from oracle.pipeline import RefPipeline

    like, f, data, psd, kw, _ = _problem(golden)
    P = golden["params"][:, :4]
    ll = like.get_ll(P, **kw)
    pipe = RefPipeline("ref" if os.path.isfile(OUT) else "np")
    ref = pipe.direct_lnl(P, f, data, psd, **kw)[0]
    d = np.abs(ll - ref)
    print(pipe.K.name, ll, ref, d)
    assert np.all(d <= 1e-6 + 1e-11 * np.abs(ref))


def test_nonuniform_grid_gradient_matches_central_fd(golden):
    from bbhx_b200.synthetic import perturb_params
    from test_gpu_gradient import _central_fd, _check

    like, _, _, _, kw, center = _problem(golden)
    P = perturb_params(center, 2, 29, rel_mass=1e-4, abs_spin_angle=1e-3, t_ref_s=1.0)
    ll, grad = like.get_ll_and_grad(P, **kw)
    np.testing.assert_allclose(ll.cpu().numpy(), like.get_ll(P, **kw), rtol=1e-12, atol=1e-8)
    fd = _central_fd(lambda Q: like.get_ll(Q, **kw), P)
    print("grad", grad.cpu().numpy()[0], "\nfd  ", fd[0])
    _check(grad.cpu().numpy(), fd, P)
