"""Gradients d lnL / d theta (11 parameters) against central finite differences of the FP64
lnL, and the torch.autograd front end.

Finite-difference steps (central, FP64): relative 1e-6 for masses and distance, absolute
1e-6 for spins and angles, 1e-3 s for t_ref.  Agreement bound per component:
direct likelihood |g - fd| <= 1e-4 |fd| (the derivative follows the sparse knots as the
observation-window regrid moves them); heterodyned |g - fd| <= 1e-4 |fd| + 1e-7 max_k
|fd_k * step_scale_k| (the second term absorbs components that are zero to FD accuracy).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROWS = (0, 1, 2, 3, 4, 5, 7, 8, 9, 10, 11)


def _steps(p):
    rel = {0: 1e-6, 1: 1e-6, 4: 1e-6}
    absolute = {2: 1e-6, 3: 1e-6, 5: 1e-6, 7: 1e-6, 8: 1e-6, 9: 1e-6, 10: 1e-6, 11: 1e-3}
    return np.array([rel[r] * abs(p[r]) if r in rel else absolute[r] for r in ROWS])


def _central_fd(fn, P):
    """fn: [12, B] -> lnL [B]; returns [B, 11] central differences."""
    B = P.shape[1]
    out = np.zeros((B, len(ROWS)))
    for k, r in enumerate(ROWS):
        h = np.array([_steps(P[:, b])[k] for b in range(B)])
        Pp, Pm = P.copy(), P.copy()
        Pp[r] += h
        Pm[r] -= h
        out[:, k] = (fn(Pp) - fn(Pm)) / (2 * h)
    return out


def _check(grad, fd, P, floor=1e-7):
    for b in range(grad.shape[0]):
        scale = np.max(np.abs(fd[b] * _steps(P[:, b]))) / 1e-6
        tol = 1e-4 * np.abs(fd[b]) + floor * scale
        bad = np.abs(grad[b] - fd[b]) > tol
        assert not np.any(bad), (b, np.array(ROWS)[bad], grad[b][bad], fd[b][bad])


def _het_setup(golden, golden_data, center_index):
    from bbhx_b200 import AET1SensitivityMatrix, BBHWaveformFD, EqualArmlengthOrbits, HeterodynedLikelihood
    from bbhx_b200.synthetic import perturb_params

    wave = BBHWaveformFD(amp_phase_kwargs=dict(run_phenomd=False),
                         response_kwargs=dict(orbits=EqualArmlengthOrbits(), TDItag="AET", tdi2=True))
    kw = dict(t_obs_start=0.0, t_obs_end=golden_data["tobs"])
    center = golden["params"][:, center_index].copy()
    inj = wave(*[np.atleast_1d(v) for v in center], freqs=golden_data["f"], length=1024, fill=True,
               direct=False, **kw)[0].cpu().numpy()
    het = HeterodynedLikelihood(wave, golden_data["f"], inj + golden_data["data"], center, 128,
                                template_gen_kwargs=dict(kw), reference_gen_kwargs=dict(kw, length=1024),
                                sens_mat=AET1SensitivityMatrix(golden_data["f"], tdi2=True))
    P = perturb_params(center, 4, 23, rel_mass=1e-4, abs_spin_angle=1e-3, t_ref_s=1.0)
    return het, kw, P


@pytest.mark.parametrize("center_index", [0, 2])
def test_heterodyned_gradient_matches_central_fd(golden, golden_data, center_index):
    het, kw, P = _het_setup(golden, golden_data, center_index)
    ll, grad = het.get_ll_and_grad(P, **kw)
    ll = ll.cpu().numpy()
    grad = grad.cpu().numpy()
    ll_ref = het.get_ll(P, **kw)
    np.testing.assert_allclose(ll, ll_ref, rtol=1e-12, atol=1e-8)
    fd = _central_fd(lambda Q: het.get_ll(Q, **kw), P)
    print("grad", grad[0], "\nfd  ", fd[0])
    _check(grad, fd, P)


def test_heterodyned_autograd_backward(golden, golden_data):
    import torch

    het, kw, P = _het_setup(golden, golden_data, 2)
    x = torch.tensor(P, dtype=torch.float64, device="cuda", requires_grad=True)
    ll = het.loglike_torch(x, **kw)
    w = torch.arange(1, P.shape[1] + 1, dtype=torch.float64, device="cuda")
    (ll * w).sum().backward()
    _, grad = het.get_ll_and_grad(P, **kw)
    expect = np.zeros((12, P.shape[1]))
    expect[list(ROWS)] = (grad.cpu().numpy() * w.cpu().numpy()[:, None]).T
    np.testing.assert_allclose(x.grad.cpu().numpy(), expect, rtol=1e-12, atol=0)
    assert np.all(x.grad.cpu().numpy()[6] == 0.0)


def _direct_setup(golden, golden_data, center_index):
    from bbhx_b200 import BBHWaveformFD, EqualArmlengthOrbits, Likelihood
    from bbhx_b200.synthetic import perturb_params

    wave = BBHWaveformFD(amp_phase_kwargs=dict(run_phenomd=False),
                         response_kwargs=dict(orbits=EqualArmlengthOrbits(), TDItag="AET", tdi2=True))
    kw = dict(t_obs_start=0.0, t_obs_end=golden_data["tobs"], length=1024)
    center = golden["params"][:, center_index].copy()
    inj = wave(*[np.atleast_1d(v) for v in center], freqs=golden_data["f"], fill=True, direct=False,
               **kw)[0].cpu().numpy()
    data = inj + golden_data["data"]
    like = Likelihood(wave, golden_data["f"], data, golden_data["psd"])
    like.test_data = data
    P = perturb_params(center, 3, 29, rel_mass=1e-4, abs_spin_angle=1e-3, t_ref_s=1.0)
    return like, kw, P


@pytest.mark.parametrize("center_index", [0, 2])
def test_direct_gradient_matches_central_fd(golden, golden_data, center_index):
    like, kw, P = _direct_setup(golden, golden_data, center_index)
    ll, grad = like.get_ll_and_grad(P, **kw)
    ll = ll.cpu().numpy()
    grad = grad.cpu().numpy()
    np.testing.assert_allclose(ll, like.get_ll(P, **kw), rtol=1e-12, atol=1e-8)
    fd = _central_fd(lambda Q: like.get_ll(Q, **kw), P)
    print("grad", grad[0], "\nfd  ", fd[0], "\nrel ", np.max(np.abs(grad - fd) / np.abs(fd), axis=0))
    _check(grad, fd, P, floor=0.0)


def test_direct_autograd_backward(golden, golden_data):
    import torch

    like, kw, P = _direct_setup(golden, golden_data, 2)
    x = torch.tensor(P, dtype=torch.float64, device="cuda", requires_grad=True)
    ll = like.loglike_torch(x, **kw)
    ll.sum().backward()
    _, grad = like.get_ll_and_grad(P, **kw)
    expect = np.zeros((12, P.shape[1]))
    expect[list(ROWS)] = grad.cpu().numpy().T
    np.testing.assert_allclose(x.grad.cpu().numpy(), expect, rtol=1e-12, atol=0)


def test_direct_gradient_matches_fd_of_oracle_lnl(golden, golden_data):
    """The GPU gradient against central differences of the oracle's CPU lnL on the same data:
    the reference's own C++ compiled for CPU (oracle/_ref) on 32 samples around the injection
    when it is built, else the numpy restatement (oracle/kernels_np.py) on one."""
    import os

    from bbhx_b200.synthetic import perturb_params
    from oracle.build_ref import OUT
    from oracle.pipeline import RefPipeline

    like, kw, P = _direct_setup(golden, golden_data, 2)
    n = 32 if os.path.isfile(OUT) else 1
    P = perturb_params(P[:, 0], n, 31, rel_mass=1e-4, abs_spin_angle=1e-3, t_ref_s=1.0)
    _, grad = like.get_ll_and_grad(P, **kw)
    grad = grad.cpu().numpy()
    pipe = RefPipeline("ref" if os.path.isfile(OUT) else "np")
    fd = _central_fd(lambda Q: pipe.direct_lnl(Q, golden_data["f"], like.test_data,
                                               golden_data["psd"], **kw)[0], P)
    print(pipe.K.name, "grad", grad[0], "\nfd  ", fd[0], "\nrel ", np.max(np.abs(grad - fd) / np.abs(fd), axis=0))
    _check(grad, fd, P, floor=0.0)
