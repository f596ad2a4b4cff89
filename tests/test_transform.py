"""Frame and sky-mode transforms against golden vectors from the reference's own
transform.py (tests/golden/make_transform_golden.py); numpy on CPU, torch on the GPU."""
import os

import numpy as np
import pytest

from conftest import REPO

G = os.path.join(REPO, "tests", "golden", "transform_golden.npz")


def _check(T, g, conv, back):
    t, lam, beta, psi = (conv(g[k]) for k in ("t", "lam", "beta", "psi"))
    t0 = float(g["t0"])
    np.testing.assert_allclose(np.array([back(v) for v in T.LISA_to_SSB(t, lam, beta, psi, t0)]),
                               g["l2s"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(np.array([back(v) for v in T.SSB_to_LISA(t, lam, beta, psi, t0)]),
                               g["s2l"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(back(T.tSSBfromLframe(t, lam, beta, 0.0)), g["tssb"], rtol=1e-15)
    np.testing.assert_allclose(back(T.tLfromSSBframe(t, lam, beta, 0.0)), g["tl"], rtol=1e-15)
    np.testing.assert_allclose(back(T.modpi(conv(g["modpi_in"]))), g["modpi"], atol=1e-13)
    np.testing.assert_allclose(back(T.mod2pi(conv(g["mod2pi_in"]))), g["mod2pi"], atol=1e-13)
    for kind in ("both", "long", "lat"):
        np.testing.assert_allclose(back(T.mbh_sky_mode_transform(conv(g["coords"].copy()), kind=kind)),
                                   g[f"sky_{kind}"], atol=1e-14)
        np.testing.assert_allclose(
            back(T.mbh_sky_mode_transform(conv(g["coords"].copy()), kind=kind, cos_i=True)),
            g[f"sky_{kind}_cosi"], atol=1e-14)


def test_transforms_numpy_match_reference():
    from bbhx_b200.utils import transform as T

    _check(T, np.load(G), lambda a: np.array(a), lambda a: np.asarray(a))


def test_sky_mode_inplace_and_errors():
    from bbhx_b200.utils.transform import mbh_sky_mode_transform

    g = np.load(G)
    tiled = np.tile(g["coords"], (8, 1))
    out = mbh_sky_mode_transform(tiled, inplace=True)
    assert out is tiled
    np.testing.assert_allclose(out, g["sky_both"], atol=1e-14)
    with pytest.raises(ValueError):
        mbh_sky_mode_transform(g["coords"].copy(), inplace=True)
    with pytest.raises(ValueError):
        mbh_sky_mode_transform(g["coords"].copy(), kind="sideways")


@pytest.mark.gpu
def test_transforms_torch_cuda_match_reference():
    import torch

    from bbhx_b200.utils import transform as T

    _check(T, np.load(G), lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda"),
           lambda a: a.cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a))
