import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

GOLDEN = os.path.join(REPO, "tests", "golden", "reference_golden.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: long-running")


def _has_cuda():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_cuda():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN))


@pytest.fixture(scope="session")
def golden_data():
    """Regenerate the golden data stream (pure seeded noise) and its grid / PSD."""
    from bbhx_b200.sensitivity import aet_psd
    from bbhx_b200.synthetic import data_grid, gaussian_noise

    g = np.load(GOLDEN)
    tobs, flo, fhi, _, seed_noise = g["meta"][:5]
    f = data_grid(tobs, flo, fhi)
    df = f[1] - f[0]
    psd = np.array([aet_psd(f, c, tdi2=True) for c in "AET"])
    data = gaussian_noise(psd, df, int(seed_noise))
    return dict(f=f, psd=psd, data=data, tobs=float(tobs))
