"""Kernel-level GPU checks that need no reference fixture."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_hot_loop_sincos_matches_cuda():
    """The Cody-Waite + Taylor sine/cosine of the fused kernels agrees with CUDA's sincos
    to 4e-16 absolute over phases up to 1e8 rad (waveform phases stay below ~1e7 rad)."""
    import torch

    from bbhx_b200 import _lib

    rng = np.random.default_rng(3)
    x = np.concatenate([rng.uniform(-10, 10, 200000), rng.uniform(-1e8, 1e8, 200000),
                        np.array([0.0, np.pi / 4, -np.pi / 4, np.pi / 2, np.pi, 1e7 * np.pi])])
    xd = torch.as_tensor(x, device="cuda")
    out = torch.empty(4 * len(x), dtype=torch.float64, device="cuda")
    _lib.call("bbhx_selftest_sincos", _lib.dptr(xd), _lib.dptr(out), len(x), _lib.stream())
    o = out.cpu().numpy().reshape(-1, 4)
    assert np.max(np.abs(o[:, 0] - o[:, 2])) < 4e-16 * max(1.0, 1.0)
    assert np.max(np.abs(o[:, 1] - o[:, 3])) < 4e-16
    # and against numpy (host libm) on the small range
    small = np.abs(x) < 10
    assert np.max(np.abs(o[small, 0] - np.sin(x[small]))) < 4e-16
    assert np.max(np.abs(o[small, 1] - np.cos(x[small]))) < 4e-16
