"""Host-side argument validation of the public classes (no GPU needed: the checks run before
any device work)."""
import pytest


def test_precision_is_validated():
    from bbhx_b200 import HeterodynedLikelihood, Likelihood
    from bbhx_b200.uneven import UnevenBatch

    with pytest.raises(ValueError, match="precision"):
        Likelihood(None, [0.0, 1.0], [[0.0, 0.0]], [[1.0, 1.0]], precision="fp32")
    with pytest.raises(ValueError, match="precision"):
        HeterodynedLikelihood(None, [0.0, 1.0], [[0.0, 0.0]], None, 8, precision="half")
    with pytest.raises(ValueError, match="precision"):
        UnevenBatch(precision="fp16")
