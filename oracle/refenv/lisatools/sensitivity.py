"""``lisatools.sensitivity`` stand-in (likelihood.py:23, tests/test_bbhx.py:30)."""
from bbhx_b200.sensitivity import AET1SensitivityMatrix, SensitivityMatrix, aet_psd  # noqa: F401


def get_sensitivity(f, sens_fn="A1TDISens", **kwargs):
    return aet_psd(f, sens_fn[0], **kwargs)
