"""Analytic LISA noise PSDs for the A, E, T channels.

The reference takes its PSDs from lisatools (``likelihood.py:23,359-362``;
``tests/test_bbhx.py:224-226``), which is not part of this project.  This module writes
the standard two-component LISA noise model out explicitly:

* test-mass acceleration noise  3e-15 m s^-2 / sqrt(Hz) with the usual
  (1 + (0.4 mHz / f)^2)(1 + (f / 8 mHz)^4) colouring,
* optical-metrology noise 15e-12 m / sqrt(Hz) with (1 + (2 mHz / f)^4),

both converted to fractional-frequency units, combined into the first-generation
A/E and T PSDs (x = 2 pi f L / c):

    S_A = S_E = 8 sin^2 x [ 2 S_acc (3 + 2 cos x + cos 2x) + S_oms (2 + cos x) ]
    S_T = 32 sin^2 x sin^2(x/2) [ 4 S_acc sin^2(x/2) + S_oms ]

and, when ``tdi2`` is set, multiplied by |2 sin 2x|^2 -- the response's first- to
second-generation factor -2i sin(4x') e^{4ix'} with its x' = pi f L / c = x / 2
(``Response.cu:205,247-258``), so that signal and noise vanish at the same frequencies.
"""
import numpy as np

from .utils.constants import C_SI, L_SI


def _noise_components(f, acc=3.0e-15, oms=15.0e-12):
    f = np.asarray(f, dtype=np.float64)
    sa_a = acc**2 * (1.0 + (0.4e-3 / f) ** 2) * (1.0 + (f / 8.0e-3) ** 4)
    sa_nu = sa_a * (2.0 * np.pi * f) ** -4 * (2.0 * np.pi * f / C_SI) ** 2
    soms_d = oms**2 * (1.0 + (2.0e-3 / f) ** 4)
    soms_nu = soms_d * (2.0 * np.pi * f / C_SI) ** 2
    return sa_nu, soms_nu


def aet_psd(f, channel, tdi2=False, armlength=L_SI, acc=3.0e-15, oms=15.0e-12):
    """PSD of channel ``"A"``, ``"E"`` or ``"T"`` at frequencies ``f`` (Hz)."""
    f = np.asarray(f, dtype=np.float64)
    sa_nu, soms_nu = _noise_components(f, acc, oms)
    x = 2.0 * np.pi * armlength / C_SI * f
    if channel in ("A", "E", 0, 1):
        out = 8.0 * np.sin(x) ** 2 * (
            2.0 * sa_nu * (3.0 + 2.0 * np.cos(x) + np.cos(2.0 * x)) + soms_nu * (2.0 + np.cos(x))
        )
    elif channel in ("T", 2):
        out = 32.0 * np.sin(x) ** 2 * np.sin(x / 2.0) ** 2 * (
            4.0 * sa_nu * np.sin(x / 2.0) ** 2 + soms_nu
        )
    else:
        raise ValueError(f"unknown channel {channel!r}")
    if tdi2:
        out = out * (2.0 * np.sin(2.0 * x)) ** 2
    return out


class AET1SensitivityMatrix:
    """A/E/T PSD container with the call pattern the heterodyne setup uses
    (``likelihood.py:361,493-496``: ``update_frequency_arr`` then ``[0]``, ``[1]``, ``[2]``)."""

    def __init__(self, f, tdi2=False, notch=False, **kwargs):
        self.tdi2 = tdi2
        self.notch = notch
        self.kwargs = kwargs
        self.update_frequency_arr(f)

    def update_frequency_arr(self, f):
        self.frequency_arr = np.asarray(f, dtype=np.float64)
        self.sens_mat = np.asarray(
            [aet_psd(self.frequency_arr, c, tdi2=self.tdi2, **self.kwargs) for c in "AET"]
        )
        if self.notch:
            from .synthetic import notch_tdi_zeros

            self.sens_mat = notch_tdi_zeros(self.frequency_arr, self.sens_mat)

    def __getitem__(self, i):
        return self.sens_mat[i]


SensitivityMatrix = AET1SensitivityMatrix
