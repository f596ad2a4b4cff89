"""Seeded synthetic workloads for tests and benchmarks.

No public data set is involved: every input is drawn from a seeded generator with the
priors of the massive-black-hole-binary workloads this package is measured on:

* total mass log-uniform in [1e5, 1e7] Msun, mass ratio q ~ U[0.1, 1]
  (m1 = M / (1 + q), m2 = M q / (1 + q)),
* aligned spins chi1z, chi2z ~ U[-0.9, 0.9],
* luminosity distance ~ U[10, 100] Gpc,
* phi_ref ~ U[0, 2 pi], cos(inc) ~ U[-1, 1], lambda ~ U[0, 2 pi], sin(beta) ~ U[-1, 1],
  psi ~ U[0, pi],
* t_ref ~ U[0.8 Tobs, Tobs] (seconds), f_ref = 0.

Parameter arrays use the reference's ordering for ``BBHWaveformFD.__call__``
(``waveformbuild.py:338-352``): m1, m2, chi1z, chi2z, distance, phi_ref, f_ref, inc, lam,
beta, psi, t_ref.
"""
import numpy as np

from .utils.constants import PC_SI, YRSID_SI

PARAM_NAMES = ["m1", "m2", "chi1z", "chi2z", "distance", "phi_ref", "f_ref", "inc", "lam",
               "beta", "psi", "t_ref"]


def draw_params(n, tobs_years, seed):
    """Return a (12, n) float64 array of source parameters."""
    rng = np.random.default_rng(seed)
    mtot = 10.0 ** rng.uniform(5.0, 7.0, n)
    q = rng.uniform(0.1, 1.0, n)
    m1 = mtot / (1.0 + q)
    m2 = mtot * q / (1.0 + q)
    chi1 = rng.uniform(-0.9, 0.9, n)
    chi2 = rng.uniform(-0.9, 0.9, n)
    dist = rng.uniform(10.0, 100.0, n) * 1e9 * PC_SI
    phi_ref = rng.uniform(0.0, 2.0 * np.pi, n)
    f_ref = np.zeros(n)
    inc = np.arccos(rng.uniform(-1.0, 1.0, n))
    lam = rng.uniform(0.0, 2.0 * np.pi, n)
    beta = np.arcsin(rng.uniform(-1.0, 1.0, n))
    psi = rng.uniform(0.0, np.pi, n)
    tobs = tobs_years * YRSID_SI
    t_ref = rng.uniform(0.8 * tobs, tobs, n)
    return np.array([m1, m2, chi1, chi2, dist, phi_ref, f_ref, inc, lam, beta, psi, t_ref])


def perturb_params(center, n, seed, rel_mass=1e-3, abs_spin_angle=1e-2, t_ref_s=10.0):
    """Walkers around ``center`` (12,): relative jitter on total mass and q, absolute jitter
    on spins and angles, seconds on t_ref.  Returns (12, n); column 0 is ``center``."""
    rng = np.random.default_rng(seed)
    c = np.asarray(center, dtype=np.float64)
    mtot = c[0] + c[1]
    q = c[1] / c[0]
    mt = mtot * (1.0 + rel_mass * rng.standard_normal(n))
    qq = np.clip(q * (1.0 + rel_mass * rng.standard_normal(n)), 1e-3, 1.0)
    out = np.repeat(c[:, None], n, axis=1)
    out[0] = mt / (1.0 + qq)
    out[1] = mt * qq / (1.0 + qq)
    out[2] = np.clip(c[2] + abs_spin_angle * rng.standard_normal(n), -0.99, 0.99)
    out[3] = np.clip(c[3] + abs_spin_angle * rng.standard_normal(n), -0.99, 0.99)
    for k in (5, 7, 8, 10):
        out[k] = c[k] + abs_spin_angle * rng.standard_normal(n)
    out[9] = np.clip(c[9] + abs_spin_angle * rng.standard_normal(n), -np.pi / 2, np.pi / 2)
    out[11] = c[11] + t_ref_s * rng.standard_normal(n)
    out[:, 0] = c
    return out


def data_grid(tobs_years, f_lo, f_hi):
    """Uniform data grid df = 1/Tobs covering [f_lo, f_hi]: f_k = k df exactly."""
    df = 1.0 / (tobs_years * YRSID_SI)
    k0 = int(np.ceil(f_lo / df))
    k1 = int(np.floor(f_hi / df))
    return np.arange(k0, k1 + 1, dtype=np.float64) * df


def gaussian_noise(psd, df, seed):
    """Complex Gaussian noise with <|n|^2> = psd / (2 df) per bin, shape of ``psd``; zero in
    notched bins (psd = inf)."""
    rng = np.random.default_rng(seed)
    psd = np.asarray(psd)
    sig = np.sqrt(np.where(np.isfinite(psd), psd, 0.0) / (4.0 * df))
    return sig * (rng.standard_normal(sig.shape) + 1j * rng.standard_normal(sig.shape))


def notch_tdi_zeros(f, psd, half_width=16, armlength=None):
    """Notch the bins around the zeros of the equal-arm A/E/T noise, f = k c / (4 L)
    (the second-generation factor sin^2(2x) and, at even k, the first-generation sin^2(x),
    x = 2 pi f L / c): psd = inf there, i.e. zero noise weight.

    At those frequencies the idealised PSD goes to zero while a spline-interpolated template
    cannot reproduce the transfer function's exact zero, so a single bin within ~1e-9 Hz of
    a zero can dominate <h|h> by many orders of magnitude.  Returns a copy."""
    from .utils.constants import C_SI, L_SI

    L = L_SI if armlength is None else armlength
    f = np.asarray(f, dtype=np.float64)
    out = np.array(psd, dtype=np.float64, copy=True)
    df = f[1] - f[0]
    f0 = C_SI / (4.0 * L)
    for k in range(1, int(f[-1] / f0) + 1):
        fz = k * f0
        m = np.abs(f - fz) <= half_width * df
        out[..., m] = np.inf
    return out
