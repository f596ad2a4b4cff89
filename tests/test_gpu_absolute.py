"""FP64 lnL at the absolute 1e-6 bar, and the summation-order floor shown, not assumed.

1. Walkers near a zero-noise injection.  The data are the injection itself
   (``BBHWaveformFD(fill=True, combine=True)``), so lnL = -<d-h|d-h>/2 is 0 at the injection
   and a few hundred to a few thousand for the walkers around it.  That is the regime where an
   absolute 1e-6 is a meaningful bar (lnL(data = template, no noise) = 0 is also a known answer).
   Both sides read the same data arrays: the GPU lnL (plain FP64) must agree with the
   reference's compiled CPU path (oracle/_ref, driven by oracle/pipeline.py) to
   |dlnL| <= 1e-6 ABSOLUTE, at the CPU-runnable size (Tobs = 0.1 yr, 1.6e5 bins) and at full
   scale (Tobs = 1 yr, 3.16e6 bins).  Each case is also checked against a compensated sum:
   <d|h>, <h|h> and <d|d> formed from the reference's own per-bin template values
   (TemplateInterpFD on the compiled reference) and summed with math.fsum, i.e. the reference's
   terms without any summation-order error.

2. Loud templates on pure noise (|lnL| up to ~1e10, the golden streams).  Here 1e-6 absolute
   is below one FP64 ulp of the sums (ulp(1e10) = 1.9e-6), so the bar is relative.  The test
   computes the compensated sums of the reference's per-bin terms and checks that the GPU's
   <d|h> and <h|h> sit within 3e-12 of sum |term| of them, while printing how far the
   reference's own (uncompensated) sums are from the same exact values.
"""
import math
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _exact_sums(pipe, params, f, data, psd, kw):
    """<d|h>, <h|h> per binary and <d|d> from the reference's per-bin template values, summed
    with math.fsum (the products are the FP64 products the reference forms,
    Likelihood.cu:356-375,492-529)."""
    df = np.zeros_like(psd)
    df[:, 1:] = np.diff(f)
    df[:, 0] = df[:, 1]
    nf = np.sqrt(1.0 / psd * df)
    dw = nf * np.asarray(data, dtype=np.complex128)
    d_d = 4 * (math.fsum((dw.real ** 2).ravel()) + math.fsum((dw.imag ** 2).ravel()))
    tmpl, starts, lengths = pipe.templates(params, f, **kw)
    out = []
    for h, s, n in zip(tmpl, starts, lengths):
        h = h.reshape(3, n) * nf[:, s:s + n]
        d = dw[:, s:s + n]
        re = d.real * h.real + d.imag * h.imag
        im = d.real * h.imag - d.imag * h.real
        hh = h.real * h.real + h.imag * h.imag
        out.append((4 * math.fsum(re.ravel()), 4 * math.fsum(im.ravel()), 4 * math.fsum(hh.ravel()),
                    4 * float(np.abs(re).sum()), 4 * float(hh.sum())))
    return np.array(out), d_d


def _near_injection_case(tobs, flo, fhi, nwalk, seed, scale):
    from bbhx_b200 import BBHWaveformFD, EqualArmlengthOrbits, Likelihood
    from bbhx_b200.sensitivity import aet_psd
    from bbhx_b200.synthetic import data_grid, draw_params, perturb_params
    from oracle.build_ref import OUT
    from oracle.pipeline import RefPipeline

    if not os.path.isfile(OUT):
        pytest.skip("compiled reference (oracle/_ref) not present")
    f = data_grid(tobs, flo, fhi)
    psd = np.array([aet_psd(f, c, tdi2=True) for c in "AET"])
    wave = BBHWaveformFD(response_kwargs=dict(orbits=EqualArmlengthOrbits(), TDItag="AET", tdi2=True))
    kw = dict(length=1024, t_obs_start=0.0, t_obs_end=tobs)
    inj = draw_params(1, tobs, seed)
    data = wave(*inj, freqs=f, direct=False, fill=True, combine=True, **kw).cpu().numpy()
    P = np.concatenate([inj, perturb_params(inj[:, 0], nwalk, seed + 1, rel_mass=2e-5 * scale,
                                            abs_spin_angle=2e-4 * scale, t_ref_s=0.5 * scale)],
                       axis=1)
    like = Likelihood(wave, f, data, psd)
    ll = like.get_ll(P, **kw)
    pipe = RefPipeline("ref")
    ref, ref_dh, ref_hh, ref_dd = pipe.direct_lnl(P, f, data, psd, **kw)
    sums, d_d = _exact_sums(pipe, P, f, data, psd, kw)
    exact = -0.5 * (d_d + sums[:, 2] - 2 * sums[:, 0])
    print(f"N={len(f)} lnL {np.round(ref, 3)}")
    print("  |gpu - ref|  ", np.abs(ll - ref))
    print("  |gpu - exact|", np.abs(ll - exact))
    print("  |ref - exact|", np.abs(ref - exact))
    return ll, ref, exact


def test_near_injection_absolute_1e6_cpu_size():
    ll, ref, exact = _near_injection_case(0.1, 1e-4, 5e-2, 7, 3041, 2.0)
    assert abs(ref[0]) <= 1e-6  # lnL(data = template, no noise) = 0
    assert np.max(np.abs(ref[1:])) > 50.0  # the walkers sit in the 1e2..1e3 regime
    assert np.all(np.abs(ll - ref) <= 1e-6)
    assert np.all(np.abs(ll - exact) <= 1e-6)


def test_near_injection_absolute_1e6_full_scale():
    ll, ref, exact = _near_injection_case(1.0, 1e-5, 0.1, 3, 1241, 3.0)
    assert abs(ref[0]) <= 1e-6
    assert np.all(np.abs(ll - ref) <= 1e-6)
    assert np.all(np.abs(ll - exact) <= 1e-6)


def test_loud_templates_against_compensated_sums(golden, golden_data):
    """Pure-noise golden stream, |lnL| up to ~1e10: the GPU's <d|h>, <h|h> against the exact sum
    of the reference's per-bin terms, relative to the sum of the terms' magnitudes."""
    from bbhx_b200 import BBHWaveformFD, EqualArmlengthOrbits, Likelihood
    from oracle.build_ref import OUT
    from oracle.pipeline import RefPipeline

    if not os.path.isfile(OUT):
        pytest.skip("compiled reference (oracle/_ref) not present")
    f, psd, data, tobs = (golden_data[k] for k in ("f", "psd", "data", "tobs"))
    P = golden["params"]
    kw = dict(length=1024, t_obs_start=0.0, t_obs_end=tobs)
    wave = BBHWaveformFD(amp_phase_kwargs=dict(run_phenomd=False),
                         response_kwargs=dict(orbits=EqualArmlengthOrbits(), TDItag="AET", tdi2=True))
    like = Likelihood(wave, f, data, psd)
    like.get_ll(P, **kw)
    gdh = like.d_h.cpu().numpy()
    ghh = like.h_h.real.cpu().numpy()
    sums, _ = _exact_sums(RefPipeline("ref"), P, f, data, psd, kw)
    rdh, rhh = golden["dl_d_h"], golden["dl_h_h"].real
    mag_dh, mag_hh = sums[:, 3], sums[:, 4]
    e_gpu_dh = np.abs(gdh.real - sums[:, 0]) / mag_dh
    e_gpu_hh = np.abs(ghh - sums[:, 2]) / mag_hh
    e_ref_dh = np.abs(rdh.real - sums[:, 0]) / mag_dh
    e_ref_hh = np.abs(rhh - sums[:, 2]) / mag_hh
    print("<h|h>", sums[:, 2])
    print("gpu  vs exact, relative to sum|terms|: d_h", e_gpu_dh, "h_h", e_gpu_hh)
    print("ref  vs exact, relative to sum|terms|: d_h", e_ref_dh, "h_h", e_ref_hh)
    assert np.all(e_gpu_dh <= 3e-12) and np.all(e_gpu_hh <= 3e-12)
