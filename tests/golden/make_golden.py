"""Generate the golden fixtures in tests/golden/ from the REFERENCE implementation.

Runs only where the reference checkout exists (this script reads it; the fixtures it
writes are what travels).  The reference's own Python classes
(``bbhx.waveforms.phenomhm.PhenomHMAmpPhase``, ``bbhx.response.fastfdresponse.
LISATDIResponse``, ``bbhx.utils.interpolate.CubicSplineInterpolant``,
``bbhx.waveformbuild.BBHWaveformFD``, ``bbhx.likelihood.Likelihood`` /
``HeterodynedLikelihood``) are imported unmodified and run on the reference's own C++
compiled for CPU (``oracle/_ref/libbbhx_ref.so``), with ``oracle/refenv`` standing in
for gpubackendtools / lisatools.

Data streams are pure seeded Gaussian noise so every consumer can regenerate them
bit-for-bit from the stored seed with ``bbhx_b200.synthetic.gaussian_noise``.

Usage:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, REPO)
from oracle.build_ref import REF_ROOT  # noqa: E402

REF_SRC = os.path.join(REF_ROOT, "src")
sys.path.insert(0, os.path.join(REPO, "oracle", "refenv"))
sys.path.insert(0, REPO)
sys.path.insert(0, REF_SRC)

from oracle.build_ref import build as build_ref  # noqa: E402

build_ref()

import warnings  # noqa: E402

warnings.filterwarnings("ignore")
from bbhx.likelihood import HeterodynedLikelihood, Likelihood  # noqa: E402
from bbhx.response.fastfdresponse import LISATDIResponse  # noqa: E402
from bbhx.utils.interpolate import CubicSplineInterpolant  # noqa: E402
from bbhx.waveformbuild import BBHWaveformFD  # noqa: E402
from bbhx.waveforms.phenomhm import PhenomHMAmpPhase  # noqa: E402
from lisatools.detector import EqualArmlengthOrbits  # noqa: E402

from bbhx_b200.sensitivity import aet_psd  # noqa: E402
from bbhx_b200.synthetic import data_grid, draw_params, gaussian_noise, perturb_params  # noqa: E402
from bbhx_b200.utils.constants import MSUN_SI, YRSID_SI  # noqa: E402

TOBS = 0.1  # years (the CPU-runnable configuration)
F_LO, F_HI = 1e-4, 5e-2
SEED_PARAMS = 20240601
SEED_NOISE = 777
SEED_WALK = 4242


def _edge_params():
    """Hand-picked edge cases: equal masses (21-mode PN amplitude vanishes), extreme
    spins, swapped mass order (m1 < m2), near-maximal mass ratio."""
    base = draw_params(4, TOBS, SEED_PARAMS + 1)
    base[0, 0], base[1, 0] = 7.5e5, 7.5e5
    base[2, 1], base[3, 1] = 0.99, -0.99
    base[0, 2], base[1, 2] = 2e5, 9e5  # m1 < m2: driver swaps masses and spins
    base[0, 3], base[1, 3] = 3.0e6, 3.0e6 / 18.0
    return base


def phenomhm_case(params, length, run_phenomd=False, direct=False):
    wave = PhenomHMAmpPhase(run_phenomd=run_phenomd)
    m1, m2, c1, c2, dist, phi, fref = (params[k].copy() for k in range(7))
    t_ref = params[11].copy()
    if direct:
        freqs = np.logspace(-4, -1, length)
        wave(m1, m2, c1, c2, dist, np.zeros_like(phi), fref, t_ref, length, freqs=freqs,
             direct=True)
    else:
        tobs = np.full(len(m1), TOBS * YRSID_SI)
        wave(m1, m2, c1, c2, dist, np.zeros_like(phi), fref, t_ref, length, Tobs=tobs)
    return dict(freqs=wave.freqs_shaped.copy(), amp=wave.amp.copy(), phase=wave.phase.copy(),
                tf=wave.tf.copy(), fring=wave.fringdown.copy(), fdamp=wave.fdamp.copy())


def response_case(params, wf, tdi_tag="AET", tdi2=True, rescaled=False):
    orbits = EqualArmlengthOrbits()
    resp = LISATDIResponse(TDItag=tdi_tag, tdi2=tdi2, rescaled=rescaled, orbits=orbits)
    B, M, L = wf["amp"].shape
    buf = np.zeros((9, B, M, L))
    buf[0], buf[1], buf[2] = wf["amp"], wf["phase"], wf["tf"]
    buf = buf.ravel()
    resp(wf["freqs"].ravel(), params[7].copy(), params[8].copy(), params[9].copy(),
         params[10].copy(), params[5].copy(), L, out_buffer=buf, direct=True)
    return buf.reshape(9, B, M, L)


def spline_case(seed):
    rng = np.random.default_rng(seed)
    B, M, L, P = 2, 6, 64, 9
    x = np.sort(rng.uniform(1e-4, 1e-1, (B, M, L)), axis=-1)
    x = np.exp(np.cumsum(rng.uniform(0.01, 0.05, (B, M, L)), axis=-1)) * 1e-4
    y = np.sin(rng.uniform(0.5, 2.0, (P, B, M, 1)) * np.log(x)[None]) * rng.uniform(1, 5, (P, B, M, 1))
    spl = CubicSplineInterpolant(x, y)
    return dict(x=x, y=y, c1=spl.c1_shaped.copy(), c2=spl.c2_shaped.copy(),
                c3=spl.c3_shaped.copy())


def direct_like_case(params):
    orbits = EqualArmlengthOrbits()
    wave_gen = BBHWaveformFD(amp_phase_kwargs=dict(run_phenomd=False),
                             response_kwargs=dict(orbits=orbits, TDItag="AET", tdi2=True))
    f = data_grid(TOBS, F_LO, F_HI)
    df = f[1] - f[0]
    psd = np.array([aet_psd(f, c, tdi2=True) for c in "AET"])
    data = gaussian_noise(psd, df, SEED_NOISE)
    like = Likelihood(wave_gen, f, data, psd)
    kw = dict(length=1024, t_obs_start=0.0, t_obs_end=TOBS)
    ll = like.get_ll(params, **kw)
    tmpl, starts, lengths = wave_gen(*params, freqs=f, direct=False, fill=False, **kw)
    return dict(lnl=ll, d_h=like.d_h.copy(), h_h=like.h_h.copy(), d_d=np.array(like.d_d),
                start_inds=np.asarray(starts), lengths=np.asarray(lengths),
                template0_decim=tmpl[0][:, ::97].copy(),
                buffer0=wave_gen.out_buffer_final[:, :1].copy())


def fill_and_modes_case(params):
    """BBHWaveformFD branches beyond the likelihood's: fill=True combined into one [3, N]
    stream and one row per binary [B, 3, N] (waveformbuild.py:663-693), stored decimated
    (every 97th bin) together with exact per-row sums; direct=True, compress=False per-mode
    templates [B, 3, M, L] (waveformbuild.py:603-636) on a 128-point grid."""
    orbits = EqualArmlengthOrbits()
    wave_gen = BBHWaveformFD(amp_phase_kwargs=dict(run_phenomd=False),
                             response_kwargs=dict(orbits=orbits, TDItag="AET", tdi2=True))
    f = data_grid(TOBS, F_LO, F_HI)
    kw = dict(length=1024, t_obs_start=0.0, t_obs_end=TOBS)
    comb = wave_gen(*params, freqs=f, direct=False, fill=True, combine=True, **kw)
    each = wave_gen(*params, freqs=f, direct=False, fill=True, combine=False, **kw)
    fr = np.logspace(-4, -1.5, 128)
    modes = wave_gen(*params, freqs=fr, direct=True, compress=False, t_obs_start=0.0,
                     t_obs_end=TOBS)
    return dict(combine_decim=comb[:, ::97].copy(), combine_abs_sum=np.abs(comb).sum(axis=-1),
                each_decim=each[:, :, ::97].copy(), each_abs_sum=np.abs(each).sum(axis=-1),
                modes=np.asarray(modes).copy(), modes_freqs=fr)


def het_like_case(center, walkers):
    orbits = EqualArmlengthOrbits()
    wave_gen = BBHWaveformFD(amp_phase_kwargs=dict(run_phenomd=False),
                             response_kwargs=dict(orbits=orbits, TDItag="AET", tdi2=True))
    f = data_grid(TOBS, F_LO, F_HI)
    df = f[1] - f[0]
    psd = np.array([aet_psd(f, c, tdi2=True) for c in "AET"])
    data = gaussian_noise(psd, df, SEED_NOISE)
    from bbhx_b200.sensitivity import AET1SensitivityMatrix

    kw = dict(t_obs_start=0.0, t_obs_end=TOBS)
    het = HeterodynedLikelihood(wave_gen, f, data, center, 128,
                                template_gen_kwargs=dict(kw),
                                reference_gen_kwargs=dict(kw, length=1024),
                                sens_mat=AET1SensitivityMatrix(f, tdi2=True))
    ll = het.get_ll(walkers, **kw)
    return dict(lnl=ll, d_h=het.hdyn_d_h.copy(), h_h=het.hdyn_h_h.copy(),
                freqs=het.freqs.copy(), data_constants=het.data_constants.copy(),
                reference_d_d=np.array(het.reference_d_d), h0_sparse=het.h0_sparse.copy(),
                h_sparse=het.h_sparse.copy())


def main():
    out = {}
    P = draw_params(4, TOBS, SEED_PARAMS)
    E = _edge_params()
    out["params"] = P
    out["edge_params"] = E
    for tag, prm in (("main", P), ("edge", E)):
        wf = phenomhm_case(prm, 256)
        for k, v in wf.items():
            out[f"phm_{tag}_{k}"] = v
        out[f"resp_{tag}_aet2"] = response_case(prm, wf)
    wfd = phenomhm_case(P, 128, direct=True)
    for k, v in wfd.items():
        out[f"phm_direct_{k}"] = v
    wfpd = phenomhm_case(P, 128, run_phenomd=True)
    for k, v in wfpd.items():
        out[f"phd_{k}"] = v
    out["resp_direct_xyz"] = response_case(P, wfd, tdi_tag="XYZ", tdi2=False)
    out["resp_direct_aet1_rescaled"] = response_case(P, wfd, tdi2=False, rescaled=True)
    sp = spline_case(11)
    for k, v in sp.items():
        out[f"spl_{k}"] = v
    dl = direct_like_case(P)
    for k, v in dl.items():
        out[f"dl_{k}"] = v
    fm = fill_and_modes_case(P[:, :3])
    for k, v in fm.items():
        out[f"wf_{k}"] = v
    W = perturb_params(P[:, 0], 8, SEED_WALK)
    out["het_walkers"] = W
    hl = het_like_case(P[:, 0], W)
    for k, v in hl.items():
        out[f"het_{k}"] = v
    out["meta"] = np.array([TOBS, F_LO, F_HI, SEED_PARAMS, SEED_NOISE, SEED_WALK, MSUN_SI])
    path = os.path.join(HERE, "reference_golden.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path) / 1e6, "MB")
    for k in sorted(out):
        print(f"  {k:32s} {np.asarray(out[k]).shape}")


if __name__ == "__main__":
    main()
