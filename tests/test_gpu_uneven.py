"""Uneven batch: direct groups with different data streams (observation spans), grid lengths and
mode sets, and heterodyned groups with different sparse grids: the direct groups' sparse grids
and splines built in one launch from their parameters, then every direct tile and heterodyned
walker evaluated in one persistent launch, autotuned, captured in a CUDA graph.

Checks: FP64 batch == per-group Likelihood.get_ll to 1e-9 relative (same arithmetic, different
summation order of the tiles); mixed batch vs FP64 |dlnL| <= 2e-6 <h|h>; graph replay with new
parameters == an eager run with them; heterodyned groups == HeterodynedLikelihood.get_ll; a
coarse grid over a 1-yr stream (L = 256: ~1.2e4 data bins per knot interval) in a mixed batch
is routed to FP64 and meets |dlnL| <= 1e-2, while a fine one (L = 2048) stays mixed.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(golden, golden_data):
    from bbhx_b200 import (AET1SensitivityMatrix, BBHWaveformFD, EqualArmlengthOrbits,
                           HeterodynedLikelihood, Likelihood)
    from bbhx_b200.sensitivity import aet_psd
    from bbhx_b200.synthetic import data_grid, draw_params, gaussian_noise, perturb_params

    def wave():
        return BBHWaveformFD(amp_phase_kwargs=dict(run_phenomd=False),
                             response_kwargs=dict(orbits=EqualArmlengthOrbits(), TDItag="AET", tdi2=True))

    like_a = Likelihood(wave(), golden_data["f"], golden_data["data"], golden_data["psd"])
    tobs_b = 0.05
    fb = data_grid(tobs_b, 1e-4, 5e-2)
    psd_b = np.array([aet_psd(fb, c, tdi2=True) for c in "AET"])
    like_b = Likelihood(wave(), fb, gaussian_noise(psd_b, fb[1] - fb[0], 5), psd_b)
    P = golden["params"]
    Pb = draw_params(2, tobs_b, 99)
    direct = [
        dict(like=like_a, params=P[:, :3], length=256, modes=[(2, 2)], tobs=golden_data["tobs"]),
        dict(like=like_a, params=P[:, 1:3], length=1024, modes=None, tobs=golden_data["tobs"]),
        dict(like=like_b, params=Pb, length=512, modes=None, tobs=tobs_b),
    ]
    kw = dict(t_obs_start=0.0, t_obs_end=golden_data["tobs"])
    het = HeterodynedLikelihood(wave(), golden_data["f"], golden_data["data"], P[:, 0], 64,
                                template_gen_kwargs=dict(kw), reference_gen_kwargs=dict(kw, length=1024),
                                sens_mat=AET1SensitivityMatrix(golden_data["f"], tdi2=True))
    walkers = perturb_params(P[:, 0], 5, 3)
    # a second heterodyned problem: another reference point, a 96-point sparse grid
    het2 = HeterodynedLikelihood(wave(), golden_data["f"], golden_data["data"], P[:, 2], 96,
                                 template_gen_kwargs=dict(kw), reference_gen_kwargs=dict(kw, length=1024),
                                 sens_mat=AET1SensitivityMatrix(golden_data["f"], tdi2=True))
    walkers2 = perturb_params(P[:, 2], 7, 5)
    return direct, [(het, walkers), (het2, walkers2)], kw


def _batch(direct, hets, kw, precision):
    from bbhx_b200.uneven import DirectGroup, HetGroup, UnevenBatch

    dg = [DirectGroup(d["like"], d["params"], length=d["length"], modes=d["modes"], t_obs_start=0.0,
                      t_obs_end=d["tobs"]) for d in direct]
    hg = [HetGroup(h, w, **kw) for h, w in hets]
    return UnevenBatch(dg, hg, precision=precision)


def test_uneven_fp64_matches_per_group(golden, golden_data):
    direct, hets, kw = _problem(golden, golden_data)
    batch = _batch(direct, hets, kw, "fp64")
    out = [o.cpu().numpy() for o in batch.run()]
    shapes = [(t, c) for t in batch.autotuner.TILES for c in batch.autotuner.CTAS]
    assert batch.shape and all(sh in shapes for sh in batch.shape.values())
    for d, got in zip(direct, out):
        ref = d["like"].get_ll(d["params"], length=d["length"], modes=d["modes"], t_obs_start=0.0,
                               t_obs_end=d["tobs"])
        np.testing.assert_allclose(got, ref, rtol=1e-9, atol=1e-6)
    # the walkers inside the persistent launch == the single-problem heterodyne kernel
    for (het, walkers), got in zip(hets, out[len(direct):]):
        het.precision = "fp64"
        np.testing.assert_allclose(got, het.get_ll(walkers, **kw), rtol=1e-12, atol=1e-8)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_uneven_heterodyned_only(golden, golden_data, precision):
    """A batch of heterodyned problems alone (two sparse grids) in one launch equals each
    problem's own fused evaluation in the same precision: to 1e-12 in FP64; in the mixed form
    the FP32 parts are compiled into two different kernels, so the two evaluations agree to the
    mixed form's own accuracy (2e-6 relative, as mixed against FP64 elsewhere)."""
    from bbhx_b200.uneven import HetGroup, UnevenBatch

    _, hets, kw = _problem(golden, golden_data)
    batch = UnevenBatch([], [HetGroup(h, w, **kw) for h, w in hets], precision=precision,
                        shape={precision: (4096, 3)})
    out = [o.cpu().numpy() for o in batch.run()]
    rtol = 1e-12 if precision == "fp64" else 2e-6
    for (het, walkers), got in zip(hets, out):
        het.precision = precision
        np.testing.assert_allclose(got, het.get_ll(walkers, **kw), rtol=rtol, atol=1e-8)


def test_uneven_mixed_error_and_graph_replay(golden, golden_data):
    direct, hets, kw = _problem(golden, golden_data)
    b64 = _batch(direct, hets, kw, "fp64")
    ref = [o.cpu().numpy() for o in b64.run()]
    hh = [g.h_h.real.cpu().numpy() for g in b64.direct]
    bm = _batch(direct, hets, kw, "mixed")
    out = [o.clone() for o in bm.capture()]
    for k, (a, r) in enumerate(zip(out, ref)):
        scale = hh[k] if k < len(hh) else np.abs(r)
        assert np.all(np.abs(a.cpu().numpy() - r) <= 2e-6 * np.maximum(scale, 1.0)), k
    # replay with new parameters for group 1 == an eager mixed run with them
    from bbhx_b200.synthetic import perturb_params

    newp = perturb_params(direct[1]["params"][:, 0], direct[1]["params"].shape[1], 8)
    bm.set_params(1, newp)
    rep = [o.cpu().numpy().copy() for o in bm.replay()]
    direct[1]["params"] = newp
    eager = _batch(direct, hets, kw, "mixed")
    eager.shape = dict(bm.shape)
    ev = [o.cpu().numpy() for o in eager.run()]
    for a, b in zip(rep, ev):
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-9)
    assert all(int(f.abs().sum().item()) == 0 for f in bm.flags())


def test_uneven_mixed_routes_coarse_grids_to_fp64():
    from bbhx_b200 import BBHWaveformFD, EqualArmlengthOrbits, Likelihood
    from bbhx_b200.sensitivity import aet_psd
    from bbhx_b200.synthetic import data_grid, draw_params, gaussian_noise, notch_tdi_zeros
    from bbhx_b200.uneven import DirectGroup, UnevenBatch
    from bbhx_b200.utils.constants import YRSID_SI

    tobs = 1.0
    f = data_grid(tobs, 1e-5, 0.1)
    psd = notch_tdi_zeros(f, np.array([aet_psd(f, c, tdi2=True) for c in "AET"]))
    wave = BBHWaveformFD(response_kwargs=dict(orbits=EqualArmlengthOrbits(), TDItag="AET", tdi2=True))
    like = Likelihood(wave, f, gaussian_noise(psd, f[1] - f[0], 21), psd)
    P = draw_params(6, tobs, 77)
    P[11] = np.random.default_rng(77).uniform(0.8, 0.95, 6) * tobs * YRSID_SI
    groups = [dict(length=256, params=P[:, :3]), dict(length=2048, params=P[:, 3:])]
    batch = UnevenBatch([DirectGroup(like, g["params"], length=g["length"], t_obs_start=0.0,
                                     t_obs_end=tobs) for g in groups], precision="mixed")
    assert batch.group_precisions() == ["fp64", "mixed"]
    out = [o.cpu().numpy() for o in batch.run()]
    for g, got in zip(groups, out):
        like.precision = "fp64"
        ref = like.get_ll(g["params"], length=g["length"], t_obs_start=0.0, t_obs_end=tobs)
        hh = like.h_h.real.cpu().numpy()
        err = np.abs(got - ref)
        if g["length"] == 256:
            # FP64 on both sides; the phase recurrences re-anchor at different bins, and a
            # recurrence phase error (<= 4e-11 rad, the drift self-test) moves the modes'
            # cross terms of h_h by up to that fraction
            assert np.all(err <= 1e-6 + 4e-11 * hh), (err, hh)
        else:
            assert np.all(err <= 2e-6 * np.maximum(hh, 1.0)), err


def test_prebuilt_spline_entry_point_matches_the_batch(golden, golden_data):
    """bbhx_direct_like_multi fed the sparse grids and splines that bbhx_uneven_batch built in
    its fused build launch gives the batch's own direct lnL (FP64)."""
    import ctypes

    from bbhx_b200 import _lib
    from bbhx_b200.uneven import DirectGroupC

    direct, _, kw = _problem(golden, golden_data)
    batch = _batch(direct, [], kw, "fp64")
    batch.shape = {"fp64": (4096, 3)}
    out = [o.cpu().numpy().copy() for o in batch.run()]
    descs = []
    for g in batch.direct:
        x, y, c1, c2, c3, ts, te = g._keep[:7]
        lk = g.like
        p = lambda a: _lib.dptr(a).value  # noqa: E731
        descs.append(DirectGroupC(p(lk.data_freqs), p(lk.data_channels), p(lk.noise_factors),
                                  int(lk.data_freqs.numel()), p(x), p(y), p(c1), p(c2), p(c3),
                                  p(ts), p(te), g.M, g.L, g.size, p(g.d_h), p(g.h_h), None, None))
    arr = (DirectGroupC * len(descs))(*descs)
    _lib.call("bbhx_direct_like_multi", ctypes.cast(arr, ctypes.c_void_p), len(descs), 0, 4096, 3,
              _lib.stream())
    for g, ref in zip(batch.direct, out):
        np.testing.assert_allclose(g.lnl().cpu().numpy(), ref, rtol=1e-12, atol=1e-9)


def test_builder_covers_phenomd_xyz_and_rescaled_groups(golden, golden_data):
    """The fused sparse build handles every waveform / response switch of the single-problem
    path: a PhenomD-only group (the tabulated 22 ringdown, one mode), an XYZ group and a
    rescaled-AET group, each equal to its own Likelihood.get_ll (FP64)."""
    from bbhx_b200 import BBHWaveformFD, EqualArmlengthOrbits, Likelihood
    from bbhx_b200.uneven import DirectGroup, UnevenBatch

    f, data, psd, tobs = golden_data["f"], golden_data["data"], golden_data["psd"], golden_data["tobs"]
    P = golden["params"]
    waves = [BBHWaveformFD(amp_phase_kwargs=dict(run_phenomd=True),
                           response_kwargs=dict(orbits=EqualArmlengthOrbits(), TDItag="AET", tdi2=True)),
             BBHWaveformFD(response_kwargs=dict(orbits=EqualArmlengthOrbits(), TDItag="XYZ")),
             BBHWaveformFD(response_kwargs=dict(orbits=EqualArmlengthOrbits(), TDItag="AET",
                                                rescaled=True))]
    likes = [Likelihood(w, f, data, psd) for w in waves]
    groups = [DirectGroup(lk, P, length=512, t_obs_start=0.0, t_obs_end=tobs) for lk in likes]
    batch = UnevenBatch(groups, precision="fp64", shape={"fp64": (4096, 3)})
    out = [o.cpu().numpy() for o in batch.run()]
    for lk, got in zip(likes, out):
        ref = lk.get_ll(P, length=512, t_obs_start=0.0, t_obs_end=tobs)
        np.testing.assert_allclose(got, ref, rtol=1e-9, atol=1e-6)
    assert all(int(fl.abs().sum().item()) == 0 for fl in batch.flags())
