"""Kernel-level GPU checks: the hot loop's sine / cosine, the phase recurrence's drift, and the
reproducibility of the queue-scheduled kernels."""
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


def test_phase_recurrence_drift_is_bounded():
    """The fused FP64 kernel's phase recurrence -- its own anchor and complex rotations, run by
    bbhx_selftest_recurrence -- against the exact phase of the cubic at the exact grid
    frequencies (mpmath, 50 digits), for phase cubics like a 1-yr stream's segments at 5e-2
    and 1e-3 Hz: the anchor is within 1e-12 and 128 steps of 32 bins (the kernel re-anchors
    every 128) stay within 4e-11, against ~2e-10 for a plain FP64 evaluation of a 1e6 rad phase."""
    import math

    import mpmath
    import torch

    from bbhx_b200 import _lib

    mpmath.mp.dps = 50
    df = 1.0 / 31558149.763545603
    lanes, steps = 32, 128
    tp = 2 * math.pi
    for k0, pc in [(1_500_000, (1.234567e6, tp * 2.0e7, tp * 3.0e9, tp * 1.0e11)),
                   (31_000, (2.0e5, tp * 3.0e7, tp * 4.0e10, tp * 5.0e13))]:
        xk = (k0 - 37) * df
        pcd = torch.tensor(pc, dtype=torch.float64, device="cuda")
        out = torch.empty(2 * lanes * steps, dtype=torch.float64, device="cuda")
        _lib.call("bbhx_selftest_recurrence", _lib.dptr(pcd), float(xk), float(k0), float(df),
                  lanes, steps, _lib.dptr(out), _lib.stream())
        e = out.cpu().numpy().reshape(lanes, steps, 2)
        y, c1, c2, c3 = (mpmath.mpf(v) for v in pc)
        err = np.zeros((lanes, steps))
        for lane in range(lanes):
            for j in range(steps):
                u = mpmath.mpf(k0 + lane + 32 * j) * mpmath.mpf(df) - mpmath.mpf(xk)
                ph = y + c1 * u + c2 * u ** 2 + c3 * u ** 3
                err[lane, j] = math.hypot(e[lane, j, 0] - float(mpmath.cos(ph)),
                                          e[lane, j, 1] - float(mpmath.sin(ph)))
        assert err[:, 0].max() < 1e-12, err[:, 0].max()
        assert err.max() < 4e-11, err.max()


def test_queue_scheduled_sums_are_bitwise_reproducible(golden, golden_data):
    """The fused kernels hand work items to warps from a queue counter, so which warp evaluates
    which (tile, binary) item changes from run to run; every item writes its own partial sums and
    the reduction adds them in a fixed order, so repeated evaluations agree bit for bit (direct
    FP64 and mixed, heterodyned FP64), here with 64x the golden binaries and 512x the golden
    walkers so that the items outnumber the resident warps."""
    from bbhx_b200 import AET1SensitivityMatrix, BBHWaveformFD, EqualArmlengthOrbits
    from bbhx_b200 import HeterodynedLikelihood, Likelihood

    wave = BBHWaveformFD(response_kwargs=dict(orbits=EqualArmlengthOrbits(), TDItag="AET",
                                              tdi2=True))
    f, tobs = golden_data["f"], golden_data["tobs"]
    kw = dict(t_obs_start=0.0, t_obs_end=tobs)
    params = np.tile(golden["params"], (1, 64))
    like = Likelihood(wave, f, golden_data["data"], golden_data["psd"])
    for precision in ("fp64", "mixed"):
        like.precision = precision
        runs = [like.get_ll(params, length=1024, **kw).copy() for _ in range(3)]
        for r in runs[1:]:
            assert np.array_equal(r, runs[0]), precision
    het = HeterodynedLikelihood(wave, f, golden_data["data"], golden["params"][:, 0], 128,
                                template_gen_kwargs=dict(kw), reference_gen_kwargs=dict(kw, length=1024),
                                sens_mat=AET1SensitivityMatrix(f, tdi2=True), precision="fp64")
    walkers = np.tile(golden["het_walkers"], (1, 512))
    runs = [het.get_ll(walkers, **kw).copy() for _ in range(3)]
    for r in runs[1:]:
        assert np.array_equal(r, runs[0])
