"""CPU tests of the oracle: the numpy restatement (``oracle/kernels_np.py``) and the
restated driver (``oracle/pipeline.py``) pinned against the golden fixtures produced by the
reference's own code, plus the compiled reference (``oracle/_ref``) when it is present.

Tolerances: waveform / response / spline arrays |a - b| <= RTOL * max|b| per (binary,
mode) row; log-likelihoods |dlnL| <= 1e-6 + 1e-11 |lnL|.
"""
import os

import numpy as np
import pytest

from oracle import kernels_np as K
from oracle.pipeline import DEFAULT_MODES, RefPipeline

RTOL = 1e-11


def rowclose(a, b, rtol=RTOL):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (a.shape, b.shape)
    scale = np.max(np.abs(b), axis=-1, keepdims=True)
    scale = np.where(scale == 0, 1.0, scale)
    worst = float(np.nanmax(np.abs(a - b) / scale))
    assert np.all(np.isfinite(a) == np.isfinite(b))
    assert worst <= rtol, f"max row-relative error {worst:.3e} > {rtol:.1e}"
    return worst


def lnl_close(a, b):
    d = np.abs(np.asarray(a) - np.asarray(b))
    tol = 1e-6 + 1e-11 * np.abs(np.asarray(b))
    assert np.all(d <= tol), f"|dlnL| {d} vs tol {tol}"


@pytest.fixture(scope="module")
def np_pipe():
    return RefPipeline("np")


def _wave(pipe, prm, length, tobs=None, freqs=None):
    """The reference driver's two-pass PhenomHM evaluation (phenomhm.py:270-614)."""
    from bbhx_b200.utils.constants import YRSID_SI

    B = prm.shape[1]
    M = 1 if pipe.run_phenomd else len(DEFAULT_MODES)
    out = np.zeros(9 * B * M * length)
    args = (prm[0], prm[1], prm[2], prm[3], prm[4], prm[6], prm[11], length)
    f, ells, mms = pipe.run_wave(*args, freqs, list(DEFAULT_MODES), out)
    if tobs is not None:
        n = B * M * length
        newf = pipe.window(f.reshape(B, M, length), out[2 * n:3 * n].reshape(B, M, length),
                           np.full((B, M), tobs * YRSID_SI))
        out[:] = 0.0
        f, ells, mms = pipe.run_wave(*args, newf, list(DEFAULT_MODES), out)
    return f.reshape(B, M, length), out.reshape(9, B, M, length), ells, mms


@pytest.mark.parametrize("tag", ["main", "edge"])
def test_oracle_phenomhm_and_response_match_golden(golden, np_pipe, tag):
    prm = golden["params"] if tag == "main" else golden["edge_params"]
    f, out, ells, mms = _wave(np_pipe, prm, 256, tobs=float(golden["meta"][0]))
    rowclose(f, golden[f"phm_{tag}_freqs"])
    for k, name in enumerate(("amp", "phase", "tf")):
        rowclose(out[k], golden[f"phm_{tag}_{name}"], rtol=1e-12)
    B, M, L = f.shape
    buf = out.ravel()
    np_pipe.resp.LISA_response_wrap(buf, ells, mms, f.ravel(), prm[5], prm[7], prm[8], prm[9],
                                    prm[10], 2, 0, 1, 0, M, L, B, 1)
    ref = golden[f"resp_{tag}_aet2"]
    for k in range(1, 9):
        rowclose(buf.reshape(9, B, M, L)[k], ref[k], rtol=1e-12)


def test_oracle_direct_freqs_ringdown_phenomd(golden):
    prm = golden["params"]
    pipe = RefPipeline("np")
    f, out, _, _ = _wave(pipe, prm, 128, freqs=np.logspace(-4, -1, 128))
    for k, name in enumerate(("amp", "phase", "tf")):
        rowclose(out[k], golden[f"phm_direct_{name}"], rtol=1e-12)
    # ringdown tables: QNM fits per mode, PhenomD spline value appended per binary
    B = prm.shape[1]
    ells = np.array([l for l, m in DEFAULT_MODES], dtype=np.int32)
    mms = np.array([m for l, m in DEFAULT_MODES], dtype=np.int32)
    m1, m2, c1, c2 = prm[0].copy(), prm[1].copy(), prm[2].copy(), prm[3].copy()
    fr = np.zeros(B * 6)
    fd = np.zeros(B * 6)
    K.get_phenomhm_ringdown_frequencies(fr, fd, m1, m2, c1, c2, ells, mms, 6, B)
    gr = golden["phm_direct_fring"].reshape(B, 7)
    gd = golden["phm_direct_fdamp"].reshape(B, 7)
    np.testing.assert_allclose(fr.reshape(B, 6), gr[:, :6], rtol=1e-13)
    np.testing.assert_allclose(fd.reshape(B, 6), gd[:, :6], rtol=1e-13)
    pd = RefPipeline("np", run_phenomd=True)
    f, out, _, _ = _wave(pd, prm, 128, tobs=float(golden["meta"][0]))
    rowclose(f, golden["phd_freqs"])
    for k, name in enumerate(("amp", "phase", "tf")):
        rowclose(out[k], golden[f"phd_{name}"], rtol=1e-12)


def test_oracle_response_xyz_and_rescaled(golden, np_pipe):
    prm = golden["params"]
    B, M, L = golden["phm_direct_amp"].shape
    ells = np.array([l for l, m in DEFAULT_MODES], dtype=np.int32)
    mms = np.array([m for l, m in DEFAULT_MODES], dtype=np.int32)
    for tag, tdi, tdi2, resc in (("resp_direct_xyz", 1, 0, 0), ("resp_direct_aet1_rescaled", 2, 0, 1)):
        buf = np.zeros((9, B, M, L))
        buf[0], buf[1], buf[2] = (golden[f"phm_direct_{k}"] for k in ("amp", "phase", "tf"))
        buf = buf.ravel()
        np_pipe.resp.LISA_response_wrap(buf, ells, mms, golden["phm_direct_freqs"].ravel(), prm[5],
                                        prm[7], prm[8], prm[9], prm[10], tdi, resc, tdi2, 0, M, L, B, 1)
        for k in range(1, 9):
            rowclose(buf.reshape(9, B, M, L)[k], golden[tag][k], rtol=1e-12)


def test_oracle_spline(golden):
    x, y = golden["spl_x"], golden["spl_y"]
    P, B, M, L = y.shape
    Bv, c1, c2, c3 = (np.zeros(y.size) for _ in range(4))
    K.interpolate(x.ravel(), y.ravel(), Bv, c1, c2, c3, L, P, M, B)
    for name, arr in (("c1", c1), ("c2", c2), ("c3", c3)):
        rowclose(arr.reshape(P, B, M, L)[..., :-1], golden[f"spl_{name}"][..., :-1], rtol=1e-10)


def test_oracle_direct_likelihood(golden, golden_data, np_pipe):
    kw = dict(length=1024, t_obs_start=0.0, t_obs_end=golden_data["tobs"])
    ll, d_h, h_h, d_d = np_pipe.direct_lnl(golden["params"], golden_data["f"], golden_data["data"],
                                           golden_data["psd"], **kw)
    assert abs(d_d - float(golden["dl_d_d"])) <= 1e-12 * abs(float(golden["dl_d_d"]))
    lnl_close(ll, golden["dl_lnl"])
    np.testing.assert_allclose(h_h.real, golden["dl_h_h"].real, rtol=1e-11)


def test_oracle_hdyn_both_forms(golden):
    """hdyn on the golden sparse templates: the CPU form (one bin short) reproduces the
    golden sums; the GPU form adds exactly the last bin's contribution."""
    r = golden["het_h_sparse"] / golden["het_h0_sparse"]  # (B, 3, L)
    B, C, L = r.shape
    tm = np.ascontiguousarray(np.transpose(r, (2, 1, 0)))  # [L, C, B]
    consts = golden["het_data_constants"]
    f = golden["het_freqs"]
    dh_cpu, hh_cpu = np.zeros(B, complex), np.zeros(B, complex)
    K.hdyn(dh_cpu, hh_cpu, tm, consts, f, B, L, C, all_bins=False)
    np.testing.assert_allclose(dh_cpu, golden["het_d_h"], rtol=1e-10, atol=1e-8)
    np.testing.assert_allclose(hh_cpu.real, golden["het_h_h"].real, rtol=1e-11)
    dh_gpu, hh_gpu = np.zeros(B, complex), np.zeros(B, complex)
    K.hdyn(dh_gpu, hh_gpu, tm, consts, f, B, L, C, all_bins=True)
    Kc = consts.reshape(4, C, L)
    j = L - 1
    r1 = (r[:, :, j] - r[:, :, j - 1]) / (f[j] - f[j - 1])
    r0 = r[:, :, j] - r1 * (f[j] - 0.5 * (f[j] + f[j - 1]))
    np.testing.assert_allclose(dh_gpu - dh_cpu, (Kc[0, :, j] * np.conj(r0) + Kc[1, :, j] * np.conj(r1)).sum(1),
                               rtol=1e-9, atol=1e-9)


def test_oracle_detects_a_planted_fit_error(golden, monkeypatch):
    """A one-part-in-1e6 change of one inspiral phase-fit coefficient in the oracle must
    break the golden comparison (the comparison is sensitive at the tolerance used).  The
    coefficient is sigma2 (the Mf^(4/3) term): a change of a term linear in Mf, such as
    alpha1, is absorbed by the C1 phase connection and the t0 / phi0 alignment."""
    bad = list(K._FITS["sigma2"])
    bad[0] *= 1.0 + 1e-6
    monkeypatch.setitem(K._FITS, "sigma2", tuple(bad))
    f, out, _, _ = _wave(RefPipeline("np"), golden["params"], 128, freqs=np.logspace(-4, -1, 128))
    with pytest.raises(AssertionError):
        rowclose(out[1], golden["phm_direct_phase"], rtol=1e-12)


_REF_SO = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                       "libbbhx_ref.so")


@pytest.mark.skipif(not os.path.isfile(_REF_SO), reason="compiled reference (oracle/_ref) not built")
def test_compiled_reference_reproduces_golden_lnl(golden, golden_data):
    pipe = RefPipeline("ref")
    kw = dict(length=1024, t_obs_start=0.0, t_obs_end=golden_data["tobs"])
    ll, d_h, h_h, d_d = pipe.direct_lnl(golden["params"], golden_data["f"], golden_data["data"],
                                        golden_data["psd"], **kw)
    np.testing.assert_array_equal(ll, golden["dl_lnl"])
