"""Edge cases through the C ABI and the public API.

* empty batches (B = 0) are no-ops that return status 0 and leave the outputs untouched;
* argument errors come back as status codes with a message (the library never exits) and
  surface in Python as ValueError, like the reference's own checks;
* a binary at the bottom edge of the band (5e8 Msun: a support of a few bins) against the
  reference's compiled CPU lnL (numpy oracle when the compiled reference is absent);
* a binary the reference rejects (4e9 Msun: the window search past the observation fails)
  raises the reference's ValueError, and so do |chi| > 1 and unknown modes.
"""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _wave():
    from bbhx_b200 import BBHWaveformFD, EqualArmlengthOrbits

    return BBHWaveformFD(amp_phase_kwargs=dict(run_phenomd=False),
                         response_kwargs=dict(orbits=EqualArmlengthOrbits(), TDItag="AET", tdi2=True))


def _raw(name):
    from bbhx_b200 import _lib

    return getattr(_lib.lib(), name)


def test_empty_batches_are_no_ops():
    import torch

    from bbhx_b200 import _lib

    s = _lib.stream()
    out = torch.full((8,), 7.0, dtype=torch.float64, device="cuda")
    p = _lib.dptr(out)
    z = _lib._VP(0)
    # fused direct likelihood, spline, PhenomHM amplitude / phase, response: B = 0
    assert _raw("bbhx_direct_like_fused")(p, p, p, p, p, 16, p, p, p, p, p, p, p, 6, 1024, 0, 1,
                                          z, z, s) == 0
    assert _raw("bbhx_interpolate")(p, p, p, p, p, p, 1024, 9, 6, 0, s) == 0
    ells = torch.tensor([2, 3, 4, 2, 3, 4], dtype=torch.int32, device="cuda")
    mms = torch.tensor([2, 3, 4, 1, 2, 3], dtype=torch.int32, device="cuda")
    e, m = _lib.dptr(ells), _lib.dptr(mms)
    assert _raw("bbhx_waveform_amp_phase")(p, e, m, p, p, p, p, p, p, p, 6, 1024, 0, p, p, 0,
                                           s) == 0
    assert _raw("bbhx_hdyn")(p, p, p, p, p, 0, 128, 3, s) == 0
    torch.cuda.synchronize()
    assert torch.all(out == 7.0)


def test_argument_errors_are_status_codes():
    import torch

    from bbhx_b200 import _lib

    s = _lib.stream()
    buf = torch.zeros(64, dtype=torch.float64, device="cuda")
    p = _lib.dptr(buf)
    z = _lib._VP(0)
    f = _raw("bbhx_direct_like_fused")
    assert f(p, p, p, p, p, 16, p, p, p, p, p, p, p, 6, 1024, 4, 2, z, z, s) == 1
    assert b"precision" in _lib.lib().bbhx_last_error_string()
    assert f(p, p, p, p, p, 16, p, p, p, p, p, p, p, 7, 1024, 4, 0, z, z, s) == 1
    assert f(p, p, p, p, p, 16, p, p, p, p, p, p, p, 6, 1024, 4, 1, p, z, s) == 1
    assert b"data32" in _lib.lib().bbhx_last_error_string()
    assert _raw("bbhx_interpolate")(p, p, p, p, p, p, 2, 9, 6, 1, s) == 1
    with pytest.raises(ValueError, match="not-a-knot"):
        _lib.call("bbhx_interpolate", p, p, p, p, p, p, 2, 9, 6, 1, s)
    # the heterodyne entry without orbit tables
    st = _raw("bbhx_hdyn_fused")(z, p, p, p, p, p, p, p, p, p, p, p, ctypes.c_double(0.0), p, p,
                                  p, p, p, 2, 0, 1, 6, 128, 4, 0, s)
    assert st != 0 and b"orbit" in _lib.lib().bbhx_last_error_string()
    torch.cuda.synchronize()  # the context is still usable
    assert float(buf.sum().item()) == 0.0


def _golden_like(golden_data):
    from bbhx_b200 import Likelihood

    return Likelihood(_wave(), golden_data["f"], golden_data["data"], golden_data["psd"])


def test_band_edge_binary_matches_reference(golden, golden_data):
    """5e8 Msun: the template covers only the lowest few bins of the 0.1-50 mHz band."""
    from oracle.build_ref import OUT
    from oracle.pipeline import RefPipeline

    P = golden["params"][:, :1].copy()
    P[0, 0], P[1, 0] = 4e8, 1e8
    kw = dict(length=1024, t_obs_start=0.0, t_obs_end=golden_data["tobs"])
    like = _golden_like(golden_data)
    ll = like.get_ll(P, **kw)
    hh = float(like.h_h.real.cpu().numpy()[0])
    pipe = RefPipeline("ref" if os.path.isfile(OUT) else "np")
    ref, _, ref_hh, _ = pipe.direct_lnl(P, golden_data["f"], golden_data["data"], golden_data["psd"],
                                        **kw)
    print(pipe.K.name, ll, ref, hh, ref_hh)
    assert 0.0 < hh < 1.0  # a few bins of support: nearly silent
    np.testing.assert_allclose(hh, ref_hh.real[0], rtol=1e-9, atol=1e-12)
    assert abs(ll[0] - ref[0]) <= 1e-6 + 1e-11 * abs(ref[0])


def test_reference_rejections_raise_the_same_errors(golden, golden_data):
    kw = dict(length=1024, t_obs_start=0.0, t_obs_end=golden_data["tobs"])
    like = _golden_like(golden_data)
    P = golden["params"][:, :1].copy()
    heavy = P.copy()
    heavy[0, 0], heavy[1, 0] = 3.2e9, 0.8e9
    with pytest.raises(ValueError, match="window at x_max did not run correctly"):
        like.get_ll(heavy, **kw)
    spin = P.copy()
    spin[2, 0] = 1.2
    with pytest.raises(ValueError, match="chi1z"):
        like.get_ll(spin, **kw)
    with pytest.raises(ValueError, match="not available"):
        like.get_ll(P, modes=[(5, 5)], **kw)
    # still usable afterwards
    ll = like.get_ll(P, **kw)
    assert np.all(np.isfinite(ll))


def test_nonfinite_output_is_status_4():
    """A NaN in the inputs of the relative-binning sums makes that walker's <d|h>, <h|h> NaN:
    the stream-ordered call returns 0, bbhx_take_status reports 4 once and clears the record,
    and finite inputs leave it at 0."""
    import torch

    from bbhx_b200 import _lib

    s = _lib.stream()
    take = _raw("bbhx_take_status")
    take(s)  # clear whatever earlier calls in this process recorded
    B, L = 3, 16
    r = torch.ones((L, 3, B), dtype=torch.complex128, device="cuda")
    consts = torch.ones((4, 3, L), dtype=torch.complex128, device="cuda")
    f = torch.linspace(1e-3, 2e-3, L, dtype=torch.float64, device="cuda")
    d_h = torch.zeros(B, dtype=torch.complex128, device="cuda")
    h_h = torch.zeros(B, dtype=torch.complex128, device="cuda")
    args = lambda: (_lib.dptr(d_h), _lib.dptr(h_h), _lib.dptr(r), _lib.dptr(consts),
                    _lib.dptr(f), B, L, 3, s)
    assert _raw("bbhx_hdyn")(*args()) == 0
    assert take(s) == 0
    r[5, 1, 2] = complex(float("nan"), 0.0)
    assert _raw("bbhx_hdyn")(*args()) == 0
    assert take(s) == 4
    assert b"not finite" in _lib.lib().bbhx_last_error_string()
    assert torch.isnan(d_h[2].real) and torch.isfinite(d_h[0].real)
    assert take(s) == 0  # the record was cleared
