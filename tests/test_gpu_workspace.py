"""Caller-provided workspace (bbhx_workspace_set): the entry points take their scratch from a
buffer the caller owns; results are the same as with the stream-ordered pool, a buffer that is
too small makes the call fail with status 2 (and reports the size it needed), and the library
works normally once the workspace is released."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _like(golden_data):
    from bbhx_b200 import BBHWaveformFD, EqualArmlengthOrbits, Likelihood

    wave = BBHWaveformFD(response_kwargs=dict(orbits=EqualArmlengthOrbits(), TDItag="AET", tdi2=True))
    return Likelihood(wave, golden_data["f"], golden_data["data"], golden_data["psd"])


def test_direct_lnl_and_gradient_in_a_workspace(golden, golden_data):
    import bbhx_b200.workspace as ws

    like = _like(golden_data)
    P = golden["params"]
    kw = dict(length=1024, t_obs_start=0.0, t_obs_end=golden_data["tobs"])
    ref = like.get_ll(P, **kw)
    g_ref = like.get_ll_and_grad(P, **kw)[1].cpu().numpy()
    with ws.workspace(256 << 20):
        got = like.get_ll(P, **kw)
        g = like.get_ll_and_grad(P, **kw)[1].cpu().numpy()
        need = ws.peak()
    assert need > 0
    np.testing.assert_array_equal(got, ref)
    np.testing.assert_array_equal(g, g_ref)


def test_too_small_workspace_fails_cleanly(golden, golden_data):
    import bbhx_b200.workspace as ws
    from bbhx_b200._lib import BBHxCudaError

    like = _like(golden_data)
    P = golden["params"]
    kw = dict(length=1024, t_obs_start=0.0, t_obs_end=golden_data["tobs"])
    ref = like.get_ll(P, **kw)
    with ws.workspace(4096):
        with pytest.raises(BBHxCudaError):
            like.get_ll(P, **kw)
        assert ws.peak() > 4096
    np.testing.assert_array_equal(like.get_ll(P, **kw), ref)
