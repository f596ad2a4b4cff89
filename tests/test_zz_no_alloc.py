"""The allocation-free waveform entry point (bbhx_waveform_amp_phase_noalloc).

Some callers cannot allocate device memory: a host application whose own memory pool owns
the GPU, a latency-critical sampling loop that cannot afford cudaMalloc's device-wide
synchronisation, or a deployment without the stream-ordered allocator.  For them the library
offers a variant of the PhenomHM amplitude / phase / t(f) evaluation whose per-(binary, mode)
scratch records live in a static device array inside the library.  This test calls it through
the C ABI twice in a row (the second call reuses the array the first one left behind) and
checks each result against the regular, allocating entry point with the parity tolerance of
the other GPU tests, and that a batch above the array's capacity is refused with status 6.
Kept in its own file, named to be collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def _inputs(seed, B):
    import torch

    from bbhx_b200 import PhenomHMAmpPhase
    from bbhx_b200.synthetic import draw_params
    from bbhx_b200.utils.constants import MSUN_SI

    prm = draw_params(B, 0.1, seed)
    w = PhenomHMAmpPhase()
    # run the public path once to get the default grid and the [B, M+1] ringdown table
    w.run_wave(prm[0], prm[1], prm[2], prm[3], prm[4], np.zeros(B), prm[6], prm[11], 256)
    m1, m2 = w._m1, w._m2
    d = dict(ells=w.ells, mms=w.mms, freqs=w.freqs.clone(), m1_SI=(m1 * MSUN_SI).contiguous(),
             m2_SI=(m2 * MSUN_SI).contiguous(),
             chi1z=torch.as_tensor(np.where(prm[0] < prm[1], prm[3], prm[2]), device="cuda"),
             chi2z=torch.as_tensor(np.where(prm[0] < prm[1], prm[2], prm[3]), device="cuda"),
             dist=torch.as_tensor(prm[4], device="cuda"), f_ref=torch.zeros(B, dtype=torch.float64, device="cuda"),
             fring=w.fringdown.clone(), fdamp=w.fdamp.clone(), M=w.num_modes, L=256, B=B)
    return d


def _call(name, d, out):
    from bbhx_b200 import _lib

    return getattr(_lib.lib(), name)(
        _lib.dptr(out), _lib.dptr(d["ells"]), _lib.dptr(d["mms"]), _lib.dptr(d["freqs"]),
        _lib.dptr(d["m1_SI"]), _lib.dptr(d["m2_SI"]), _lib.dptr(d["chi1z"]), _lib.dptr(d["chi2z"]),
        _lib.dptr(d["dist"]), _lib.dptr(d["f_ref"]), d["M"], d["L"], d["B"], _lib.dptr(d["fring"]),
        _lib.dptr(d["fdamp"]), 0, _lib.stream())


def _rowclose(a, b):
    scale = np.abs(b).max(axis=-1, keepdims=True)
    scale = np.where(scale == 0, 1.0, scale)
    err = float((np.abs(a - b) / scale).max())
    assert err <= RTOL, err


def test_noalloc_matches_allocating_entry_point_twice():
    import torch

    for seed, B in ((101, 64), (202, 48)):
        d = _inputs(seed, B)
        n = 3 * B * d["M"] * d["L"]
        ref = torch.zeros(n, dtype=torch.float64, device="cuda")
        got = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
        assert _call("bbhx_waveform_amp_phase", d, ref) == 0
        assert _call("bbhx_waveform_amp_phase_noalloc", d, got) == 0
        torch.cuda.synchronize()
        a = got.cpu().numpy().reshape(3, B * d["M"], d["L"])
        b = ref.cpu().numpy().reshape(3, B * d["M"], d["L"])
        assert np.all(np.isfinite(a))
        for k in range(3):
            _rowclose(a[k], b[k])


def test_noalloc_rejects_batches_above_capacity():
    import torch

    from bbhx_b200 import _lib

    d = _inputs(7, 4)
    d = dict(d, B=8192 // d["M"] + 1)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = _call("bbhx_waveform_amp_phase_noalloc", d, out)
    assert st == 6
    msg = _lib.lib().bbhx_last_error_string().decode()
    assert "exceeds the static scratch capacity" in msg
