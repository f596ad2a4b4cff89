"""The drop-in boundary, end to end: BBHx's own drivers on this library's backend methods.

``tests/golden/dropin_trace.npz`` (made by ``tests/golden/make_dropin_trace.py``) holds every
call that the reference's unmodified ``Likelihood.get_ll`` and ``HeterodynedLikelihood``
(set-up + ``get_ll``) made into the nine backend methods (src/bbhx/cutils/__init__.py:13-23)
while running on the reference's compiled CPU code: 36 calls covering all nine methods and
``pyFastLISAResponse``, with their positional arguments as the drivers passed them and every
array after the call.  Here each call is replayed, in the recorded order, through
``bbhx_b200.backend.b200_methods()`` with the recorded inputs on the GPU (device arrays where
the reference's GPU backend gets cupy arrays, host arrays for the pointer arrays and
``direct_like``'s ``d_h`` / ``h_h``, device pointer arrays rebuilt from the recorded per-binary
buffers), and EVERY array argument is compared after the call with what the reference left in
it.  That is exactly what BBHx's drivers would see with this backend registered.

Tolerances: waveform / response / spline arrays within 1e-10 of each row's scale (the
reference's own ``1e-10`` waveform bar); templates within 1e-9 of each binary's scale; the
inner products <d|h>, <h|h> within 1e-6 + 1e-11 |x| (absolute 1e-6 at the |lnL| ~ 1e3-1e4 of
this workload); integer arrays exactly.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TRACE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "dropin_trace.npz")


def _get(d, key):
    v = d[key]
    if v.dtype.kind == "U":
        s = str(v)
        if s.startswith("ref:"):
            return _get(d, s[4:])
    return v


def _orbit_args():
    from bbhx_b200.orbits import EqualArmlengthOrbits

    return list(EqualArmlengthOrbits().pycppdetector_args)


def _digest(a):
    import hashlib

    a = np.ascontiguousarray(a)
    return hashlib.sha256(str(a.dtype).encode() + str(a.shape).encode() + a.tobytes()).hexdigest()


def _row_rel(got, ref, rows):
    """max |got - ref| / scale of each row (rows = number of equal-length rows)."""
    g = np.asarray(got).reshape(rows, -1)
    r = np.asarray(ref).reshape(rows, -1)
    scale = np.maximum(np.abs(r).max(axis=1, keepdims=True), 1e-300)
    return float(np.max(np.abs(g - r) / scale))


def _row_len(name, args):
    """Length of the rows (last axis) of the arrays a call works on, for row-relative checks."""
    return {"waveform_amp_phase_wrap": lambda: args[11],
            "pyFastLISAResponse.LISA_response_wrap": lambda: args[14],
            "interpolate_wrap": lambda: args[6],
            "direct_sum_wrap": lambda: args[3]}.get(name, lambda: 1)()


def _check(name, k, got, ref, call, row_len):
    """Compare one array argument after the call with the reference's."""
    got = np.asarray(got)
    ref = np.asarray(ref)
    assert got.shape == ref.shape and got.dtype == ref.dtype, (call, name, k)
    if ref.dtype.kind in "iu":
        np.testing.assert_array_equal(got, ref, err_msg=f"call {call} {name} arg {k}")
        return
    if name in ("direct_like_wrap", "hdyn_wrap") and k in (0, 1):
        tol = 1e-6 + 1e-11 * np.abs(ref)
        assert np.all(np.abs(got - ref) <= tol), (call, name, k, got, ref)
        return
    if ref.size == 0:
        return
    rows = ref.size // row_len if ref.size % row_len == 0 else 1
    if name == "interpolate_wrap" and k in (3, 4, 5):
        # c1, c2, c3 live in the tridiagonal solver's diagonals (Interpolate.cu:332-334); their
        # last entry of each row is never written as a coefficient and holds what the solver
        # left there (LAPACK dgtsv's LU factors on the reference's CPU backend, other values on
        # its GPU backend), and no spline evaluation reads it: compare the L - 1 segments
        got = got.reshape(rows, row_len)[:, :-1]
        ref = ref.reshape(rows, row_len)[:, :-1]
    tol = 1e-9 if name in ("direct_sum_wrap", "InterpTDI_wrap", "direct_like_wrap") else 1e-10
    err = _row_rel(got, ref, rows)
    assert err <= tol, f"call {call} {name} arg {k}: row-relative error {err:.2e} > {tol}"


def _hdyn_all_bins(d, i, ref_dh, ref_hh):
    """The reference's CPU hdynLikelihood stops one relative-binning bin short of its GPU kernel
    (Likelihood.cu:150 vs :57,75); this library follows the GPU kernel.  The recorded CPU
    results plus the last bin's term (numpy oracle, both forms on the recorded inputs) give the
    GPU-semantics values."""
    from oracle import kernels_np

    B, L, C = (int(d[f"c{i}_a{k}"]) for k in (5, 6, 7))
    r, K, f = (np.array(_get(d, f"c{i}_a{k}")) for k in (2, 3, 4))
    full = [np.zeros(B, np.complex128), np.zeros(B, np.complex128)]
    short = [np.zeros(B, np.complex128), np.zeros(B, np.complex128)]
    kernels_np.hdyn(full[0], full[1], r, K, f, B, L, C, all_bins=True)
    kernels_np.hdyn(short[0], short[1], r, K, f, B, L, C, all_bins=False)
    return ref_dh + (full[0] - short[0]), ref_hh + (full[1] - short[1])


def test_reference_driver_calls_replayed_through_b200_backend():
    import torch

    from bbhx_b200 import backend

    d = np.load(TRACE)
    meth = backend.b200_methods()
    n = int(d["ncalls"])
    orbit = None
    names_seen = set()
    for i in range(n):
        name = str(d[f"c{i}_name"])
        names_seen.add(name.split(".")[0])
        kinds = d[f"c{i}_kinds"]
        if name == "pyFastLISAResponse.add_orbit_information":
            args = _orbit_args()
            for k, kind in enumerate(kinds):
                if kind == 0:  # the regenerated table is the one the reference read
                    assert "sha256:" + _digest(np.asarray(args[k])) == str(d[f"c{i}_a{k}"]), k
                else:
                    assert float(args[k]) == float(d[f"c{i}_a{k}"]), k
            orbit = meth.pyFastLISAResponse()
            orbit.add_orbit_information(*args)
            continue
        if name == "pyFastLISAResponse.LISA_response_wrap":
            slots = backend._RESPONSE_SLOTS
            fn = orbit.LISA_response_wrap
        else:
            slots = backend._METHODS[name][1]
            fn = getattr(meth, name)
        ptr_slots = {"InterpTDI_wrap": {0: torch.complex128, 13: torch.int32},
                     "direct_like_wrap": {4: torch.complex128}}.get(name, {})
        args, per_binary = [], {}
        for k, kind in enumerate(kinds):
            key = f"c{i}_a{k}"
            if kind == 0 and k in ptr_slots:
                nb = int(d[key])
                bufs = [torch.from_numpy(np.array(_get(d, f"c{i}_p{k}_{b}"))).to("cuda")
                        for b in range(nb)]
                per_binary[k] = bufs
                args.append(np.array([t.data_ptr() for t in bufs], dtype=np.int64))
            elif kind == 0:
                arr = np.array(_get(d, key))
                args.append(torch.from_numpy(arr).to("cuda") if slots[k][0] == "D" else arr)
            elif kind == 1:
                args.append(int(d[key]))
            elif kind == 2:
                args.append(float(d[key]))
            else:
                args.append(bool(d[key]))
        fn(*args)
        torch.cuda.synchronize()
        for k, kind in enumerate(kinds):
            if kind != 0:
                continue
            if k in per_binary:
                for b, t in enumerate(per_binary[k]):
                    qk = f"c{i}_q{k}_{b}"
                    ref = _get(d, qk) if qk in d else _get(d, f"c{i}_p{k}_{b}")
                    got = t.cpu().numpy()
                    if ref.dtype.kind == "c" and ref.size:
                        scale = max(np.abs(ref).max(), 1e-300)
                        err = float(np.max(np.abs(got - ref)) / scale)
                        assert err <= 1e-9, f"call {i} {name} arg {k} binary {b}: {err:.2e}"
                    else:
                        np.testing.assert_array_equal(got, ref)
                continue
            ok = f"c{i}_o{k}"
            ref = _get(d, ok) if ok in d else _get(d, f"c{i}_a{k}")
            if name == "hdyn_wrap" and k in (0, 1):
                ref = _hdyn_all_bins(d, i, _get(d, f"c{i}_o0"), _get(d, f"c{i}_o1"))[k]
            a = args[k]
            got = a.cpu().numpy() if isinstance(a, torch.Tensor) else a
            _check(name, k, got, ref, i, _row_len(name, args))
    assert names_seen == set(backend.METHOD_NAMES), names_seen


def test_backend_refuses_host_memory_in_device_slots():
    """A numpy array where the C entry point reads device memory (and a CUDA tensor where it
    reads host memory) is refused before any launch."""
    import torch

    from bbhx_b200 import backend

    meth = backend.b200_methods()
    B, L = 2, 8
    with pytest.raises(TypeError, match="device memory"):
        meth.hdyn_wrap(np.zeros(B, np.complex128), torch.zeros(B, dtype=torch.complex128, device="cuda"),
                       torch.zeros(L * 3 * B, dtype=torch.complex128, device="cuda"),
                       torch.zeros(4 * 3 * L, dtype=torch.complex128, device="cuda"),
                       torch.zeros(L, dtype=torch.float64, device="cuda"), B, L, 3)
    with pytest.raises(TypeError, match="host memory"):
        meth.direct_like_wrap(torch.zeros(B, dtype=torch.complex128, device="cuda"),
                              np.zeros(B, np.complex128),
                              torch.zeros(3 * 16, dtype=torch.complex128, device="cuda"),
                              torch.zeros(3 * 16, dtype=torch.float64, device="cuda"),
                              np.zeros(B, np.int64), np.zeros(B, np.int32), np.zeros(B, np.int32),
                              16, B)
    with pytest.raises(TypeError, match="expected torch.float64"):
        meth.hdyn_wrap(*(torch.zeros(B, dtype=torch.complex128, device="cuda") for _ in range(4)),
                       torch.zeros(L, dtype=torch.float32, device="cuda"), B, L, 3)
