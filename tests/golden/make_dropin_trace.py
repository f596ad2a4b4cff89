"""Record the backend calls that the REFERENCE drivers make, for the drop-in replay test.

The reference's own Python classes (``bbhx.likelihood.Likelihood`` /
``HeterodynedLikelihood``, which drive ``BBHWaveformFD``, ``PhenomHMAmpPhase``,
``LISATDIResponse``, ``CubicSplineInterpolant`` and ``TemplateInterpFD``) run unmodified on the
reference's C++ compiled for CPU (``oracle/_ref/libbbhx_ref.so``, with ``oracle/refenv``
standing in for gpubackendtools / lisatools).  Every call they make into the nine backend methods
(src/bbhx/cutils/__init__.py:13-23) is intercepted: its name, its positional arguments as passed
(arrays copied before the call) and the arrays after the call are stored in
``tests/golden/dropin_trace.npz``.  For the pointer arrays of ``InterpTDI_wrap`` and
``direct_like_wrap`` the pointed-to per-binary templates / index arrays are stored instead of
the addresses.  ``tests/test_gpu_dropin.py`` replays the calls through
``bbhx_b200.backend.b200_methods()`` and compares the outputs.

Runs only where the reference checkout exists.  Usage: python tests/golden/make_dropin_trace.py
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, REPO)
from oracle.build_ref import REF_ROOT  # noqa: E402

sys.path.insert(0, os.path.join(REPO, "oracle", "refenv"))
sys.path.insert(0, os.path.join(REF_ROOT, "src"))

from oracle.build_ref import build as build_ref  # noqa: E402

build_ref()

import warnings  # noqa: E402

warnings.filterwarnings("ignore")
import bbhx_backend_cpu.interp as _interp  # noqa: E402
import bbhx_backend_cpu.likelihood as _like  # noqa: E402
import bbhx_backend_cpu.phenomhm as _phm  # noqa: E402
import bbhx_backend_cpu.response as _resp  # noqa: E402
import bbhx_backend_cpu.waveformbuild as _wb  # noqa: E402

TOBS = 0.01  # years
F_LO, F_HI = 2e-3, 8e-3
SEED_PARAMS = 20261204
SEED_NOISE = 4711
SEED_WALK = 99
LENGTH = 128
LENGTH_HET = 32

CALLS = []


def _deref(addr, dtype, count):
    """Copy of ``count`` elements of ``dtype`` at host address ``addr``."""
    nbytes = np.dtype(dtype).itemsize * int(count)
    buf = (ctypes.c_char * nbytes).from_address(int(addr))
    return np.frombuffer(bytes(buf), dtype=dtype).copy()


def _pointer_targets(name, args):
    """{arg index: (dtype, per-binary element counts)} of the host pointer arrays."""
    if name == "InterpTDI_wrap":
        lengths = np.asarray(args[15])
        M = int(args[12])
        return {0: (np.complex128, 3 * lengths), 13: (np.int32, M * lengths)}
    if name == "direct_like_wrap":
        return {4: (np.complex128, 3 * np.asarray(args[6]))}
    return {}


def _digest(a):
    import hashlib

    a = np.ascontiguousarray(a)
    return hashlib.sha256(str(a.dtype).encode() + str(a.shape).encode() + a.tobytes()).hexdigest()


def _record(name, fn):
    def wrapped(*args):
        rec = {"name": name, "args": [], "ptr_before": {}, "ptr_after": {}, "after": {}}
        targets = _pointer_targets(name, args)
        for k, a in enumerate(args):
            if isinstance(a, np.ndarray):
                rec["args"].append(("arr", a.copy()))
            elif isinstance(a, (bool, np.bool_)):
                rec["args"].append(("bool", bool(a)))
            elif isinstance(a, (int, np.integer)):
                rec["args"].append(("int", int(a)))
            elif isinstance(a, (float, np.floating)):
                rec["args"].append(("float", float(a)))
            else:
                raise TypeError(f"{name}: argument {k} of type {type(a)}")
        for k, (dt, counts) in targets.items():
            rec["ptr_before"][k] = [_deref(p, dt, c) for p, c in zip(np.asarray(args[k]), counts)]
        fn(*args)
        for k, a in enumerate(args):
            if isinstance(a, np.ndarray):
                rec["after"][k] = a.copy()
        for k, (dt, counts) in targets.items():
            rec["ptr_after"][k] = [_deref(p, dt, c) for p, c in zip(np.asarray(args[k]), counts)]
        CALLS.append(rec)

    wrapped.__name__ = name
    return wrapped


def _install():
    for mod, names in ((_phm, ["waveform_amp_phase_wrap", "get_phenomhm_ringdown_frequencies",
                               "get_phenomd_ringdown_frequencies"]),
                       (_interp, ["interpolate_wrap"]),
                       (_wb, ["InterpTDI_wrap", "direct_sum_wrap"]),
                       (_like, ["direct_like_wrap", "hdyn_wrap"])):
        for n in names:
            setattr(mod, n, _record(n, getattr(mod, n)))
    cls = _resp.pyFastLISAResponse
    for n in ("add_orbit_information", "LISA_response_wrap"):
        orig = getattr(cls, n)

        def bound(self, *args, _orig=orig, _n=n):
            return _record("pyFastLISAResponse." + _n, lambda *a: _orig(self, *a))(*args)

        setattr(cls, n, bound)


def main():
    _install()
    from bbhx.likelihood import HeterodynedLikelihood, Likelihood
    from bbhx.waveformbuild import BBHWaveformFD
    from lisatools.detector import EqualArmlengthOrbits

    from bbhx_b200.sensitivity import AET1SensitivityMatrix, aet_psd
    from bbhx_b200.synthetic import data_grid, draw_params, gaussian_noise, perturb_params

    f = data_grid(TOBS, F_LO, F_HI)
    psd = np.array([aet_psd(f, c, tdi2=True) for c in "AET"])
    data = gaussian_noise(psd, f[1] - f[0], SEED_NOISE)
    P = draw_params(2, TOBS, SEED_PARAMS)
    wave = BBHWaveformFD(response_kwargs=dict(orbits=EqualArmlengthOrbits(), TDItag="AET", tdi2=True))
    kw = dict(t_obs_start=0.0, t_obs_end=TOBS)
    like = Likelihood(wave, f, data, psd)
    ll = like.get_ll(P, length=LENGTH, **kw)
    W = perturb_params(P[:, 0], 3, SEED_WALK)
    het = HeterodynedLikelihood(wave, f, data, P[:, 0], LENGTH_HET, template_gen_kwargs=dict(kw),
                                reference_gen_kwargs=dict(kw, length=LENGTH),
                                sens_mat=AET1SensitivityMatrix(f, tdi2=True))
    ll_het = het.get_ll(W, **kw)

    out = {"meta": np.array([TOBS, F_LO, F_HI, SEED_PARAMS, SEED_NOISE, SEED_WALK, LENGTH,
                             LENGTH_HET]),
           "params": P, "walkers": W, "lnl": ll, "lnl_het": ll_het, "ncalls": np.array(len(CALLS))}
    kinds = {"arr": 0, "int": 1, "float": 2, "bool": 3}
    seen = {}

    def put(key, arr):
        """Store arr under key, or a reference to an identical array stored before."""
        arr = np.asarray(arr)
        dg = _digest(arr)
        if dg in seen:
            out[key] = np.array("ref:" + seen[dg])
        else:
            seen[dg] = key
            out[key] = arr

    for i, rec in enumerate(CALLS):
        out[f"c{i}_name"] = np.array(rec["name"])
        out[f"c{i}_kinds"] = np.array([kinds[k] for k, _ in rec["args"]], dtype=np.int8)
        orbit_call = rec["name"] == "pyFastLISAResponse.add_orbit_information"
        for k, (kind, v) in enumerate(rec["args"]):
            if k in rec["ptr_before"]:
                for b, arr in enumerate(rec["ptr_before"][k]):
                    put(f"c{i}_p{k}_{b}", arr)
                out[f"c{i}_a{k}"] = np.array(len(rec["ptr_before"][k]))  # binaries
            elif kind == "arr" and orbit_call:
                # the orbit tables are bbhx_b200.orbits.EqualArmlengthOrbits' (the lisatools
                # stand-in re-exports it): stored as a digest, regenerated by the replay
                out[f"c{i}_a{k}"] = np.array("sha256:" + _digest(v))
            elif kind == "arr":
                put(f"c{i}_a{k}", v)
            else:
                out[f"c{i}_a{k}"] = np.array(v)
        for k, v in rec["after"].items():
            if k in rec["ptr_before"]:
                continue
            if not np.array_equal(v, rec["args"][k][1], equal_nan=True):
                put(f"c{i}_o{k}", v)
        for k, arrs in rec["ptr_after"].items():
            for b, arr in enumerate(arrs):
                if not np.array_equal(arr, rec["ptr_before"][k][b], equal_nan=True):
                    put(f"c{i}_q{k}_{b}", arr)
    path = os.path.join(HERE, "dropin_trace.npz")
    np.savez_compressed(path, **out)
    names = [str(out[f"c{i}_name"]) for i in range(len(CALLS))]
    print(path, f"{os.path.getsize(path) / 1e6:.2f} MB,", len(CALLS), "calls")
    print(sorted(set(names)))
    print("lnl", ll, "lnl_het", ll_het)


if __name__ == "__main__":
    main()
