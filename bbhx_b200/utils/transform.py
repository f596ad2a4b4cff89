"""Frame and sky-mode transforms for massive-black-hole binaries (the reference's
src/bbhx/utils/transform.py), on numpy arrays or torch tensors (CPU or CUDA) alike.

* ``tSSBfromLframe`` / ``tLfromSSBframe`` (transform.py:75-135): retarded time at the LISA
  constellation centre <-> SSB time for a source at ecliptic (lambda, beta), first order in
  the orbit plus the O(R^2/c^2) correction (Marsat et al., arXiv:2003.00357).
* ``LISA_to_SSB`` / ``SSB_to_LISA`` (transform.py:136-294): time, sky position and
  polarisation between the constellation frame and the SSB frame.  The constellation plane is
  inclined by zeta = pi/3 to the ecliptic and its orientation follows the orbital phase
  alpha = Omega t + Phi0, so a sky direction maps as k_SSB = Rz(alpha) Ry(-zeta) Rz(-alpha) k_L
  (inverse with +zeta); the polarisation rotates by the angle between the two frames' "north"
  directions projected on the sky.  LISA -> SSB needs the SSB time inside alpha and is solved
  by three fixed-point passes, as in the reference.
* ``mbh_sky_mode_transform`` (transform.py:296-426): the 8 (4 longitudinal x 2 latitudinal)
  degenerate sky modes of a source.
* ``mT_q``, ``modpi``, ``mod2pi`` (transform.py:28-72).

numpy inputs are transformed with numpy on the host, as the reference does; CUDA tensors go
through the library's kernels (bbhx_tssb_from_lframe, bbhx_frame_transform,
bbhx_sky_mode_transform), one launch per call.
"""
import math

import numpy as np

from .constants import C_SI, ConstOmega, OrbitR, YRSID_SI

ZETA = math.pi / 3.0


def _is_torch(x):
    try:
        import torch

        return isinstance(x, torch.Tensor)
    except ImportError:
        return False


def _is_cuda(*xs):
    return any(_is_torch(x) and x.is_cuda for x in xs)


def _cuda_args(*xs):
    """float64 contiguous device tensors of a common broadcast shape, and that shape."""
    import torch

    ts = [x if _is_torch(x) else torch.as_tensor(x, dtype=torch.float64) for x in xs]
    dev = next(t.device for t in ts if t.is_cuda)
    ts = torch.broadcast_tensors(*[t.to(device=dev, dtype=torch.float64) for t in ts])
    shape = ts[0].shape
    return [t.contiguous().reshape(-1) for t in ts], shape


class _Ops:
    """The handful of elementwise functions used here, for numpy or torch."""

    def __init__(self, *xs):
        self.torch = any(_is_torch(x) for x in xs)
        if self.torch:
            import torch

            self.m = torch
            self.atan2 = torch.atan2
            self.asin = torch.asin
        else:
            self.m = np
            self.atan2 = np.arctan2
            self.asin = np.arcsin

    def __getattr__(self, name):
        return getattr(self.m, name)


def mT_q(mT, q):
    """(m1, m2) from total mass and mass ratio q < 1."""
    return mT / (1 + q), mT * q / (1 + q)


def modpi(phase):
    """phase reduced to [0, pi)."""
    ops = _Ops(phase)
    return phase - ops.floor(phase / np.pi) * np.pi


def mod2pi(phase):
    """phase reduced to [0, 2 pi)."""
    ops = _Ops(phase)
    return phase - ops.floor(phase / (2 * np.pi)) * 2 * np.pi


def _tssb_cuda(t, lam, beta, t0, inverse):
    """tSSBfromLframe / tLfromSSBframe of CUDA tensors in one library kernel."""
    import torch

    from .. import _lib

    (t, lam, beta), shape = _cuda_args(t, lam, beta)
    out = torch.empty_like(t)
    _lib.call("bbhx_tssb_from_lframe", _lib.dptr(out), _lib.dptr(t), _lib.dptr(lam),
              _lib.dptr(beta), t.numel(), float(t0), int(inverse), _lib.stream())
    return out.reshape(shape)


def tSSBfromLframe(tL, lambdaSSB, betaSSB, t0=0.0):
    if _is_cuda(tL, lambdaSSB, betaSSB):
        return _tssb_cuda(tL, lambdaSSB, betaSSB, t0, 0)
    ops = _Ops(tL, lambdaSSB, betaSSB)
    phase = ConstOmega * tL + ConstOmega * t0 - lambdaSSB
    RoC = OrbitR / C_SI
    cb = ops.cos(betaSSB)
    return tL + RoC * cb * ops.cos(phase) - 0.5 * ConstOmega * (RoC * cb) ** 2 * ops.sin(2.0 * phase)


def tLfromSSBframe(tSSB, lambdaSSB, betaSSB, t0=0.0):
    if _is_cuda(tSSB, lambdaSSB, betaSSB):
        return _tssb_cuda(tSSB, lambdaSSB, betaSSB, t0, 1)
    ops = _Ops(tSSB, lambdaSSB, betaSSB)
    phase = ConstOmega * tSSB + ConstOmega * t0 - lambdaSSB
    return tSSB - OrbitR / C_SI * ops.cos(betaSSB) * ops.cos(phase)


def _rotate_sky(lam, beta, alpha, zeta, ops):
    """(lambda', beta') of the direction (lambda, beta) rotated by Rz(alpha) Ry(-zeta)
    Rz(-alpha), and the polarisation-frame angle between the two frames."""
    d = lam - alpha
    cb, sb = ops.cos(beta), ops.sin(beta)
    cd, sd = ops.cos(d), ops.sin(d)
    cz, sz = math.cos(zeta), math.sin(zeta)
    # Rz(-alpha): (cb cd, cb sd, sb); Ry(-zeta): x' = x cz - z sz, z' = x sz + z cz
    x1 = cb * cd * cz - sb * sz
    y1 = cb * sd
    z1 = cb * cd * sz + sb * cz
    ca, sa = ops.cos(alpha), ops.sin(alpha)
    lam_new = ops.atan2(x1 * sa + y1 * ca, x1 * ca - y1 * sa)
    beta_new = ops.asin(z1)
    dpsi = ops.atan2(sz * sd, cb * cz - sb * sz * cd)
    return lam_new, beta_new, dpsi


def _frame_cuda(t, lam, beta, psi, t0, to_ssb):
    import torch

    from .. import _lib

    ins, shape = _cuda_args(t, lam, beta, psi)
    outs = [torch.empty_like(ins[0]) for _ in range(4)]
    _lib.call("bbhx_frame_transform", *[_lib.dptr(o) for o in outs], *[_lib.dptr(i) for i in ins],
              ins[0].numel(), float(t0 * YRSID_SI), int(to_ssb), _lib.stream())
    return tuple(o.reshape(shape) for o in outs)


def LISA_to_SSB(tL, lambdaL, betaL, psiL, t0=0.0):
    """(tSSB, lambdaSSB, betaSSB, psiSSB) from the constellation-frame values; t0 in years.
    CUDA tensors run in one library kernel (bbhx_frame_transform)."""
    if _is_cuda(tL, lambdaL, betaL, psiL):
        return _frame_cuda(tL, lambdaL, betaL, psiL, t0, 1)
    ops = _Ops(tL, lambdaL, betaL, psiL)
    t0 = t0 * YRSID_SI
    tSSB = tL
    for _ in range(3):
        alpha = ConstOmega * tSSB + ConstOmega * t0
        lam, beta, dpsi = _rotate_sky(lambdaL, betaL, alpha, ZETA, ops)
        tSSB = tSSBfromLframe(tL, lam, beta, t0)
    return tSSB, lam % (2 * np.pi), beta, modpi(psiL + dpsi)


def SSB_to_LISA(tSSB, lambdaSSB, betaSSB, psiSSB, t0=0.0):
    """(tL, lambdaL, betaL, psiL) from the SSB-frame values; t0 in years.  CUDA tensors run in
    one library kernel (bbhx_frame_transform)."""
    if _is_cuda(tSSB, lambdaSSB, betaSSB, psiSSB):
        return _frame_cuda(tSSB, lambdaSSB, betaSSB, psiSSB, t0, 0)
    ops = _Ops(tSSB, lambdaSSB, betaSSB, psiSSB)
    t0 = t0 * YRSID_SI
    alpha = ConstOmega * tSSB + ConstOmega * t0
    lam, beta, dpsi = _rotate_sky(lambdaSSB, betaSSB, alpha, -ZETA, ops)
    return tLfromSSBframe(tSSB, lambdaSSB, betaSSB, t0), lam, beta, modpi(psiSSB + dpsi)


def mbh_sky_mode_transform(coords, ind_map=None, kind="both", inplace=False, cos_i=False):
    """Copies of each parameter set in its 8 ("both"), 4 longitudinal ("long") or 2
    latitudinal ("lat") sky modes, interleaved as in the reference (row r of the output is mode
    r % factor of set r // ...); with ``inplace`` the rows of ``coords`` are taken as already
    tiled and are transformed in place.  coords: (num_sets, ndim), numpy or torch."""
    if ind_map is None:
        ind_map = dict(inc=7, lam=8, beta=9, psi=10)
    elif not isinstance(ind_map, dict):
        raise ValueError("If providing the ind_map kwarg, it must be a dict.")
    factors = {"both": 8, "long": 4, "lat": 2}
    if kind not in factors:
        raise ValueError("The kwarg 'kind' must be lat for latitudinal transformation, long for "
                         "longitudinal transformation, or both for both.")
    factor = factors[kind]
    torch_in = _is_torch(coords)
    if torch_in and coords.is_cuda:
        import torch

        from .. import _lib

        if inplace and coords.shape[0] % factor != 0:
            raise ValueError(
                "If performing an inplace transformation, the coords provided must have a first "
                "dimension size divisible by {} for a '{}' transformation.".format(factor, kind))
        out = coords if inplace else coords.repeat(factor, 1)
        work = out if (out.dtype == torch.float64 and out.is_contiguous()) else \
            out.to(torch.float64).contiguous()
        _lib.call("bbhx_sky_mode_transform", _lib.dptr(work), work.shape[0], work.shape[1],
                  ind_map["inc"], ind_map["lam"], ind_map["beta"], ind_map["psi"],
                  {"both": 0, "long": 1, "lat": 2}[kind], int(bool(cos_i)), _lib.stream())
        if work is not out:
            out.copy_(work)
        return out
    if inplace:
        if coords.shape[0] % factor != 0:
            raise ValueError(
                "If performing an inplace transformation, the coords provided must have a first "
                "dimension size divisible by {} for a '{}' transformation.".format(factor, kind))
    else:
        coords = coords.repeat(factor, 1) if torch_in else np.tile(coords, (factor, 1))
    inc, lam, beta, psi = ind_map["inc"], ind_map["lam"], ind_map["beta"], ind_map["psi"]
    if kind in ("both", "lat"):  # latitudinal mirror: beta -> -beta, inc -> pi - inc, psi -> pi - psi
        if cos_i:
            coords[1::2, inc] *= -1
        else:
            coords[1::2, inc] = np.pi - coords[1::2, inc]
        coords[1::2, beta] *= -1
        coords[1::2, psi] = np.pi - coords[1::2, psi]
    # longitudinal: lambda + i pi/2 (mod 2 pi), psi + i pi/2 (mod pi), i = 1..3
    rows = [(i, slice(i, None, 4)) for i in range(1, 4)] if kind == "long" else []
    if kind == "both":
        rows = [(i, slice(2 * i + j, None, 8)) for i in range(1, 4) for j in range(2)]
    for i, sl in rows:
        coords[sl, lam] = (coords[sl, lam] + np.pi / 2 * i) % (2 * np.pi)
        coords[sl, psi] = (coords[sl, psi] + np.pi / 2 * i) % np.pi
    return coords
