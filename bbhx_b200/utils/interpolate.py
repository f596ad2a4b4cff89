"""Batched not-a-knot cubic splines on the GPU.

Drop-in for the reference's ``CubicSplineInterpolant`` (src/bbhx/utils/interpolate.py:42-257):
same constructor (flattened arrays with explicit sizes, or shaped (B, M, L) / (P, B, M, L)
arrays), the ``c1`` / ``c2`` / ``c3`` / ``container`` attributes in the reference layout,
and ``__call__`` evaluation.  The coefficients come from the library's shared-memory
cyclic-reduction solve (``bbhx_interpolate``).
"""
from .. import _lib
from ..utils.arrays import device, to_dev, torch


class CubicSplineInterpolant:
    def __init__(self, x, y_all, num_interp_params=None, num_bin_all=None, num_modes=None,
                 length=None, force_backend=None):
        t = torch()
        x = to_dev(x)
        y_all = to_dev(y_all)
        if x.ndim == 1 or y_all.ndim == 1:
            if x.ndim != 1 or y_all.ndim != 1:
                raise ValueError("If providing flattened x and y_all, need to both be flattened.")
            if length is None or num_modes is None or num_bin_all is None or num_interp_params is None:
                raise ValueError(
                    "If providing flattened arrays, need to provide dimensional information: "
                    "length, num_modes, num_bin_all, num_interp_params.")
            if len(x) != length * num_modes * num_bin_all:
                raise ValueError(
                    f"Length of the x array is not correct. It is supposed to be "
                    f"{length * num_modes * num_bin_all}. It is currently {len(x)}.")
            if len(y_all) != length * num_modes * num_bin_all * num_interp_params:
                raise ValueError(
                    f"Length of the y_all array is not correct. It is supposed to be "
                    f"{length * num_modes * num_bin_all * num_interp_params}. It is currently {len(y_all)}.")
        else:
            if x.ndim != 3:
                raise ValueError("If providing shaped array, needs to be 3D with shape (num_bin_all, num_modes, length).")
            if y_all.ndim != 4:
                raise ValueError(
                    "If providing shaped array, needs to be 4D with shape (num_interp_params, num_bin_all, num_modes, length).")
            num_interp_params, num_bin_all, num_modes, length = y_all.shape
            assert tuple(y_all.shape[1:]) == tuple(x.shape)
            x = x.flatten()
            y_all = y_all.flatten()
        ninterps = num_modes * num_interp_params * num_bin_all
        self.degree = 3
        self.length = length
        self.reshape_shape = (num_interp_params, num_bin_all, num_modes, length)
        self.x_reshape_shape = (num_bin_all, num_modes, length)
        self.B = t.empty(ninterps * length, dtype=t.float64, device=device())
        self.c1 = t.empty_like(self.B)
        self.c2 = t.empty_like(self.B)
        self.c3 = t.empty_like(self.B)
        self.y = y_all
        _lib.call("bbhx_interpolate", _lib.dptr(x), _lib.dptr(y_all), _lib.dptr(self.B),
                  _lib.dptr(self.c1), _lib.dptr(self.c2), _lib.dptr(self.c3), length,
                  num_interp_params, num_modes, num_bin_all, _lib.stream())
        self.x = x

    @property
    def xp(self):
        return torch()

    @property
    def x_shaped(self):
        return self.x.reshape(self.x_reshape_shape)

    @property
    def y_shaped(self):
        return self.y.reshape(self.reshape_shape)

    @property
    def c1_shaped(self):
        return self.c1.reshape(self.reshape_shape)

    @property
    def c2_shaped(self):
        return self.c2.reshape(self.reshape_shape)

    @property
    def c3_shaped(self):
        return self.c3.reshape(self.reshape_shape)

    @property
    def container(self):
        return [self.x, self.y, self.c1, self.c2, self.c3]

    def __call__(self, x_new):
        """Evaluate at x_new with shape (B, M, n) (interpolate.py:213-257)."""
        t = torch()
        x_new = to_dev(x_new)
        if x_new.ndim == 3 and tuple(x_new.shape[:2]) != self.x_reshape_shape[:2]:
            raise ValueError("x_new must have 3D shape of (num_bin_all, num_modes, # of new points)")
        xs = self.x_shaped
        assert bool((x_new <= xs.max(dim=-1).values[:, :, None]).all()) and bool(
            (x_new >= xs.min(dim=-1).values[:, :, None]).all())
        seg = t.searchsorted(xs.reshape(-1, self.length).contiguous(),
                             x_new.reshape(-1, x_new.shape[-1]).contiguous(), right=True) - 1
        seg = seg.reshape(x_new.shape)
        seg = t.where(seg == self.length - 1, self.length - 2, seg)
        x0 = t.take_along_dim(xs, seg, dim=-1)
        idx = seg[None].expand(self.reshape_shape[0], *seg.shape)
        y0 = t.take_along_dim(self.y_shaped, idx, dim=-1)
        c1 = t.take_along_dim(self.c1_shaped, idx, dim=-1)
        c2 = t.take_along_dim(self.c2_shaped, idx, dim=-1)
        c3 = t.take_along_dim(self.c3_shaped, idx, dim=-1)
        dx = x_new - x0
        return y0 + c1 * dx + c2 * dx ** 2 + c3 * dx ** 3
