"""torch.autograd front end of the gradient kernels.

``HeterodynedLnL`` and ``DirectLnL`` are ``torch.autograd.Function``s whose forward pass is
the fused likelihood kernel and whose backward pass recomputes the waveform and runs the
gradient chain on the GPU (reverse through the likelihood reduction, forward-mode tangents
through PhenomHM + TDI); nothing from the forward pass is kept except the parameters.

Parameters are a [12, B] tensor in the BBHWaveformFD order (m1, m2, chi1z, chi2z, distance,
phi_ref, f_ref, inc, lam, beta, psi, t_ref); the gradient with respect to f_ref is zero
because the model does not depend on it (the reference frequency is the amplitude peak).
"""
from .utils.arrays import device, torch

GRAD_ROWS = (0, 1, 2, 3, 4, 5, 7, 8, 9, 10, 11)


def scatter_grad(grad, g_out):
    """[B, 11] d lnL / d theta and the upstream [B] gradient -> [12, B] parameter gradient."""
    t = torch()
    B = grad.shape[0]
    out = t.zeros((12, B), dtype=t.float64, device=grad.device)
    out[list(GRAD_ROWS)] = (grad * g_out.reshape(-1, 1)).T
    return out


def _het_function():
    t = torch()

    class HeterodynedLnL(t.autograd.Function):
        @staticmethod
        def forward(ctx, params, like, kw):
            ctx.like, ctx.kw = like, kw
            ctx.save_for_backward(params)
            ll, _ = like._fused_ll(params, kw, "fp64")
            return ll

        @staticmethod
        def backward(ctx, g_out):
            (params,) = ctx.saved_tensors
            _, grad = ctx.like.get_ll_and_grad(params, **ctx.kw)
            return scatter_grad(grad, g_out), None, None

    return HeterodynedLnL


def _direct_function():
    t = torch()

    class DirectLnL(t.autograd.Function):
        @staticmethod
        def forward(ctx, params, like, kw):
            ctx.like, ctx.kw = like, kw
            ctx.save_for_backward(params)
            return like._device_ll(params, kw)

        @staticmethod
        def backward(ctx, g_out):
            (params,) = ctx.saved_tensors
            _, grad = ctx.like.get_ll_and_grad(params, **ctx.kw)
            return scatter_grad(grad, g_out), None, None

    return DirectLnL


_cache = {}


def function(kind):
    """The autograd Function class for "heterodyned" or "direct" (built on first use)."""
    if kind not in _cache:
        _cache[kind] = _het_function() if kind == "heterodyned" else _direct_function()
    return _cache[kind]


def as_param_tensor(params):
    """[12, B] float64 device tensor from a (12,) / (12, B) array or tensor."""
    t = torch()
    p = t.as_tensor(params, dtype=t.float64, device=device())
    if p.ndim == 1:
        p = p.reshape(-1, 1)
    if p.shape[0] != 12 and p.shape[-1] == 12:
        p = p.T
    return p.contiguous()
