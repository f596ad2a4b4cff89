"""Array plumbing: torch CUDA tensors are the device container (the reference uses cupy)."""
import numpy as np


def torch():
    import torch as _t

    return _t


def device():
    t = torch()
    if not t.cuda.is_available():
        raise RuntimeError("bbhx_b200 needs a CUDA device (there is no CPU fallback)")
    return t.device("cuda", t.cuda.current_device())


def to_dev(x, dtype=None):
    """numpy / scalar / torch -> contiguous CUDA tensor (float64 unless dtype given)."""
    t = torch()
    dtype = dtype or t.float64
    if isinstance(x, t.Tensor):
        return x.to(device=device(), dtype=dtype).contiguous()
    return t.as_tensor(np.ascontiguousarray(x), dtype=dtype, device=device()).contiguous()


def to_np(x):
    t = torch()
    if isinstance(x, t.Tensor):
        return x.detach().cpu().numpy()
    return np.asarray(x)


def atleast_1d(x):
    t = torch()
    if isinstance(x, t.Tensor):
        return x.reshape(-1) if x.ndim == 0 else x
    return np.atleast_1d(x)
