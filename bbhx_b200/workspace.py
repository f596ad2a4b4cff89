"""Caller-provided device workspace for the library's scratch (``bbhx_workspace_set``).

A framework that owns the GPU's memory (PyTorch's caching allocator here) can hand the library
one buffer; every entry point called on this thread inside the block takes its scratch from it
instead of the stream-ordered pool, and the buffer's address stays fixed (useful under CUDA
graph capture).  The buffer serves the current stream: calls on other streams must not overlap.
"""
import contextlib

from . import _lib
from .utils.arrays import device, torch


@contextlib.contextmanager
def workspace(buf):
    """Use ``buf`` (a CUDA tensor, or a size in bytes for a new uint8 tensor) as the library's
    scratch for the calls made inside the block; yields the tensor."""
    t = torch()
    if isinstance(buf, int):
        buf = t.empty(buf + 256, dtype=t.uint8, device=device())
    if not isinstance(buf, t.Tensor) or not buf.is_cuda:
        raise TypeError("workspace: expected a CUDA tensor or a size in bytes")
    addr = buf.data_ptr()
    base = (addr + 255) & ~255
    size = buf.numel() * buf.element_size() - (base - addr)
    _lib.call("bbhx_workspace_set", _lib._VP(base), size)
    try:
        yield buf
    finally:
        _lib.call("bbhx_workspace_set", _lib._VP(0), 0)


def peak():
    """Largest scratch extent (bytes) the calling thread's calls needed since the workspace was
    set, including a request that did not fit."""
    return int(_lib.lib().bbhx_workspace_peak())
