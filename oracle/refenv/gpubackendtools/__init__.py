"""Stand-in for the external ``gpubackendtools`` package (dispatch only).

Provides what the reference uses: ``Globals().backends_manager.add_backends``
(__init__.py:40), ``get_backend``/``has_backend``/``get_first_backend`` (:44-47),
``ParallelModuleBase`` (utils/parallelbase.py:5-11) and ``wrapper`` (the .pyx files).
Every request resolves to the CPU backend, i.e. the reference's own C++ compiled for CPU.
"""
import numpy as np

from . import exceptions
from .gpubackendtools import Backend, BackendMethods, CpuBackend  # noqa: F401


class _BackendsManager:
    def __init__(self):
        self.classes = {}
        self.instances = {}

    def add_backends(self, d):
        self.classes.update(d)

    def get(self, name):
        if "cpu" not in name:
            name = "bbhx_cpu"
        if name not in self.instances:
            self.instances[name] = self.classes[name]()
        return self.instances[name]


class Globals:
    _mgr = _BackendsManager()

    @property
    def backends_manager(self):
        return Globals._mgr


def get_backend(name):
    return Globals._mgr.get(name)


def has_backend(name):
    return "cpu" in name


def get_first_backend(name):
    return Globals._mgr.get(name)


class ParallelModuleBase:
    def __init__(self, force_backend=None):
        self._force_backend = force_backend
        self._backend_obj = Globals._mgr.get("bbhx_cpu")

    @property
    def backend(self):
        return self._backend_obj

    @classmethod
    def GPU_RECOMMENDED(cls):
        return ["cpu"]

    @classmethod
    def CPU_ONLY(cls):
        return ["cpu"]


def wrapper(*args, **kwargs):
    out = [a.__array_interface__["data"][0] if isinstance(a, np.ndarray) else a for a in args]
    return out, kwargs
