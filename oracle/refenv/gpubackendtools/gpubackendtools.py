"""Minimal backend classes with the names the reference imports
(cutils/__init__.py:10, __init__.py:50).  CPU only: ``xp`` is numpy."""
import dataclasses
import typing

import numpy


@dataclasses.dataclass
class BackendMethods:
    xp: typing.Any


class Backend:
    _name = "base"

    @property
    def name(self):
        return self._name


class CpuBackend(Backend):
    def __init__(self, *args, **kwargs):
        self.xp = numpy
        self.uses_gpu = False
        self.uses_cupy = False

    @staticmethod
    def check_numpy():
        return numpy


class Cuda11xBackend(Backend):
    def __init__(self, *args, **kwargs):
        raise RuntimeError("CUDA backends are not part of the reference oracle")


class Cuda12xBackend(Cuda11xBackend):
    pass
