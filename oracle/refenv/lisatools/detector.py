"""``lisatools.detector`` stand-in (fastfdresponse.py:23): analytic equal-arm orbits."""
from bbhx_b200.orbits import EqualArmlengthOrbits as _EAO
from bbhx_b200.orbits import Orbits  # noqa: F401


class _CpuName:
    name = "lisatools_cpu"


class EqualArmlengthOrbits(_EAO):
    def __init__(self, *args, force_backend=None, **kwargs):
        super().__init__(*args, **kwargs)
        self.backend = _CpuName()
