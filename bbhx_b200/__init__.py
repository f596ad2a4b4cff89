"""bbhx_b200: B200-native (sm_100a) implementation of the BBHx batched
waveform -> likelihood path (PhenomHM -> fast LISA TDI response -> cubic spline ->
direct and heterodyned likelihood), drop-in for the reference's Python API.

Device arrays are torch CUDA tensors; compute runs in ``libbbhx_b200.so`` (C ABI in
``include/bbhx_b200.h``).  There is no CPU fallback.
"""
__version__ = "0.1.0"

from .orbits import EqualArmlengthOrbits, Orbits  # noqa: F401
from .sensitivity import AET1SensitivityMatrix, aet_psd  # noqa: F401
from .utils.constants import *  # noqa: F401,F403


def __getattr__(name):
    # the GPU classes import torch lazily so that host-only utilities load without CUDA
    if name in ("PhenomHMAmpPhase", "PhenomHMAMPPhase"):
        from .waveforms.phenomhm import PhenomHMAmpPhase

        return PhenomHMAmpPhase
    if name == "LISATDIResponse":
        from .response.fastfdresponse import LISATDIResponse

        return LISATDIResponse
    if name == "CubicSplineInterpolant":
        from .utils.interpolate import CubicSplineInterpolant

        return CubicSplineInterpolant
    if name in ("BBHWaveformFD", "TemplateInterpFD"):
        from . import waveformbuild

        return getattr(waveformbuild, name)
    if name in ("Likelihood", "HeterodynedLikelihood"):
        from . import likelihood

        return getattr(likelihood, name)
    if name == "workspace":
        from .workspace import workspace

        return workspace
    raise AttributeError(name)
