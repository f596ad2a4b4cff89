"""Frame-time transforms used when setting the observation window.

Restates ``tSSBfromLframe`` / ``tLfromSSBframe`` of the reference
(src/bbhx/utils/transform.py:75-135, after Marsat et al., arXiv:2003.00357): conversion
between the retarded time at the LISA constellation centre and the SSB time for a source
at ecliptic (lambda, beta), to first order in the orbit with the O(R^2/c^2) correction.
These run on the host on (B,) parameter arrays, as in the reference.
"""
import numpy as np

from .constants import C_SI, ConstOmega, OrbitR


def tSSBfromLframe(tL, lambdaSSB, betaSSB, t0=0.0):
    ConstPhi0 = ConstOmega * t0
    phase = ConstOmega * tL + ConstPhi0 - lambdaSSB
    RoC = OrbitR / C_SI
    return (tL + RoC * np.cos(betaSSB) * np.cos(phase)
            - 1.0 / 2 * ConstOmega * pow(RoC * np.cos(betaSSB), 2) * np.sin(2.0 * phase))


def tLfromSSBframe(tSSB, lambdaSSB, betaSSB, t0=0.0):
    ConstPhi0 = ConstOmega * t0
    phase = ConstOmega * tSSB + ConstPhi0 - lambdaSSB
    RoC = OrbitR / C_SI
    return tSSB - RoC * np.cos(betaSSB) * np.cos(phase)
