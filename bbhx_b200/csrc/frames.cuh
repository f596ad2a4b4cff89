// LISA-frame <-> SSB-frame time of arrival, shared by the driver kernels (driver.cu) and the
// observation-window tangents of the direct gradient (gradient.cu).
#pragma once

#include "bbhx_common.cuh"

namespace bbhx {

constexpr double ORBIT_R = AU_SI;                // OrbitR (utils/constants.py)
constexpr double CONST_OMEGA = 1.99098659277e-7;  // 2 pi / sidereal year (ConstOmega)

// tSSBfromLframe (transform.py:75-105): SSB time of constellation time tL for a source at
// ecliptic (lambda, beta), first order in R/c plus the R^2/c^2 term.  T = double, or a dual
// number in (lam, beta) for the derivative of the SSB observation limits.
template <typename T>
__device__ __forceinline__ T tssb_from_l(double tL, const T& lam, const T& beta, double t0) {
  const T phase = CONST_OMEGA * tL + CONST_OMEGA * t0 - lam;
  const double RoC = ORBIT_R / C_SI;
  const T rc = RoC * cos(beta);
  return tL + rc * cos(phase) - 0.5 * CONST_OMEGA * (rc * rc) * sin(2.0 * phase);
}

}  // namespace bbhx
