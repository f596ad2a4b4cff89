// Block-cooperative tridiagonal solver shared by the spline build (spline.cu) and its
// adjoint (gradient.cu).
#pragma once

#include "bbhx_common.cuh"

namespace bbhx {

// In-place cyclic reduction on a[n], b[n], c[n] and P right-hand sides d[p*ld + i];
// solution returned in d.  All threads of the block participate.
__device__ inline void cr_solve(double* a, double* b, double* c, double* d, int ld, int P, int n) {
  for (int s = 1; s < n; s <<= 1) {
    int cnt = n / (2 * s);
    for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
      int i = 2 * s * k + 2 * s - 1;
      int im = i - s, ip = i + s;
      bool hp = ip < n;
      double al = -a[i] / b[im];
      double ga = hp ? -c[i] / b[ip] : 0.0;
      double an = al * a[im];
      double bn = b[i] + al * c[im] + (hp ? ga * a[ip] : 0.0);
      double cn = hp ? ga * c[ip] : 0.0;
      for (int p = 0; p < P; ++p) {
        double* dp = d + (size_t)p * ld;
        dp[i] = dp[i] + al * dp[im] + (hp ? ga * dp[ip] : 0.0);
      }
      a[i] = an;
      b[i] = bn;
      c[i] = cn;
    }
    __syncthreads();
  }
  int top = 1;
  while (top < n) top <<= 1;
  for (int s = top; s >= 1; s >>= 1) {
    int cnt = (n >= s) ? (n - s) / (2 * s) + 1 : 0;
    for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
      int i = s - 1 + 2 * s * k;
      int im = i - s, ip = i + s;
      for (int p = 0; p < P; ++p) {
        double* dp = d + (size_t)p * ld;
        double xm = (im >= 0) ? dp[im] : 0.0;
        double xp = (ip < n) ? dp[ip] : 0.0;
        dp[i] = (dp[i] - a[i] * xm - c[i] * xp) / b[i];
      }
    }
    __syncthreads();
  }
}

}  // namespace bbhx
