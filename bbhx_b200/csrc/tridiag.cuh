// Block-cooperative tridiagonal solver shared by the spline build (spline.cu) and its
// adjoint (gradient.cu).
#pragma once

#include "bbhx_common.cuh"

namespace bbhx {

// Forward-reduction step of cyclic reduction at stride s for row i = 2 s k + 2 s - 1.
__device__ __forceinline__ void cr_reduce_row(double* a, double* b, double* c, double* d, int ld,
                                              int P, int n, int s, int k) {
  const int i = 2 * s * k + 2 * s - 1;
  const int im = i - s, ip = i + s;
  const bool hp = ip < n;
  const double al = -a[i] / b[im];
  const double ga = hp ? -c[i] / b[ip] : 0.0;
  const double an = al * a[im];
  const double bn = b[i] + al * c[im] + (hp ? ga * a[ip] : 0.0);
  const double cn = hp ? ga * c[ip] : 0.0;
  for (int p = 0; p < P; ++p) {
    double* dp = d + (size_t)p * ld;
    dp[i] = dp[i] + al * dp[im] + (hp ? ga * dp[ip] : 0.0);
  }
  a[i] = an;
  b[i] = bn;
  c[i] = cn;
}

// Back-substitution step at stride s for row i = s - 1 + 2 s k (one division per row).
__device__ __forceinline__ void cr_solve_row(const double* a, const double* b, const double* c,
                                             double* d, int ld, int P, int n, int s, int k) {
  const int i = s - 1 + 2 * s * k;
  const int im = i - s, ip = i + s;
  const double ib = 1.0 / b[i], ai = a[i], ci = c[i];
  for (int p = 0; p < P; ++p) {
    double* dp = d + (size_t)p * ld;
    const double xm = (im >= 0) ? dp[im] : 0.0;
    const double xp = (ip < n) ? dp[ip] : 0.0;
    dp[i] = (dp[i] - ai * xm - ci * xp) * ib;
  }
}

// In-place cyclic reduction on a[n], b[n], c[n] and P right-hand sides d[p*ld + i];
// solution returned in d.  All threads of the block participate.  The levels with at most 32
// active rows (the deep end of the reduction and the start of the substitution) run in warp 0
// with warp-level synchronisation only, so the block meets at a barrier once per wide level.
__device__ inline void cr_solve(double* a, double* b, double* c, double* d, int ld, int P, int n) {
  const int t = threadIdx.x;
  int s = 1;
  for (; s < n && n / (2 * s) > 32; s <<= 1) {
    const int cnt = n / (2 * s);
    for (int k = t; k < cnt; k += blockDim.x) cr_reduce_row(a, b, c, d, ld, P, n, s, k);
    __syncthreads();
  }
  if (t < 32) {
    for (; s < n; s <<= 1) {
      if (t < n / (2 * s)) cr_reduce_row(a, b, c, d, ld, P, n, s, t);
      __syncwarp();
    }
  }
  __syncthreads();
  int top = 1;
  while (top < n) top <<= 1;
  auto count = [n](int st) { return (n >= st) ? (n - st) / (2 * st) + 1 : 0; };
  s = top;
  if (t < 32) {
    for (; s >= 1 && count(s) <= 32; s >>= 1) {
      if (t < count(s)) cr_solve_row(a, b, c, d, ld, P, n, s, t);
      __syncwarp();
    }
  } else {
    while (s >= 1 && count(s) <= 32) s >>= 1;
  }
  __syncthreads();
  for (; s >= 1; s >>= 1) {
    const int cnt = count(s);
    for (int k = t; k < cnt; k += blockDim.x) cr_solve_row(a, b, c, d, ld, P, n, s, k);
    __syncthreads();
  }
}

}  // namespace bbhx
