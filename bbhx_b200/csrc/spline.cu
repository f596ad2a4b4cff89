// Batched not-a-knot cubic splines.
//
// Reference interface replaced: interpolate() (src/bbhx/cutils/Interpolate.hh:4-6,
// Interpolate.cu:320-359) which fills the tridiagonal system for every (param, binary,
// mode) (fill_B, :14-182), solves it with cusparseDgtsv2StridedBatch / LAPACKE_dgtsv
// (:201-241) and converts slopes to cubic coefficients (:245-318).
//
// Here one CTA owns one (binary, mode) system: the P interpolated quantities share the
// same knots x and therefore the same matrix, so the CTA builds the matrix once, carries
// all P right-hand sides through one cyclic reduction in shared memory (log2 L levels
// down, log2 L levels back up), and writes the slopes and coefficients coalesced.
//
// System for the slopes s_i (scipy CubicSpline "not-a-knot"):
//   row 0:     (x2-x1) s0 + (x2-x0) s1 = ((dx1 + 2 d) dx2 m1 + dx1^2 m2) / d
//   row i:     dx2 s_{i-1} + 2 (dx1 + dx2) s_i + dx1 s_{i+1} = 3 (dx2 m1 + dx1 m2)
//   row L-1:   d s_{L-2} + dx1 s_{L-1} = (dx2^2 m1 + (2 d + dx2) dx1 m2) / d
// (dx1, dx2 the two intervals around the row, d = dx1 + dx2, m1, m2 their secant slopes).
// Coefficients on segment i: y(x) = y_i + c1 u + c2 u^2 + c3 u^3, u = x - x_i, with
//   c1 = s_i,  t = (s_i + s_{i+1} - 2 m) / h,  c2 = (m - s_i) / h - t,  c3 = t / h.
// Entry L-1 of c1/c2/c3 (no segment) holds the last row's (upper, diagonal, lower)
// coefficients, as the reference GPU path leaves them.
#include "capi_internal.cuh"
#include "sparse_stages.cuh"

namespace bbhx {

// x: [S, L]; y: [P, S, L]; outputs slopes / c1 / c2 / c3 in y's layout (any may alias the
// reference's B / upper / diag / lower buffers).  `scratch` (used only when the system does
// not fit in shared memory) holds gridDim.x * (4 + P) * L doubles.
__global__ void k_spline(const double* __restrict__ x, const double* __restrict__ y,
                         double* slopes, double* c1, double* c2, double* c3, int L, int P,
                         long long S, bool use_smem, double* scratch) {
  extern __shared__ double smem[];
  double* work = use_smem ? smem : scratch + (size_t)blockIdx.x * (4 + P) * L;
  for (long long sys = blockIdx.x; sys < S; sys += gridDim.x) {
    const long long o = sys * L;
    spline_system(x + o, y + o, S * L, slopes ? slopes + o : nullptr, c1 + o, c2 + o, c3 + o, L,
                  P, work);
  }
}

}  // namespace bbhx

using namespace bbhx;

namespace {
constexpr size_t kMaxSplineSmem = 200 * 1024;
}

extern "C" {

// Interpolate.hh:4-6: freqs [B*M, L], y [P, B, M, L]; B_ receives the slopes, upper_diag /
// diag / lower_diag receive c1 / c2 / c3 (the reference reuses those buffers the same way).
int bbhx_interpolate(const double* freqs, const double* y, double* B_, double* upper_diag,
                     double* diag, double* lower_diag, int length, int num_interp_params,
                     int num_modes, int num_bin_all, void* stream) {
  BBHX_REQUIRE(length >= 3, "spline length must be >= 3 (not-a-knot)");
  BBHX_REQUIRE(num_interp_params >= 1 && num_modes >= 1 && num_bin_all >= 0, "bad sizes");
  long long S = (long long)num_modes * num_bin_all;
  if (S == 0) return OK;
  cudaStream_t s = (cudaStream_t)stream;
  size_t smem = sizeof(double) * (size_t)(4 + num_interp_params) * length;
  bool use_smem = smem <= kMaxSplineSmem;
  int threads = 256;
  const long long nsm = sm_count();
  unsigned int grid = (unsigned int)(S < nsm * 16 ? S : nsm * 16);
  double* scratch = nullptr;
  if (use_smem) {
    BBHX_CHECK_CUDA(cudaFuncSetAttribute(k_spline, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kMaxSplineSmem));
  } else {
    grid = (unsigned int)(S < nsm * 2 ? S : nsm * 2);
    BBHX_CHECK_CUDA(pool_alloc((void**)&scratch, sizeof(double) * grid * (4 + num_interp_params) * (size_t)length, s));
  }
  k_spline<<<grid, threads, use_smem ? smem : 0, s>>>(freqs, y, B_, upper_diag, diag, lower_diag,
                                                      length, num_interp_params, S, use_smem,
                                                      scratch);
  int st = launch_status("k_spline");
  if (scratch) pool_free(scratch, s);
  return st;
}

}  // extern "C"
