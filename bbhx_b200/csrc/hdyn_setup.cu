// Heterodyne (relative-binning) set-up on the device.
//
// Replaces the per-bin Python loop of HeterodynedLikelihood.init_heterodyne_info
// (src/bbhx/likelihood.py:480-530): for the dense points of the narrowed band, with the
// reference template h0, data d, PSD S and bin width df,
//   A0 = 4 conj(h0) d / S df,   A1 = A0 (f - f_m),   B0 = 4 |h0|^2 / S df,   B1 = B0 (f - f_m),
// summed per relative-binning bin j (freqs[j] <= f < freqs[j+1], the reference's
// searchsorted(side="right") - 1) into slot j + 1, the last dense point excluded (the
// reference's inds_keep[-1] = False), and the reference sums <d|d>, <h0|h0>, Re<d|h0> over the
// whole band.  The bins are contiguous runs of the sorted dense grid, so each CTA finds its run
// by binary search and reduces it in a fixed order (deterministic); no atomics.
#include "capi_internal.cuh"

namespace bbhx {

constexpr int HS_THREADS = 256;

__device__ __forceinline__ int lower_bound_dev(const double* __restrict__ f, int n, double v) {
  int lo = 0, hi = n;  // first i with f[i] >= v
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (f[mid] < v) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// Block-wide sum of NV doubles per thread (fixed shuffle tree, then warp 0); the totals end up
// in sh[0..NV) on return.
template <int NV>
__device__ __forceinline__ void block_sum(double* v, double (*sh)[HS_THREADS / 32]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) sh[k][warp] = v[k];
  __syncthreads();
  if (threadIdx.x < NV) {
    double t = 0.0;
    for (int w = 0; w < HS_THREADS / 32; ++w) t += sh[threadIdx.x][w];
    sh[threadIdx.x][0] = t;
  }
  __syncthreads();
}

// One CTA per bin j = 0 .. L-2.  consts [4, 3, L] complex (slot 0 zeroed by CTA 0);
// partial [L-1, 3]: this run's <d|d>, <h0|h0>, Re<d|h0> for the final sum.
__global__ void __launch_bounds__(HS_THREADS) k_hdyn_bins(
    cplx* __restrict__ consts, double* __restrict__ partial, const double* __restrict__ f,
    const cplx* __restrict__ d, int ld_d, const cplx* __restrict__ h0, int ld_h,
    const double* __restrict__ S, int ld_s, int n, const double* __restrict__ freqs, int L,
    double df) {
  __shared__ int run[3];
  __shared__ double sh[27][HS_THREADS / 32];
  const int j = blockIdx.x;
  if (threadIdx.x == 0) {
    const int lo = (j == 0) ? 0 : lower_bound_dev(f, n, freqs[j]);
    const int hi = lower_bound_dev(f, n, freqs[j + 1]);
    run[0] = lo;
    run[1] = min(hi, n - 1);             // constants: the last dense point excluded
    run[2] = (j == L - 2) ? n : hi;      // reference sums: every point of the band
  }
  __syncthreads();
  const int lo = run[0], hi_c = run[1], hi_r = run[2];
  const double fm = (freqs[j + 1] + freqs[j]) / 2;
  double v[27];
#pragma unroll
  for (int k = 0; k < 27; ++k) v[k] = 0.0;
  for (int i = lo + threadIdx.x; i < hi_r; i += HS_THREADS) {
    const double fi = f[i];
    const bool in_c = i < hi_c;
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
      const cplx h = h0[(long long)ch * ld_h + i];
      const cplx dd = d[(long long)ch * ld_d + i];
      const double s = S[(long long)ch * ld_s + i];
      // same operation order as the reference: ((4 (conj(h0) x)) / S) df
      const double ar = (4.0 * (h.re * dd.re + h.im * dd.im)) / s * df;
      const double ai = (4.0 * (h.re * dd.im - h.im * dd.re)) / s * df;
      const double b0 = (4.0 * (h.re * h.re + h.im * h.im)) / s * df;
      const double w = fi - fm;
      double* a = v + 8 * ch;  // A0 re, A0 im, A1 re, A1 im, B0, B1 of this channel
      if (in_c) {
        a[0] += ar;
        a[1] += ai;
        a[2] += ar * w;
        a[3] += ai * w;
        a[4] += b0;
        a[5] += b0 * w;
      }
      v[24] += (4.0 * (dd.re * dd.re + dd.im * dd.im)) / s * df;
      v[25] += b0;
      v[26] += ar;
    }
  }
  block_sum<27>(v, sh);
  if (threadIdx.x < 3) {
    const int ch = threadIdx.x;
    const long long slot = j + 1;
    const double* a = &sh[8 * ch][0];
    const int st = HS_THREADS / 32;  // row stride of sh
    consts[(0LL * 3 + ch) * L + slot] = mk(a[0 * st], a[1 * st]);
    consts[(1LL * 3 + ch) * L + slot] = mk(a[2 * st], a[3 * st]);
    consts[(2LL * 3 + ch) * L + slot] = mk(a[4 * st], 0.0);
    consts[(3LL * 3 + ch) * L + slot] = mk(a[5 * st], 0.0);
    partial[3LL * j + ch] = sh[24 + ch][0];
    if (j == 0)
      for (int k = 0; k < 4; ++k) consts[((long long)k * 3 + ch) * L] = mk(0.0, 0.0);
  }
}

// ref[0..2] = <d|d>, <h0|h0>, Re<d|h0>: the L-1 run partials summed in bin order.
__global__ void k_hdyn_ref_sums(const double* __restrict__ partial, int nb, double* ref) {
  if (threadIdx.x < 3) {
    double t = 0.0;
    for (int j = 0; j < nb; ++j) t += partial[3LL * j + threadIdx.x];
    ref[threadIdx.x] = t;
  }
}

}  // namespace bbhx

using namespace bbhx;

extern "C" {

// Relative-binning constants of HeterodynedLikelihood (no C counterpart in the reference: the
// Python loop of likelihood.py:480-530).  f [n]: the narrowed dense grid (sorted); d, h0:
// complex128 rows of 3 channels with row strides ld_d, ld_h (elements); S: PSD rows, stride
// ld_s; freqs [L]: the sparse grid, freqs[0] <= f[0] and f[n-1] <= freqs[L-1]; df: the dense
// bin width.  consts: complex128 [4, 3, L] (A0, A1, B0, B1, overwritten); ref: double [3] =
// <d|d>, <h0|h0>, Re<d|h0> over the band (device).
int bbhx_hdyn_constants(void* consts, double* ref, const double* f, const void* d, int ld_d,
                        const void* h0, int ld_h, const double* S, int ld_s, int n,
                        const double* freqs, int L, double df, void* stream) {
  BBHX_REQUIRE(L >= 2 && n >= 2, "need L >= 2 sparse and n >= 2 dense frequencies");
  BBHX_REQUIRE(ld_d >= n && ld_h >= n && ld_s >= n, "row strides must be >= n");
  cudaStream_t s = (cudaStream_t)stream;
  double* partial = nullptr;
  BBHX_CHECK_CUDA(pool_alloc((void**)&partial, sizeof(double) * 3 * (size_t)(L - 1), s));
  k_hdyn_bins<<<L - 1, HS_THREADS, 0, s>>>((cplx*)consts, partial, f, (const cplx*)d, ld_d,
                                           (const cplx*)h0, ld_h, S, ld_s, n, freqs, L, df);
  int st = launch_status("k_hdyn_bins");
  if (!st) {
    k_hdyn_ref_sums<<<1, 32, 0, s>>>(partial, L - 1, ref);
    st = launch_status("k_hdyn_ref_sums");
  }
  pool_free(partial, s);
  return st;
}

}  // extern "C"
