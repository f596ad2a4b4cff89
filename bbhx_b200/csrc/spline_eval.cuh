// Shared device helpers for evaluating the nine splined quantities on the data grid.
#pragma once

#include "bbhx_common.cuh"

namespace bbhx {

// The reference's tf gate (WaveformBuild.cu:50): accept when t_start <= tf and
// (tf <= t_end or t_end <= 0).
__device__ __forceinline__ bool tf_gate(double tf, double t_start, double t_end) {
  return (tf >= t_start) && ((tf <= t_end) || (t_end <= 0.0));
}

// conj(T_c * A e^{i phi}) for the three channels (WaveformBuild.cu:48-60)
__device__ __forceinline__ void combine_channels(double amp, double phase, cplx T1, cplx T2,
                                                 cplx T3, cplx& h1, cplx& h2, cplx& h3) {
  double s, c;
  sincos_cw(phase, &s, &c);
  cplx ap = mk(amp * c, amp * s);
  h1 = conj(T1 * ap);
  h2 = conj(T2 * ap);
  h3 = conj(T3 * ap);
}

// warp-cooperative searchsorted(row, v, side='right') - 1 over a sorted row of length L;
// every lane passes the same v and receives the same result in [-1, L-1].
__device__ __forceinline__ int warp_segment_search(const double* __restrict__ row, int L, double v) {
  int lane = threadIdx.x & 31;
  int lo = 0, hi = L;  // answer count = #{row[j] <= v} lies in [lo, hi]
  while (hi - lo > 32) {
    int step = (hi - lo + 31) / 32;
    int idx = lo + lane * step;
    bool le = (idx < hi) ? (__ldg(row + idx) <= v) : false;
    unsigned m = __ballot_sync(0xffffffffu, le);
    int c = __popc(m);  // lanes 0..c-1 satisfy row[idx] <= v
    if (c == 0) {
      hi = lo;  // v < row[lo] is impossible to refine further: count == lo
      break;
    }
    int nlo = lo + (c - 1) * step + 1;
    int nhi = lo + c * step;
    if (nhi > hi) nhi = hi;
    lo = nlo;
    hi = nhi;
  }
  // final: count = lo + #{j in [lo, hi) : row[j] <= v}
  int idx = lo + lane;
  bool le = (idx < hi) ? (__ldg(row + idx) <= v) : false;
  unsigned m = __ballot_sync(0xffffffffu, le);
  return lo + __popc(m) - 1;
}

}  // namespace bbhx
