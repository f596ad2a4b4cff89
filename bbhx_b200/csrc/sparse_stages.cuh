// Per-element steps of the sparse-grid build (PhenomHM records, default grid, t(f), the
// observation-window regrid, waveform + TDI response, not-a-knot spline), shared by the
// one-stage-per-launch kernels (phenomhm.cu, response.cu, spline.cu, driver.cu) and the fused
// row builder of uneven batches (sparse_build.cu), so that both compute the same numbers.
#pragma once

#include "bbhx_common.cuh"
#include "frames.cuh"
#include "phenomhm_model.cuh"
#include "response_model.cuh"
#include "tridiag.cuh"

namespace bbhx {

// m1 >= m2 ordering (the spins follow their masses) and the SI masses (phenomhm.py:303-316).
struct FrontMasses {
  double m1, m2, chi1, chi2, m1_SI, m2_SI;
};
__device__ __forceinline__ FrontMasses front_masses(double a1, double a2, double x1, double x2) {
  const bool sw = a1 < a2;
  FrontMasses o;
  o.m1 = sw ? a2 : a1;
  o.m2 = sw ? a1 : a2;
  o.chi1 = sw ? x2 : x1;
  o.chi2 = sw ? x1 : x2;
  o.m1_SI = o.m1 * MSUN_SI;
  o.m2_SI = o.m2 * MSUN_SI;
  return o;
}

// Ringdown / damping frequency of mode (ell, mm) from the QNM fits at the final mass and spin
// (get_phenomhm_ringdown_frequencies, PhenomHMWaveform.cu:1816-1928).
__device__ __forceinline__ void ringdown_hm(double m1, double m2, double chi1, double chi2,
                                            int ell, int mm, double* fr, double* fd) {
  double fm, fs;
  final_mass_spin(m1, m2, chi1, chi2, &fm, &fs);
  const cplx z = qnm_cw(fs, ell, mm);
  *fr = (0.5 / PI) * z.re / fm;
  *fd = (0.5 / PI) * z.im / fm;
}

// PhenomD 22 ringdown / damping frequency at final spin fs, final mass fm from the tabulated
// final-spin splines (get_phenomd_ringdown_frequencies, PhenomHMWaveform.cu:1930-2062).
__device__ __forceinline__ void phenomd_qnm_lookup(double fs, double fm, const double* y_rd,
                                                   const double* c1_rd, const double* c2_rd,
                                                   const double* c3_rd, const double* y_dm,
                                                   const double* c1_dm, const double* c2_dm,
                                                   const double* c3_dm, double dspin,
                                                   double* fr, double* fd) {
  int ind = int((fs - (-1.0)) / dspin);
  double x = fs - (dspin * ind + (-1.0));
  double x2 = x * x, x3 = x2 * x;
  double r = y_rd[ind] + c1_rd[ind] * x + c2_rd[ind] * x2 + c3_rd[ind] * x3;
  double d = y_dm[ind] + c1_dm[ind] * x + c2_dm[ind] * x2 + c3_dm[ind] * x3;
  *fr = r / fm;
  *fd = d / fm;
}

// The same for binary masses / spins; T: [8, nq] table (y, c1, c2, c3 of the ringdown spline,
// then of the damping spline).
__device__ __forceinline__ void ringdown_d(double m1, double m2, double chi1, double chi2,
                                           const double* T, int nq, double dspin, double* fr,
                                           double* fd) {
  double fm, fs;
  final_mass_spin(m1, m2, chi1, chi2, &fm, &fs);
  phenomd_qnm_lookup(fs, fm, T, T + nq, T + 2 * nq, T + 3 * nq, T + 4 * nq, T + 5 * nq,
                     T + 6 * nq, T + 7 * nq, dspin, fr, fd);
}

// Point k of the default sparse grid (phenomhm.py:208-224): logspace(mf_min, mf_max, L) over
// the total mass in seconds, times m / 2.
__device__ __forceinline__ double default_freq(int k, int L, double mf_min, double mf_max,
                                               double m1, double m2, int mm) {
  const double start = log10(mf_min), stop = log10(mf_max);
  const double step = (stop - start) / (double)(L - 1);
  const double y = (k == L - 1) ? stop : __dadd_rn(__dmul_rn((double)k, step), start);
  const double base = pow(10.0, y);
  const double Msec = (m1 + m2) * MTSUN_SI;
  return base / Msec * (double)mm / 2;
}

// t(f) of one mode without the t_ref shift (the first pass of phenomhm.py:485-507).
__device__ __forceinline__ double phm_tf_value(const ModeCoeffs& c, double f) {
  const double Mf = f * c.M_sec;
  double Mfp;
  if (c.phenomd_only)
    Mfp = Mf;
  else if (!(Mf > c.ph_fi))
    Mfp = c.ph_ai * Mf;
  else if (!(Mf > c.ph_fr))
    Mfp = c.ph_am * Mf + c.ph_bm;
  else
    Mfp = c.ph_ar * Mf;
  if (c.phenomd_only)
    return c.M_sec * phenomd_dphase(c.d, Mfp) / (2 * PI) - (c.t0 / (2. * PI) * c.M_sec);
  return c.M_sec * (phenomd_dphase(c.d, Mfp) / (2. * PI)) - (c.t0 / (2. * PI) * c.M_sec);
}

// Observation-window edges of one (binary, mode) row (phenomhm.py:520-606): the default
// grid's ends, or where the chord of t(f) over f crosses 0 (lower) or To (upper).  err: 0, or
// 1 / 2 when the lower / upper edge needs clipping but the row does not cross exactly once.
struct WindowEdges {
  double flo, fhi;
  int err;
};
// The edges of one row by the whole block: the minima and maxima of t(f) and f, and the number
// and first index of the intervals whose t(f) crosses 0 and To, by block reductions (exact, so
// independent of the block size), then the crossing formulas of phenomhm.py:520-606.
__device__ inline WindowEdges tf_window_edges_block(const double* f, const double* x, int L,
                                                    double To) {
  __shared__ double r_d[4][32];
  __shared__ int r_i[4][32];
  __shared__ WindowEdges out;
  double tmin = x[0], tmax = x[0], flo = f[0], fhi = f[0];
  int c0 = 0, c1 = 0, s0 = L, s1 = L;
  for (int i = threadIdx.x; i < L; i += blockDim.x) {
    tmin = fmin(tmin, x[i]);
    tmax = fmax(tmax, x[i]);
    flo = fmin(flo, f[i]);
    fhi = fmax(fhi, f[i]);
    if (i < L - 1) {
      if ((0.0 < x[i + 1]) && (0.0 > x[i])) {
        ++c0;
        s0 = min(s0, i);
      }
      if ((To < x[i + 1]) && (To > x[i])) {
        ++c1;
        s1 = min(s1, i);
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    tmin = fmin(tmin, __shfl_xor_sync(0xffffffffu, tmin, o));
    tmax = fmax(tmax, __shfl_xor_sync(0xffffffffu, tmax, o));
    flo = fmin(flo, __shfl_xor_sync(0xffffffffu, flo, o));
    fhi = fmax(fhi, __shfl_xor_sync(0xffffffffu, fhi, o));
    c0 += __shfl_xor_sync(0xffffffffu, c0, o);
    c1 += __shfl_xor_sync(0xffffffffu, c1, o);
    s0 = min(s0, __shfl_xor_sync(0xffffffffu, s0, o));
    s1 = min(s1, __shfl_xor_sync(0xffffffffu, s1, o));
  }
  const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if ((threadIdx.x & 31) == 0) {
    r_d[0][w] = tmin; r_d[1][w] = tmax; r_d[2][w] = flo; r_d[3][w] = fhi;
    r_i[0][w] = c0; r_i[1][w] = c1; r_i[2][w] = s0; r_i[3][w] = s1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < nw; ++k) {
      tmin = fmin(tmin, r_d[0][k]);
      tmax = fmax(tmax, r_d[1][k]);
      flo = fmin(flo, r_d[2][k]);
      fhi = fmax(fhi, r_d[3][k]);
      c0 += r_i[0][k];
      c1 += r_i[1][k];
      s0 = min(s0, r_i[2][k]);
      s1 = min(s1, r_i[3][k]);
    }
    WindowEdges e;
    e.err = 0;
    e.flo = flo;
    e.fhi = fhi;
    if (tmin < 0.0) {
      if (c0 != 1) {
        e.err = 1;
      } else {
        double m = (f[s0 + 1] - f[s0]) / (x[s0 + 1] - x[s0]);
        e.flo = m * (0.0 - x[s0]) + f[s0];
      }
    }
    if (tmax > To) {
      if (c1 != 1) {
        if (e.err == 0) e.err = 2;
      } else {
        double m = (f[s1 + 1] - f[s1]) / (x[s1 + 1] - x[s1]);
        e.fhi = m * (To - x[s1]) + f[s1];
      }
    }
    out = e;
  }
  __syncthreads();
  return out;
}

// Knot k of the regridded row (phenomhm.py:608-610, numpy.logspace: y_k = k * step + start
// with two roundings, the last y = stop, f = 10**y).
__device__ __forceinline__ double window_knot(int k, int L, double flo, double fhi) {
  const double start = log10(flo), stop = log10(fhi);
  const double step = (stop - start) / (double)(L - 1);
  const double y = (k == L - 1) ? stop : __dadd_rn(__dmul_rn((double)k, step), start);
  return pow(10.0, y);
}

// The nine sparse-buffer slots of one (binary, mode, frequency) point: amplitude, phase (with
// the t_ref shift and the Roemer delay), t(f) (with t_ref) and the six TDI transfer components;
// buf slot p at buf[p * n + t].
__device__ __forceinline__ void phm_response_point(double* buf, long long n, long long t, double f,
                                                   const ModeCoeffs& c, const ResponseMode& r,
                                                   const OrbitTables& orb, double tr,
                                                   double t_init, int TDItag, int rescaled,
                                                   int tdi2) {
  PointOut o = phm_eval_point(c, f);
  o.phase += f * (tr - t_init) * 2 * PI;
  o.tf += tr;
  const Transfer T = response_point(r, orb, f, o.tf, TDItag, rescaled, tdi2);
  buf[t] = o.amp;
  buf[n + t] = o.phase + T.phaseRdelay;
  buf[2 * n + t] = o.tf;
  buf[3 * n + t] = T.L1.re;
  buf[4 * n + t] = T.L1.im;
  buf[5 * n + t] = T.L2.re;
  buf[6 * n + t] = T.L2.im;
  buf[7 * n + t] = T.L3.re;
  buf[8 * n + t] = T.L3.im;
}

// Not-a-knot spline of one system (knots xg[L], P quantities y[p * pstride + i]) by the whole
// block: matrix once, P right-hand sides through one cyclic reduction in `work`
// ((4 + P) L doubles: x, a, b, c, d[P][L]); slopes (optional) and c1, c2, c3 written in y's
// layout.  Entry L-1 of c1 / c2 / c3 holds the last row's (0, diagonal, lower) entries.
// PT > 0 fixes P at compile time: a row's 3 PT (right-hand sides) and 2 PT (coefficients)
// global loads are then issued together into registers instead of one quantity at a time.
template <int PT>
__device__ inline void spline_system_t(const double* xg, const double* y, long long pstride,
                                       double* slopes, double* c1, double* c2, double* c3, int L,
                                       int Pr, double* work) {
  const int P = PT > 0 ? PT : Pr;
  constexpr int NV = PT > 0 ? PT : 1;
  double* xs = work;
  double* a = xs + L;
  double* b = a + L;
  double* c = b + L;
  double* d = c + L;
  for (int i = threadIdx.x; i < L; i += blockDim.x) xs[i] = xg[i];
  __syncthreads();
  for (int i = threadIdx.x; i < L; i += blockDim.x) {
    int i0, i1, i2;
    if (i == 0) {
      i0 = 0; i1 = 1; i2 = 2;
    } else if (i == L - 1) {
      i0 = L - 3; i1 = L - 2; i2 = L - 1;
    } else {
      i0 = i - 1; i1 = i; i2 = i + 1;
    }
    const double dx1 = xs[i1] - xs[i0];
    const double dx2 = xs[i2] - xs[i1];
    const double dd = xs[i2] - xs[i0];
    if (i == 0) {
      a[i] = 0.0; b[i] = dx2; c[i] = dd;
    } else if (i == L - 1) {
      a[i] = dd; b[i] = dx1; c[i] = 0.0;
    } else {
      a[i] = dx2; b[i] = 2 * (dx1 + dx2); c[i] = dx1;
    }
    for (int p0 = 0; p0 < P; p0 += NV) {
      double v0[NV], v1[NV], v2[NV];
#pragma unroll
      for (int q = 0; q < NV; ++q) {
        const double* yg = y + (long long)(p0 + q) * pstride;
        v0[q] = yg[i0];
        v1[q] = yg[i1];
        v2[q] = yg[i2];
      }
#pragma unroll
      for (int q = 0; q < NV; ++q) {
        const double m1 = (v1[q] - v0[q]) / dx1;
        const double m2 = (v2[q] - v1[q]) / dx2;
        double r;
        if (i == 0)
          r = ((dx1 + 2 * dd) * dx2 * m1 + dx1 * dx1 * m2) / dd;
        else if (i == L - 1)
          r = (dx2 * dx2 * m1 + (2 * dd + dx2) * dx1 * m2) / dd;
        else
          r = 3.0 * (dx2 * m1 + dx1 * m2);
        d[(size_t)(p0 + q) * L + i] = r;
      }
    }
  }
  __syncthreads();
  // keep the last row's matrix entries for the c1/c2/c3[L-1] convention
  const double last_a = a[L - 1], last_b = b[L - 1];
  __syncthreads();
  cr_solve(a, b, c, d, L, P, L);
  for (int i = threadIdx.x; i < L; i += blockDim.x) {
    const bool seg = i < L - 1;
    const double h = seg ? xs[i + 1] - xs[i] : 1.0;
    for (int p0 = 0; p0 < P; p0 += NV) {
      double ylo[NV], yhi[NV];
#pragma unroll
      for (int q = 0; q < NV; ++q) {
        const double* yg = y + (long long)(p0 + q) * pstride;
        ylo[q] = yg[i];
        yhi[q] = seg ? yg[i + 1] : 0.0;
      }
#pragma unroll
      for (int q = 0; q < NV; ++q) {
        const long long o = (long long)(p0 + q) * pstride;
        const double* sp = d + (size_t)(p0 + q) * L;
        const double si = sp[i];
        if (slopes) slopes[o + i] = si;
        if (seg) {
          const double m = (yhi[q] - ylo[q]) / h;
          const double t = (si + sp[i + 1] - 2 * m) / h;
          c1[o + i] = si;
          c2[o + i] = (m - si) / h - t;
          c3[o + i] = t / h;
        } else {
          c1[o + i] = 0.0;
          c2[o + i] = last_b;
          c3[o + i] = last_a;
        }
      }
    }
  }
  __syncthreads();
}

// The interpolants of the sparse buffer are nine quantities (amplitude, phase, t(f) and six
// transfer components); other counts take the generic path.
__device__ inline void spline_system(const double* xg, const double* y, long long pstride,
                                     double* slopes, double* c1, double* c2, double* c3, int L,
                                     int P, double* work) {
  if (P == 9)
    spline_system_t<9>(xg, y, pstride, slopes, c1, c2, c3, L, P, work);
  else
    spline_system_t<0>(xg, y, pstride, slopes, c1, c2, c3, L, P, work);
}

}  // namespace bbhx
