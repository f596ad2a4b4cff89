// Forward-mode (tangent) parts of the gradient chain: dual-number setup of the per-mode
// PhenomHM and response records, and the contraction of the per-point tangents with the
// adjoint weights produced by the reverse part (heterodyne bin sums or spline adjoint).
//
// Gradient parameters (NGRAD = 11), in this order, with their index in the 12-row
// parameter array of BBHWaveformFD (waveformbuild.py:338-352):
//   0 m1 [Msun] (row 0)   1 m2 [Msun] (1)   2 chi1z (2)   3 chi2z (3)   4 distance [m] (4)
//   5 phi_ref (5)   6 inc (7)   7 lam (8)   8 beta (9)   9 psi (10)   10 t_ref [s] (11)
// f_ref (row 6) does not enter the model (the reference frequency is the amplitude peak).
//
// The 11 directions are carried GRAD_CHUNK at a time (passes k0 = 0, GRAD_CHUNK, ...): a
// dual number of GRAD_CHUNK tangents keeps much more of the model's working set in registers
// than one of 11 tangents, which spills to local memory.
#pragma once

#include "bbhx_common.cuh"
#include "dual.cuh"
#include "phenomhm_model.cuh"
#include "response_model.cuh"
#include "spline_eval.cuh"

namespace bbhx {

constexpr int NGRAD = 11;
constexpr int GRAD_CHUNK = 3;  // 3 per pass (4 passes): 11 % faster heterodyned gradients than 4 or 2
constexpr int GRAD_PASSES = (NGRAD + GRAD_CHUNK - 1) / GRAD_CHUNK;
using GD = ad::Dual<GRAD_CHUNK>;

// x seeded with tangent 1 in direction k (global index) when k is in this pass's chunk
__device__ __forceinline__ GD seed(double v, int k, int k0) {
  GD x(v);
  const int i = k - k0;
  if (i >= 0 && i < GRAD_CHUNK) x.d[i] = 1.0;
  return x;
}

struct GradParams {
  GD m1, m2, chi1, chi2, dist, phi_ref, inc, lam, beta, psi, t_ref;
};

// P: [12, B] row-major parameter array (device).
__device__ inline GradParams load_grad_params(const double* P, int B, int b, int k0) {
  GradParams g;
  g.m1 = seed(P[0 * (size_t)B + b], 0, k0);
  g.m2 = seed(P[1 * (size_t)B + b], 1, k0);
  g.chi1 = seed(P[2 * (size_t)B + b], 2, k0);
  g.chi2 = seed(P[3 * (size_t)B + b], 3, k0);
  g.dist = seed(P[4 * (size_t)B + b], 4, k0);
  g.phi_ref = seed(P[5 * (size_t)B + b], 5, k0);
  g.inc = seed(P[7 * (size_t)B + b], 6, k0);
  g.lam = seed(P[8 * (size_t)B + b], 7, k0);
  g.beta = seed(P[9 * (size_t)B + b], 8, k0);
  g.psi = seed(P[10 * (size_t)B + b], 9, k0);
  g.t_ref = seed(P[11 * (size_t)B + b], 10, k0);
  return g;
}

// Dual-number records of binaries [b0, b0 + nb): the same chain as the forward path
// (ringdown frequencies -> phm_setup_mode; response_mode_setup), with tangents seeded on the
// directions [k0, k0 + GRAD_CHUNK).  qnm: [8, nq] table y/c1/c2/c3 of the ringdown and damping
// splines.
static __global__ void k_grad_setup(ModeCoeffsT<GD>* coeffs, ResponseModeT<GD>* rmodes,
                                    const double* P, int B, int b0, int nb, const int* ells,
                                    const int* mms, int M, const double* qnm, int nq,
                                    double dspin, int run_phenomd, int k0) {
  const long long n = (long long)nb * M;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int bl = (int)(t / M), i = (int)(t % M);
    const int b = b0 + bl;
    const GradParams g = load_grad_params(P, B, b, k0);
    GD fm, fs;
    final_mass_spin(g.m1, g.m2, g.chi1, g.chi2, &fm, &fs);
    // PhenomD 22 ringdown / damping from the tabulated spline (PhenomHMWaveform.cu:1930-1993)
    const int ind = int((fs.v - (-1.0)) / dspin);
    const GD x = fs - (dspin * ind + (-1.0));
    const GD x2 = x * x, x3 = x2 * x;
    const double* y_rd = qnm;
    const double* y_dm = qnm + 4 * (size_t)nq;
    const GD rd22 = (y_rd[ind] + y_rd[nq + ind] * x + y_rd[2 * nq + ind] * x2 +
                     y_rd[3 * nq + ind] * x3) / fm;
    const GD dm22 = (y_dm[ind] + y_dm[nq + ind] * x + y_dm[2 * nq + ind] * x2 +
                     y_dm[3 * nq + ind] * x3) / fm;
    const int ell = run_phenomd ? 2 : ells[i];
    const int mm = run_phenomd ? 2 : mms[i];
    GD rd_lm = rd22, dm_lm = dm22;
    if (!run_phenomd) {
      const cplxT<GD> z = qnm_cw(fs, ell, mm);
      rd_lm = (0.5 / PI) * z.re / fm;
      dm_lm = (0.5 / PI) * z.im / fm;
    }
    phm_setup_mode(coeffs[t], g.m1 * MSUN_SI, g.m2 * MSUN_SI, g.chi1, g.chi2, g.dist, ell, mm,
                   rd_lm, dm_lm, rd22, dm22, run_phenomd);
    response_mode_setup(rmodes[t], ell, mm, g.phi_ref, g.inc, g.lam, g.beta, g.psi);
  }
}

// Waveform phasor term W_c = T_c A e^{i (phase + Roemer)} of one (mode, frequency) with
// tangents, and its t(f) (for the observation gate).  Phase and t(f) include the t_ref shift
// (phenomhm.py:485-507).
struct PointTangents {
  cplxT<GD> W[3];
  GD amp, phase;  // phase including the t_ref shift and the Roemer delay
  cplxT<GD> T[3];
  double tf;
};

// The frequency is a double (fixed grid) or a GD whose tangents are the knot's own motion
// dx/dtheta, in which case the tangents are total derivatives along the moving knot.
template <typename F>
__device__ inline PointTangents point_tangents(const ModeCoeffsT<GD>& c, const ResponseModeT<GD>& r,
                                               const OrbitTables& orb, const F& f, const GD& t_ref,
                                               double t_init, int TDItag, int rescaled, int tdi2) {
  PointTangents o;
  const PointOutT<GD> w = phm_eval_point(c, GD(f));
  const GD tf = w.tf + t_ref;
  o.tf = tf.v;
  const TransferT<GD> T = response_point(r, orb, f, tf, TDItag, rescaled, tdi2);
  o.amp = w.amp;
  o.phase = w.phase + (2 * PI * f) * (t_ref - t_init) + T.phaseRdelay;
  const cplxT<GD> ap = w.amp * expi(o.phase);
  o.T[0] = T.L1;
  o.T[1] = T.L2;
  o.T[2] = T.L3;
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) o.W[ch] = o.T[ch] * ap;
  return o;
}

// Sum of the GRAD_CHUNK partials over the block into out[k0 + k] for the directions < NGRAD.
__device__ inline void block_reduce_grad(double* acc, double* out, int k0) {
  __shared__ double red[GRAD_CHUNK][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < GRAD_CHUNK; ++k) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[k][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < GRAD_CHUNK && k0 + (int)threadIdx.x < NGRAD) {
    double s = 0.0;
    for (int q = 0; q < nw; ++q) s += red[threadIdx.x][q];
    out[k0 + threadIdx.x] = s;
  }
  __syncthreads();
}

// Heterodyne contraction: grad[b] = sum_{mode, j, channel} Re(gh[b, c, j] dW_c/dtheta) over
// the sparse grid freqs[j] (lnL depends on h = sum_modes conj(W), and dL = Re(gh dW)).
// One CTA per binary of [b0, b0 + nb); records indexed relative to b0.
static __global__ void k_contract_het(double* grad, const ModeCoeffsT<GD>* coeffs,
                                      const ResponseModeT<GD>* rmodes, OrbitTables orb,
                                      const double* P, int B, int b0, int nb,
                                      const double* t_start, const double* t_end, double t_init,
                                      const double* freqs, const cplx* gh, int TDItag,
                                      int rescaled, int tdi2, int M, int L, int k0) {
  for (int bl = blockIdx.x; bl < nb; bl += gridDim.x) {
    const int b = b0 + bl;
    const GD t_ref = seed(P[11 * (size_t)B + b], 10, k0);
    const double ts = t_start[b], te = t_end[b];
    double acc[GRAD_CHUNK];
#pragma unroll
    for (int k = 0; k < GRAD_CHUNK; ++k) acc[k] = 0.0;
    for (int p = threadIdx.x; p < M * L; p += blockDim.x) {
      const int m = p / L, j = p % L;
      const PointTangents o =
          point_tangents(coeffs[(size_t)bl * M + m], rmodes[(size_t)bl * M + m], orb, freqs[j],
                         t_ref, t_init, TDItag, rescaled, tdi2);
      if (!tf_gate(o.tf, ts, te)) continue;
#pragma unroll
      for (int ch = 0; ch < 3; ++ch) {
        const cplx u = gh[((size_t)b * 3 + ch) * L + j];
#pragma unroll
        for (int k = 0; k < GRAD_CHUNK; ++k)
          acc[k] += u.re * o.W[ch].re.d[k] - u.im * o.W[ch].im.d[k];
      }
    }
    block_reduce_grad(acc, grad + (size_t)b * NGRAD, k0);
  }
}

// Direct-likelihood contraction at the spline knots: grad[b] = sum_{mode, i} (sum_p
// ybar[p, b, m, i] d q_p / d theta + xbar[b, m, i] d x_i / d theta), with q_p the sparse-grid
// quantities of the [9, B, M, L] buffer (amplitude, phase with t_ref shift and Roemer delay,
// the six transfer components; t(f), p = 2, only gates) and x_i the knots.  The knots move
// with theta through the observation-window regrid: d x_i = x_i ((1 - r_i) wlo + r_i whi),
// r_i = i / (L - 1), with (wlo, whi) = (d flo / flo, d fhi / fhi) of the row from
// k_regrid_tangents (wreg [nb * M][2][GRAD_CHUNK], local rows); q_p is differentiated along the
// moving knot (the frequency is a dual carrying d x_i).
static __global__ void k_contract_direct(double* grad, const ModeCoeffsT<GD>* coeffs,
                                         const ResponseModeT<GD>* rmodes, OrbitTables orb,
                                         const double* P, int B, int b0, int nb, double t_init,
                                         const double* x, const double* ybar, const double* xbar,
                                         const double* wreg, int TDItag, int rescaled, int tdi2,
                                         int M, int L, int k0) {
  const size_t n = (size_t)B * M * L;
  const double inv_span = 1.0 / (double)(L - 1);
  for (int bl = blockIdx.x; bl < nb; bl += gridDim.x) {
    const int b = b0 + bl;
    const GD t_ref = seed(P[11 * (size_t)B + b], 10, k0);
    double acc[GRAD_CHUNK];
#pragma unroll
    for (int k = 0; k < GRAD_CHUNK; ++k) acc[k] = 0.0;
    for (int p = threadIdx.x; p < M * L; p += blockDim.x) {
      const int m = p / L, i = p % L;
      const size_t o = ((size_t)b * M + m) * L + i;
      const double w0 = ybar[o], w1 = ybar[n + o], xb = xbar[o];
      double wt[6];
      bool any = (w0 != 0.0) || (w1 != 0.0) || (xb != 0.0);
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        wt[q] = ybar[(size_t)(3 + q) * n + o];
        any = any || (wt[q] != 0.0);
      }
      if (!any) continue;
      const double* wr = wreg + ((size_t)bl * M + m) * 2 * GRAD_CHUNK;
      const double r = i * inv_span;
      GD fk(x[o]);
#pragma unroll
      for (int k = 0; k < GRAD_CHUNK; ++k)
        fk.d[k] = x[o] * ((1.0 - r) * wr[k] + r * wr[GRAD_CHUNK + k]);
      const PointTangents pt = point_tangents(coeffs[(size_t)bl * M + m], rmodes[(size_t)bl * M + m],
                                              orb, fk, t_ref, t_init, TDItag, rescaled, tdi2);
#pragma unroll
      for (int k = 0; k < GRAD_CHUNK; ++k) {
        double v = w0 * pt.amp.d[k] + w1 * pt.phase.d[k] + xb * fk.d[k];
#pragma unroll
        for (int ch = 0; ch < 3; ++ch)
          v += wt[2 * ch] * pt.T[ch].re.d[k] + wt[2 * ch + 1] * pt.T[ch].im.d[k];
        acc[k] += v;
      }
    }
    block_reduce_grad(acc, grad + (size_t)b * NGRAD, k0);
  }
}

}  // namespace bbhx
