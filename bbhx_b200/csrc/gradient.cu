// Gradient of the direct likelihood, d lnL / d theta for the 11 parameters of
// gradient_model.cuh, without stored templates.
//
// lnL = Re<d|h> - <h|h> / 2 - <d|d> / 2 on the data grid, with h the cubic-spline
// interpolation of the sparse [9, B, M, L] buffer (amplitude, phase, t(f), six transfer
// components) summed over modes (TemplateInterpFD + direct_like: waveformbuild.py:89-239,
// Likelihood.cu:356-471).  The chain, for a batch of binaries:
//   1. the FP64 fused likelihood kernel (likelihood.cu, direct_fused_gh) writes d lnL / d h
//                     at every (binary, data bin):  g = 4 w (d~ - w h)                  (reverse)
//                     and the batch's <d|h>, <h|h>
//   2. k_adj_coeffs   warp per (binary, mode, spline segment): d lnL / d (y, c1, c2, c3) of
//                     the 8 interpolated quantities, summed over the segment's data bins
//   3. k_spline_adj   CTA per (binary, mode): adjoint of the not-a-knot spline build; the
//                     slopes' system K s = r is transposed and solved by the same cyclic
//                     reduction (K^T lambda = s_bar), giving d lnL / d y at the knots
//                     and d lnL / d x (the knots' positions, y held fixed)
//   4. k_grad_setup + k_regrid_tangents + k_contract_direct: dual-number tangents of the
//                     model at the knots and of the knots themselves (the observation-window
//                     regrid moves them with theta), contracted with d lnL / d y and
//                     d lnL / d x                                                  (forward)
#include <algorithm>
#include <vector>

#include "capi_internal.cuh"
#include "frames.cuh"
#include "gradient_model.cuh"
#include "tridiag.cuh"

namespace bbhx {
int direct_fused_gh(cplx* gh, const long long* gh_off, double* d_h, double* h_h,
                    const int* start, const int* len, const double* data_freqs,
                    const double* data, const double* noise, int N, const double* x,
                    const double* y, const double* c1, const double* c2, const double* c3,
                    const double* t_start, const double* t_end, int M, int L, int B_all, int b0,
                    int nb, cudaStream_t s);
}  // namespace bbhx

extern "C" int bbhx_template_support(int* start, int* len, const double* x, int num_modes,
                                     int length, int num_bin_all, const double* data_freqs,
                                     int data_length, void* stream);

namespace bbhx {

// segment of knot row xs[0..L) holding f: s = (#x <= f) - 1 (searchsorted right - 1)
__device__ __forceinline__ int knot_segment(const double* xs, int L, double f) {
  int a = 0, c = L;
  while (a < c) {
    const int mid = (a + c) >> 1;
    if (xs[mid] <= f) a = mid + 1;
    else c = mid;
  }
  return a - 1;
}

// first index k with f[k] >= v
__device__ __forceinline__ int lower_bound_d(const double* f, int n, double v) {
  int a = 0, c = n;
  while (a < c) {
    const int mid = (a + c) >> 1;
    if (f[mid] < v) a = mid + 1;
    else c = mid;
  }
  return a;
}

// lower_bound_d with the index guessed from the grid's end points (exact for a uniform grid,
// the common case) and checked by at most four one-step moves; otherwise the binary search.
// Same result as lower_bound_d for any sorted grid.
__device__ __forceinline__ int lower_bound_guess(const double* f, int n, double v) {
  if (n == 0) return 0;
  const double f0 = f[0], f1 = f[n - 1];
  if (!(v > f0)) return 0;
  if (v > f1) return n;  // here f0 < v <= f1, so n >= 2 and the answer is in [1, n - 1]
  int k = (int)ceil((v - f0) / (f1 - f0) * (double)(n - 1));
  k = min(max(k, 1), n - 1);
  for (int it = 0; it < 4; ++it) {
    if (f[k] < v) {
      ++k;  // k < answer <= n - 1
    } else if (f[k - 1] >= v) {
      --k;  // k - 1 >= answer >= 1
    } else {
      return k;
    }
  }
  return lower_bound_d(f, n, v);
}

struct SplineRefs {
  const double *x, *y, *c1, *c2, *c3;  // x [B, M, L]; y, c1..c3 [9, B, M, L]
  size_t n;                            // B * M * L
  int M, L;
};

// 2. Warp per (local binary, mode, segment s < L-1): sums over the segment's data bins of
// a_p, a_p u, a_p u^2, a_p u^3 with a_p = d lnL / d q_p (p = amp, phase, 6 transfers), into
// ybd (d lnL / d y directly) and cb1..cb3 (d lnL / d c1..c3), all [9, B, M, L].
// Each lane walks its own bins of the segment (k0 + lane, + 32, ...) and keeps the 32 moment
// sums of those bins in registers; at the end of the segment one transposing reduction across
// the warp (31 shuffles) leaves the total of moment l = (p, k) = (l / 4, l % 4) in lane l.
constexpr int ADJ_THREADS = 128;

// m[0..31] of every lane -> lane l returns the warp total of m[l] (recursive halving: at the
// step of width w a lane keeps the half of its w values whose index bit matches its lane bit).
__device__ __forceinline__ double warp_transpose_sum32(double (&m)[32], int lane) {
#pragma unroll
  for (int w = 16; w >= 1; w >>= 1) {
    const bool upper = (lane & w) != 0;
#pragma unroll
    for (int i = 0; i < w; ++i) {
      const double send = upper ? m[i] : m[i + w];
      const double keep = upper ? m[i + w] : m[i];
      m[i] = keep + __shfl_xor_sync(0xffffffffu, send, w);
    }
  }
  return m[0];
}

__global__ void __launch_bounds__(ADJ_THREADS, 3)
k_adj_coeffs(double* ybd, double* cb1, double* cb2, double* cb3, const cplx* gh,
             const long long* off, const int* start, const int* len, SplineRefs S,
             const double* data_freqs, int N, const double* t_start, const double* t_end, int b0,
             int nb, unsigned long long* next) {
  __shared__ double scw[ADJ_THREADS / 32][36];  // the segment's (y, c1, c2, c3) x 9
  const int lane = threadIdx.x & 31;
  double* cw = scw[threadIdx.x >> 5];
  const int mp = lane >> 2, mk = lane & 3;
  const long long nseg = (long long)S.L - 1;
  const long long total = (long long)nb * S.M * nseg;
  for (long long wid = claim_item(next, lane); wid < total; wid = claim_item(next, lane)) {
    const int bl = (int)(wid / (S.M * nseg));
    const int m = (int)((wid / nseg) % S.M);
    const int s = (int)(wid % nseg);
    const int b = b0 + bl;
    const size_t row = (size_t)b * S.M + m;
    const double* xs = S.x + row * S.L;
    const int st = start[b], n = len[b];
    int k0 = lower_bound_guess(data_freqs, N, xs[s]);
    int k1 = lower_bound_guess(data_freqs, N, xs[s + 1]);
    k0 = max(k0, st);
    k1 = min(k1, st + n);
    const double ts = t_start[b], te = t_end[b];
    __syncwarp();  // the previous item's coefficients are no longer read
    for (int i = lane; i < 36; i += 32) {
      const double* src = (i & 3) == 0 ? S.y : (i & 3) == 1 ? S.c1 : (i & 3) == 2 ? S.c2 : S.c3;
      cw[i] = src[(size_t)(i >> 2) * S.n + row * S.L + s];
    }
    __syncwarp();
    double mom[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) mom[i] = 0.0;
    const double xk = xs[s];
    for (int k = k0 + lane; k < k1; k += 32) {
      const double u = data_freqs[k] - xk;
      double q[9];
#pragma unroll
      for (int p = 0; p < 9; ++p)
        q[p] = cw[4 * p] + u * (cw[4 * p + 1] + u * (cw[4 * p + 2] + u * cw[4 * p + 3]));
      if (!tf_gate(q[2], ts, te)) continue;
      const cplx* g = gh + (off[bl] + (k - st)) * 3;
      double sn, cs;
      sincos_cw(q[1], &sn, &cs);
      const double er = cs, ei = sn;                  // e^{i phase}
      const double aer = q[0] * er, aei = q[0] * ei;  // A e^{i phase}
      double a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
      for (int ch = 0; ch < 3; ++ch) {
        const cplx u_ = g[ch];
        const double tr = q[3 + 2 * ch], ti = q[4 + 2 * ch];
        // dL = Re(u dW), W = T A e^{i phase}
        const double wr = tr * aer - ti * aei, wi = tr * aei + ti * aer;
        a[0] += u_.re * (tr * er - ti * ei) - u_.im * (tr * ei + ti * er);
        a[1] += -(u_.re * wi + u_.im * wr);
        a[2 + 2 * ch] = u_.re * aer - u_.im * aei;
        a[3 + 2 * ch] = -(u_.re * aei + u_.im * aer);
      }
      const double u2 = u * u, u3 = u2 * u;
#pragma unroll
      for (int p = 0; p < 8; ++p) {
        mom[4 * p] += a[p];
        mom[4 * p + 1] = fma(a[p], u, mom[4 * p + 1]);
        mom[4 * p + 2] = fma(a[p], u2, mom[4 * p + 2]);
        mom[4 * p + 3] = fma(a[p], u3, mom[4 * p + 3]);
      }
    }
    const double acc = warp_transpose_sum32(mom, lane);
    const int slot = (mp == 0) ? 0 : (mp == 1 ? 1 : mp + 1);  // skip t(f), slot 2
    const size_t i = (size_t)slot * S.n + row * S.L + s;
    double* dst = (mk == 0) ? ybd : (mk == 1) ? cb1 : (mk == 2) ? cb2 : cb3;
    dst[i] = acc;
  }
}

// d lnL / d m_j (j in [0, L-2]) of one row of the spline build: through c2, c3 (the t path)
// and through the right-hand sides r(m) of the slope system (lam = K^{-T} s_bar).
__device__ __forceinline__ double spline_mbar(int j, const double* xs, int L, const double* lam,
                                              const double* cb2, const double* cb3) {
  const double h = xs[j + 1] - xs[j];
  const double tbar = -cb2[j] + cb3[j] / h;
  double v = (cb2[j] - 2.0 * tbar) / h;
  // interior rows r = 1..L-2: r_r = 3 (h_r m_{r-1} + h_{r-1} m_r)
  if (j >= 1 && j <= L - 2) v += 3.0 * lam[j] * (xs[j] - xs[j - 1]);
  if (j + 1 <= L - 2) v += 3.0 * lam[j + 1] * (xs[j + 2] - xs[j + 1]);
  // row 0: r_0 = ((h0 + 2 d0) h1 m_0 + h0^2 m_1) / d0
  const double h0 = xs[1] - xs[0], h1 = xs[2] - xs[1], d0 = xs[2] - xs[0];
  if (j == 0) v += lam[0] * (h0 + 2 * d0) * h1 / d0;
  if (j == 1) v += lam[0] * h0 * h0 / d0;
  // row L-1: r = (h_{L-2}^2 m_{L-3} + (2 dL + h_{L-2}) h_{L-3} m_{L-2}) / dL
  const double hl = xs[L - 1] - xs[L - 2], hp = xs[L - 2] - xs[L - 3];
  const double dL = xs[L - 1] - xs[L - 3];
  if (j == L - 3) v += lam[L - 1] * hl * hl / dL;
  if (j == L - 2) v += lam[L - 1] * (2 * dL + hl) * hp / dL;
  return v;
}

// 3. Adjoint of the not-a-knot spline build of k_spline (spline.cu) for the 9 rows of one
// (binary, mode): inputs ybd, cb1..cb3 (entries s < L-1), outputs ybar (d lnL / d y, x held
// fixed) and xbar (d lnL / d x at the knots, y held fixed, summed over the rows).
// Forward: h_i = x_{i+1} - x_i, m_i = (y_{i+1} - y_i) / h_i; K(h) s = r(h, m); c1 = s_i,
// t = (s_i + s_{i+1} - 2 m_i) / h_i, c2 = (m_i - s_i) / h_i - t, c3 = t / h_i; a data bin f of
// segment i reads y_i + c1 u + c2 u^2 + c3 u^3 with u = f - x_i.  Shared memory: x, a, b, c,
// d[9][L].
__global__ void k_spline_adj(double* ybar, double* xbar, const double* ybd, const double* cb1,
                             const double* cb2, const double* cb3, SplineRefs S, int b0, int nb) {
  extern __shared__ double sm[];
  const int L = S.L;
  double* xs = sm;
  double* a = xs + L;
  double* bb = a + L;
  double* c = bb + L;
  double* d = c + L;
  const int nsys = nb * S.M;
  for (int sys = blockIdx.x; sys < nsys; sys += gridDim.x) {
    const size_t row = (size_t)b0 * S.M + sys;
    for (int i = threadIdx.x; i < L; i += blockDim.x) xs[i] = S.x[row * L + i];
    __syncthreads();
    // transposed matrix of the forward rows: a'_i = c_{i-1}, b'_i = b_i, c'_i = a_{i+1}
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
      auto fwd = [&](int r, double* fa, double* fb, double* fc) {
        if (r == 0) {
          *fa = 0.0; *fb = xs[2] - xs[1]; *fc = xs[2] - xs[0];
        } else if (r == L - 1) {
          *fa = xs[L - 1] - xs[L - 3]; *fb = xs[L - 2] - xs[L - 3]; *fc = 0.0;
        } else {
          *fa = xs[r + 1] - xs[r]; *fb = 2 * ((xs[r] - xs[r - 1]) + (xs[r + 1] - xs[r]));
          *fc = xs[r] - xs[r - 1];
        }
      };
      double ta, tb, tc, pa, pb, pc, na, nb_, nc;
      fwd(i, &ta, &tb, &tc);
      if (i > 0) fwd(i - 1, &pa, &pb, &pc); else pc = 0.0;
      if (i < L - 1) fwd(i + 1, &na, &nb_, &nc); else na = 0.0;
      a[i] = (i > 0) ? pc : 0.0;
      bb[i] = tb;
      c[i] = (i < L - 1) ? na : 0.0;
      // right-hand sides: s_bar from the coefficient adjoints
      for (int p = 0; p < 9; ++p) {
        double sb = 0.0;
        if (p != 2) {
          const size_t o = (size_t)p * S.n + row * L;
          if (i < L - 1) {
            const double h = xs[i + 1] - xs[i];
            const double tbar = -cb2[o + i] + cb3[o + i] / h;
            sb += cb1[o + i] - cb2[o + i] / h + tbar / h;
          }
          if (i > 0) {
            const double h = xs[i] - xs[i - 1];
            const double tbar = -cb2[o + i - 1] + cb3[o + i - 1] / h;
            sb += tbar / h;
          }
        }
        d[(size_t)p * L + i] = sb;
      }
    }
    __syncthreads();
    cr_solve(a, bb, c, d, L, 9, L);  // lambda = K^{-T} s_bar (r_bar)
    // y_bar from m_bar
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
      for (int p = 0; p < 9; ++p) {
        const size_t o = (size_t)p * S.n + row * L;
        if (p == 2) {
          ybar[o + i] = 0.0;
          continue;
        }
        const double* lam = d + (size_t)p * L;
        double yb = (i < L - 1) ? ybd[o + i] : 0.0;
        if (i < L - 1) yb -= spline_mbar(i, xs, L, lam, cb2 + o, cb3 + o) / (xs[i + 1] - xs[i]);
        if (i > 0) yb += spline_mbar(i - 1, xs, L, lam, cb2 + o, cb3 + o) / (xs[i] - xs[i - 1]);
        ybar[o + i] = yb;
      }
    }
    // x_bar.  Per segment i: e_i = d lnL / d u-shift (evaluation, u = f - x_i) and
    // hb_i = d lnL / d h_i (coefficients c2, c3 explicitly, m_i = (y_{i+1} - y_i) / h_i, and
    // the rows of K(h) s = r(h, m): lam^T (dr/dh - dK/dh s)); then
    // x_bar_i = -e_i - hb_i + hb_{i-1}.  The slopes are s_j = c1_j (j < L-1) and
    // s_{L-1} = c3_{L-2} h^2 - s_{L-2} + 2 m_{L-2}.  a[] and bb[] are free after the solve.
    for (int i = threadIdx.x; i < L - 1; i += blockDim.x) {
      double e = 0.0, hb = 0.0;
      for (int p = 0; p < 9; ++p) {
        if (p == 2) continue;
        const size_t o = (size_t)p * S.n + row * L;
        const double* lam = d + (size_t)p * L;
        const double* y = S.y + o;
        const double* s1 = S.c1 + o;
        auto hh = [&](int j) { return xs[j + 1] - xs[j]; };
        auto mm = [&](int j) { return (y[j + 1] - y[j]) / hh(j); };
        auto sl = [&](int j) {
          if (j < L - 1) return s1[j];
          const double h = hh(L - 2);
          return S.c3[o + L - 2] * h * h - s1[L - 2] + 2.0 * mm(L - 2);
        };
        const double h = hh(i);
        const double c2i = S.c2[o + i], c3i = S.c3[o + i];
        e += s1[i] * ybd[o + i] + 2.0 * c2i * cb1[o + i] + 3.0 * c3i * cb2[o + i];
        hb -= (cb2[o + i] * c2i + 2.0 * cb3[o + i] * c3i) / h;
        hb -= spline_mbar(i, xs, L, lam, cb2 + o, cb3 + o) * mm(i) / h;
        if (i >= 1 && i <= L - 2) hb += lam[i] * (3.0 * mm(i - 1) - sl(i - 1) - 2.0 * sl(i));
        if (i <= L - 3) hb += lam[i + 1] * (3.0 * mm(i + 1) - 2.0 * sl(i + 1) - sl(i + 2));
        if (i <= 1) {  // row 0: h1 s0 + d0 s1 = ((3 h0 + 2 h1) h1 m0 + h0^2 m1) / d0
          const double h0 = hh(0), h1 = hh(1), d0 = h0 + h1;
          const double rhs = ((3.0 * h0 + 2.0 * h1) * h1 * mm(0) + h0 * h0 * mm(1)) / d0;
          if (i == 0) hb += lam[0] * ((3.0 * h1 * mm(0) + 2.0 * h0 * mm(1) - rhs) / d0 - sl(1));
          else hb += lam[0] * (((3.0 * h0 + 4.0 * h1) * mm(0) - rhs) / d0 - sl(0) - sl(1));
        }
        if (i >= L - 3) {  // row L-1: dL s_{L-2} + A s_{L-1} = (Bh^2 m_{L-3} + (2A + 3Bh) A m_{L-2}) / dL
          const double A = hh(L - 3), Bh = hh(L - 2), dL = A + Bh;
          const double mq = mm(L - 3), mr = mm(L - 2);
          const double rhs = (Bh * Bh * mq + (2.0 * A + 3.0 * Bh) * A * mr) / dL;
          if (i == L - 3) hb += lam[L - 1] * (((4.0 * A + 3.0 * Bh) * mr - rhs) / dL - sl(L - 2) - sl(L - 1));
          else hb += lam[L - 1] * ((2.0 * Bh * mq + 3.0 * A * mr - rhs) / dL - sl(L - 2));
        }
      }
      a[i] = e;
      bb[i] = hb;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
      double v = 0.0;
      if (i < L - 1) v -= a[i] + bb[i];
      if (i > 0) v += bb[i - 1];
      xbar[row * L + i] = v;
    }
    __syncthreads();
  }
}

// 4a. Knot motion of the observation-window regrid (forward: k_tf_window, phenomhm.cu; the
// reference's phenomhm.py:520-610).  Row (b, m) has knots x_k = flo^(1 - r_k) fhi^(r_k),
// r_k = k / (L - 1), between band edges that are either the default grid's end points (which
// scale as 1 / (m1 + m2)) or where the linear interpolation of t(f) over the default grid
// crosses 0 (lower edge) or the SSB observation span To = tSSB(t_end) - tSSB(t_start) (upper
// edge).  t(f) at a default-grid point moves with the intrinsic parameters, t_ref and the
// point's own frequency; To moves with lam and beta.  One thread per (local binary, mode)
// repeats the forward's crossing search on the forward's default grid f0 and its t(f) tf0
// ([B, M, L] each), evaluates the straddling points as duals and writes
// wreg[row][0][k] = d flo / flo and wreg[row][1][k] = d fhi / fhi for the pass's directions.
__global__ void k_regrid_tangents(double* wreg, const ModeCoeffsT<GD>* coeffs, const double* P,
                                  int B, int b0, int nb, int M, int L, const double* f0,
                                  const double* tf0, const double* t_start, const double* t_end,
                                  double tL_start, double tL_end, int k0) {
  const long long n = (long long)nb * M;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int bl = (int)(t / M), m = (int)(t % M);
    const int b = b0 + bl;
    const size_t row = ((size_t)b * M + m) * L;
    const double* f = f0 + row;
    const double* x = tf0 + row;
    const ModeCoeffsT<GD>& c = coeffs[t];
    const GD msum = seed(P[0 * (size_t)B + b], 0, k0) + seed(P[1 * (size_t)B + b], 1, k0);
    const GD t_ref = seed(P[11 * (size_t)B + b], 10, k0);
    // default-grid point j: f_j proportional to 1 / (m1 + m2)
    auto fdual = [&](int j) {
      GD r(f[j]);
#pragma unroll
      for (int k = 0; k < GRAD_CHUNK; ++k) r.d[k] = -f[j] / msum.v * msum.d[k];
      return r;
    };
    // t(f_j) + t_ref along the moving point (value: the forward's)
    auto tdual = [&](int j) {
      const GD fj = fdual(j);
      GD ph, tf;
      mode_phase_tf(c, fj * c.M_sec, &ph, &tf);
      GD r = tf + t_ref;
      r.v = x[j];
      return r;
    };
    // f where the chord of t(f) over [f_s, f_s+1] reaches T
    auto cross = [&](int s, const GD& T) {
      const GD fa = fdual(s), fb = fdual(s + 1), ta = tdual(s), tb = tdual(s + 1);
      return (fb - fa) / (tb - ta) * (T - ta) + fa;
    };
    double tmin = x[0], tmax = x[0];
    for (int i = 1; i < L; ++i) {
      tmin = fmin(tmin, x[i]);
      tmax = fmax(tmax, x[i]);
    }
    GD flo = fdual(0), fhi = fdual(L - 1);
    if (tmin < 0.0) {
      int cnt = 0, seg = -1;
      for (int i = 0; i < L - 1; ++i)
        if ((0.0 < x[i + 1]) && (0.0 > x[i])) {
          if (cnt == 0) seg = i;
          ++cnt;
        }
      if (cnt == 1) flo = cross(seg, GD(0.0));
    }
    const GD lam = seed(P[8 * (size_t)B + b], 7, k0), beta = seed(P[9 * (size_t)B + b], 8, k0);
    GD To = tssb_from_l(tL_end, lam, beta, 0.0) - tssb_from_l(tL_start, lam, beta, 0.0);
    To.v = t_end[b] - t_start[b];  // the forward's span
    if (tmax > To.v) {
      int cnt = 0, seg = -1;
      for (int i = 0; i < L - 1; ++i)
        if ((To.v < x[i + 1]) && (To.v > x[i])) {
          if (cnt == 0) seg = i;
          ++cnt;
        }
      if (cnt == 1) fhi = cross(seg, To);
    }
    double* w = wreg + (size_t)t * 2 * GRAD_CHUNK;
#pragma unroll
    for (int k = 0; k < GRAD_CHUNK; ++k) {
      w[k] = flo.d[k] / flo.v;
      w[GRAD_CHUNK + k] = fhi.d[k] / fhi.v;
    }
  }
}

}  // namespace bbhx

using namespace bbhx;

namespace {
constexpr long long kGhBudget = 1ll << 29;  // complex entries of d lnL / d h per batch (8 GB)
constexpr int kDirectGradChunk = 512;
}  // namespace

extern "C" {

// d lnL / d theta [B, 11] of the direct likelihood (no reference counterpart).  Inputs are
// the forward path's sparse buffer y and its spline coefficients c1..c3 ([9, B, M, L]), the
// knots x [B, M, L], the noise-weighted data [3, N] (complex128) and noise weights [3, N],
// params [12, B] (device) and the QNM table for the dual-number setup.  The knots' own motion
// (the observation-window regrid) is differentiated from the forward's default grid f_default
// and its t(f) tf_default ([B, M, L], t_ref included) and the L-frame observation limits
// t_obs_start_L, t_obs_end_L [s]; with f_default or tf_default null the knots are held fixed.
// The host reads the support lengths once (one synchronisation).
int bbhx_direct_like_grad(void* orbits, void* d_h, void* h_h, double* grad, const double* params,
                          const int* ells,
                          const int* mms, const double* qnm_table, int qnm_n, double dspin,
                          double t_init, const double* data_freqs, const void* data,
                          const double* noise, int data_length, const double* x, const double* y,
                          const double* c1, const double* c2, const double* c3,
                          const double* t_start, const double* t_end, const double* f_default,
                          const double* tf_default, double t_obs_start_L, double t_obs_end_L,
                          int TDItag, int rescaled, int tdi2, int run_phenomd, int num_modes,
                          int length, int num_bin_all, void* stream) {
  BBHX_REQUIRE(orbits && ((OrbitHandle*)orbits)->ready, "orbit information not added");
  BBHX_REQUIRE(TDItag == 1 || TDItag == 2, "TDItag must be 1 (XYZ) or 2 (AET)");
  BBHX_REQUIRE(num_modes > 0 && num_modes <= MAX_MODES, "num_modes must be 1..6");
  BBHX_REQUIRE(length >= 4 && length <= 2048, "gradient spline length must be 4..2048");
  BBHX_REQUIRE(qnm_n >= 2 && dspin > 0.0, "bad QNM table");
  if (num_bin_all == 0) return OK;
  cudaStream_t s = (cudaStream_t)stream;
  const int B = num_bin_all, M = num_modes, L = length;
  SplineRefs S{x, y, c1, c2, c3, (size_t)B * M * L, M, L};
  int *start = nullptr, *len = nullptr;
  int st = OK;
  BBHX_CHECK_CUDA(pool_alloc((void**)&start, sizeof(int) * 2 * (size_t)B, s));
  len = start + B;
  st = bbhx_template_support(start, len, x, M, L, B, data_freqs, data_length, stream);
  std::vector<int> hlen(B);
  if (!st) {
    if (cudaMemcpyAsync(hlen.data(), len, sizeof(int) * B, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      set_error("reading the template supports failed");
      st = ERR_CUDA;
    }
  }
  // adjoint arrays over all binaries, dual records and d lnL / d h per batch
  const size_t nall = (size_t)9 * B * M * L;
  const bool moving = f_default != nullptr && tf_default != nullptr;
  double *ybd = nullptr, *cb = nullptr, *ybar = nullptr, *xbar = nullptr, *wreg = nullptr;
  ModeCoeffsT<GD>* cD = nullptr;
  ResponseModeT<GD>* rD = nullptr;
  const int chunk = std::min(B, kDirectGradChunk);
  if (!st) {
    const size_t nscratch = nall * 5 + (size_t)B * M * L + (size_t)chunk * M * 2 * GRAD_CHUNK;
    // + one 8-byte word after the arrays: the work-queue counter of k_adj_coeffs
    if (pool_alloc((void**)&ybd, sizeof(double) * (nscratch + 1), s) != cudaSuccess ||
        pool_alloc((void**)&cD, sizeof(ModeCoeffsT<GD>) * (size_t)chunk * M, s) != cudaSuccess ||
        pool_alloc((void**)&rD, sizeof(ResponseModeT<GD>) * (size_t)chunk * M, s) != cudaSuccess) {
      set_error("device allocation of the gradient scratch failed");
      st = ERR_CUDA;
    }
  }
  if (!st) {
    cb = ybd + nall;  // cb1, cb2, cb3
    ybar = cb + 3 * nall;
    xbar = ybar + nall;
    wreg = xbar + (size_t)B * M * L;
    // ybd / cb rows not written by k_adj_coeffs stay zero; wreg is zero for fixed knots
    if (cudaMemsetAsync(ybd, 0, sizeof(double) * nall * 4, s) != cudaSuccess ||
        cudaMemsetAsync(wreg, 0, sizeof(double) * (size_t)chunk * M * 2 * GRAD_CHUNK, s) != cudaSuccess) {
      set_error("cudaMemsetAsync failed");
      st = ERR_CUDA;
    }
  }
  const int nsm = sm_count();
  const size_t smem = sizeof(double) * (size_t)(4 + 9) * L;
  if (!st && cudaFuncSetAttribute(k_spline_adj, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem) != cudaSuccess) {
    set_error("cudaFuncSetAttribute failed for k_spline_adj");
    st = ERR_CUDA;
  }
  for (int b0 = 0; !st && b0 < B;) {
    // batch: at most `chunk` binaries and kGhBudget complex entries of d lnL / d h
    std::vector<long long> hoff;
    long long tot = 0;
    int nb = 0;
    while (b0 + nb < B && nb < chunk && (nb == 0 || tot + 3ll * hlen[b0 + nb] <= kGhBudget)) {
      hoff.push_back(tot / 3);
      tot += 3ll * hlen[b0 + nb];
      ++nb;
    }
    long long* off = nullptr;
    cplx* gh = nullptr;
    if (pool_alloc((void**)&off, sizeof(long long) * nb, s) != cudaSuccess ||
        pool_alloc((void**)&gh, sizeof(cplx) * std::max(tot, 3ll), s) != cudaSuccess) {
      set_error("device allocation of d lnL / d h failed");
      st = ERR_CUDA;
    }
    if (!st && cudaMemcpyAsync(off, hoff.data(), sizeof(long long) * nb, cudaMemcpyHostToDevice,
                               s) != cudaSuccess) {
      set_error("copy of the support offsets failed");
      st = ERR_CUDA;
    }
    if (!st)  // d lnL / d h by the FP64 fused likelihood kernel (staged segments, tile-major)
      st = direct_fused_gh(gh, off, (double*)d_h, (double*)h_h, start, len, data_freqs,
                           (const double*)data, noise, data_length, x, y, c1, c2, c3, t_start,
                           t_end, M, L, B, b0, nb, s);
    if (!st) {
      const long long warps = (long long)nb * M * (L - 1);
      unsigned long long* next = reinterpret_cast<unsigned long long*>(
          ybd + nall * 5 + (size_t)B * M * L + (size_t)chunk * M * 2 * GRAD_CHUNK);
      st = cuda_status(cudaMemsetAsync(next, 0, sizeof(unsigned long long), s),
                       "work-queue counter");
      // resident CTAs only: every warp claims segments until the queue drains (a segment holds
      // from zero to ~10^4 data bins)
      int per_sm = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_adj_coeffs, ADJ_THREADS, 0) !=
              cudaSuccess ||
          per_sm < 1) {
        (void)cudaGetLastError();
        per_sm = 1;
      }
      const unsigned grid =
          (unsigned)std::min<long long>((warps + 7) / 8, (long long)nsm * per_sm);
      if (!st) {
        k_adj_coeffs<<<grid, ADJ_THREADS, 0, s>>>(ybd, cb, cb + nall, cb + 2 * nall, gh, off,
                                                  start, len, S, data_freqs, data_length, t_start,
                                                  t_end, b0, nb, next);
        st = launch_status("k_adj_coeffs");
      }
    }
    if (!st) {
      k_spline_adj<<<(unsigned)std::min(nb * M, nsm * 4), 256, smem, s>>>(
          ybar, xbar, ybd, cb, cb + nall, cb + 2 * nall, S, b0, nb);
      st = launch_status("k_spline_adj");
    }
    for (int k0 = 0; !st && k0 < NGRAD; k0 += GRAD_CHUNK) {
      k_grad_setup<<<grid_for((long long)nb * M, 64), 64, 0, s>>>(cD, rD, params, B, b0, nb, ells,
                                                                  mms, M, qnm_table, qnm_n, dspin,
                                                                  run_phenomd, k0);
      st = launch_status("k_grad_setup");
      if (st) break;
      if (moving) {
        k_regrid_tangents<<<grid_for((long long)nb * M, 64), 64, 0, s>>>(
            wreg, cD, params, B, b0, nb, M, L, f_default, tf_default, t_start, t_end,
            t_obs_start_L, t_obs_end_L, k0);
        st = launch_status("k_regrid_tangents");
        if (st) break;
      }
      k_contract_direct<<<(unsigned)std::min(nb, nsm * 8), 128, 0, s>>>(
          grad, cD, rD, ((OrbitHandle*)orbits)->tab, params, B, b0, nb, t_init, x, ybar, xbar,
          wreg, TDItag, rescaled, tdi2, M, L, k0);
      st = launch_status("k_contract_direct");
    }
    if (gh) pool_free(gh, s);
    if (off) pool_free(off, s);
    b0 += nb;
  }
  if (rD) pool_free(rD, s);
  if (cD) pool_free(cD, s);
  if (ybd) pool_free(ybd, s);
  if (start) pool_free(start, s);
  return st;
}

}  // extern "C"
