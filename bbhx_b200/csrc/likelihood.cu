// Likelihood kernels.
//
// Reference interfaces replaced (src/bbhx/cutils/Likelihood.hh:6-13):
//   direct_like (Likelihood.cu:356-471): noise-weight each stored template in place, then
//               6 cuBLAS Zdotc per binary, each followed by a stream sync; results
//               accumulated into HOST d_h / h_h.
//   hdyn        (Likelihood.cu:20-120 GPU form): relative-binning sums, one thread per binary.
// New (no reference counterpart, same result as InterpTDI + direct_like):
//   bbhx_direct_like_fused: evaluates the splines on the data grid, sums the modes,
//   noise-weights and reduces <d|h>, <h|h> without ever storing a template.
//
// Reductions are deterministic: per-(tile, binary) partials in FP64, then a fixed-order sum.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "capi_internal.cuh"
#include "het_item.cuh"
#include "spline_eval.cuh"

namespace bbhx {

// set by the reduce kernels when a <d|h> or <h|h> is not finite (read by bbhx_take_status)
static __device__ unsigned g_nonfinite_likelihood = 0;

int take_nonfinite_likelihood(cudaStream_t s, unsigned* any) {
  static const unsigned zero = 0;
  unsigned v = 0;
  BBHX_CHECK_CUDA(cudaMemcpyFromSymbolAsync(&v, g_nonfinite_likelihood, sizeof(v), 0,
                                            cudaMemcpyDeviceToHost, s));
  BBHX_CHECK_CUDA(cudaMemcpyToSymbolAsync(g_nonfinite_likelihood, &zero, sizeof(zero), 0,
                                          cudaMemcpyHostToDevice, s));
  BBHX_CHECK_CUDA(cudaStreamSynchronize(s));
  *any |= v;
  return OK;
}

// ---------------------------------------------------------------------------- direct_like
struct DirectJob {
  cplx* tmpl;
  int start, len;
  long long part0;  // first partial slot of this binary
  int nparts;
};

constexpr int DL_CHUNK = 2048;

__global__ void k_direct_like_partials(const DirectJob* jobs, const cplx* __restrict__ data,
                                       const double* __restrict__ noise, int N, double* partials) {
  const int b = blockIdx.y;
  const DirectJob J = jobs[b];
  __shared__ double red[3][32];
  for (int part = blockIdx.x; part < J.nparts; part += gridDim.x) {
    int i0 = part * DL_CHUNK;
    int i1 = min(i0 + DL_CHUNK, J.len);
    double dr = 0, di = 0, hh = 0;
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
      for (int ch = 0; ch < 3; ++ch) {
        long long gi = (long long)ch * N + J.start + i;
        double w = noise[gi];
        cplx h = J.tmpl[(long long)ch * J.len + i] * w;  // weighted in place (reference side effect)
        J.tmpl[(long long)ch * J.len + i] = h;
        cplx d = data[gi];
        dr += d.re * h.re + d.im * h.im;  // conj(d) * h
        di += d.re * h.im - d.im * h.re;
        hh += h.re * h.re + h.im * h.im;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      dr += __shfl_xor_sync(0xffffffffu, dr, o);
      di += __shfl_xor_sync(0xffffffffu, di, o);
      hh += __shfl_xor_sync(0xffffffffu, hh, o);
    }
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
      red[0][w] = dr;
      red[1][w] = di;
      red[2][w] = hh;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0, bb = 0, c = 0;
      for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
        a += red[0][k];
        bb += red[1][k];
        c += red[2][k];
      }
      double* P = partials + 3 * (J.part0 + part);
      P[0] = a;
      P[1] = bb;
      P[2] = c;
    }
    __syncthreads();
  }
}

__global__ void k_sum_partials(const DirectJob* jobs, const double* partials, double* out, int B) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B; b += gridDim.x * blockDim.x) {
    double a = 0, c = 0, h = 0;
    for (int p = 0; p < jobs[b].nparts; ++p) {
      const double* P = partials + 3 * (jobs[b].part0 + p);
      a += P[0];
      c += P[1];
      h += P[2];
    }
    out[4 * b + 0] = 4.0 * a;
    out[4 * b + 1] = 4.0 * c;
    out[4 * b + 2] = 4.0 * h;
    out[4 * b + 3] = 0.0;
  }
}

// ---------------------------------------------------------------------------- hdyn
// residuals r[(j*3 + ch)*B + b], constants [(k*3 + ch)*L + j] (k = A0, A1, B0, B1)
__global__ void k_hdyn(cplx* d_h, cplx* h_h, const cplx* __restrict__ r,
                       const cplx* __restrict__ K, const double* __restrict__ f, int B, int L,
                       int nch) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B; b += gridDim.x * blockDim.x) {
    cplx dh = mk(0, 0);
    double hh_re = 0.0, hh_im = 0.0;
    for (int ch = 0; ch < nch; ++ch) {
      cplx prev = r[((long long)0 * nch + ch) * B + b];
      double fprev = f[0];
      for (int j = 1; j < L; ++j) {
        cplx cur = r[((long long)j * nch + ch) * B + b];
        double fj = f[j];
        if (fprev != 0.0) {
          double df = fj - fprev;
          cplx r1 = mk((cur.re - prev.re) / df, (cur.im - prev.im) / df);
          double fmid = (fj + fprev) / 2.0;
          cplx r0 = cur - r1 * (fj - fmid);
          cplx A0 = K[((long long)0 * nch + ch) * L + j];
          cplx A1 = K[((long long)1 * nch + ch) * L + j];
          cplx B0 = K[((long long)2 * nch + ch) * L + j];
          cplx B1 = K[((long long)3 * nch + ch) * L + j];
          dh = dh + A0 * conj(r0) + A1 * conj(r1);
          double mag2 = r0.re * r0.re + r0.im * r0.im;
          double re01 = r0.re * r1.re + r0.im * r1.im;  // Re(r0 conj(r1))
          hh_re += B0.re * mag2 + 2.0 * B1.re * re01;
          hh_im += B0.im * mag2 + 2.0 * B1.im * re01;
        }
        prev = cur;
        fprev = fj;
      }
    }
    d_h[b] = dh;
    h_h[b] = mk(hh_re, hh_im);
    note_nonfinite(&g_nonfinite_likelihood, dh.re, dh.im, hh_re, hh_im);
  }
}

// ---------------------------------------------------------------------------- fused direct
// Support of each binary on the data grid (waveformbuild.py:136-177): [start, start+len) with
// start = searchsorted(f, min x, 'right'), end = searchsorted(f, max x, 'right').
// Support [start, start + len) on the data grid of binary b (whole block): the data bins in
// [min x, max x] of its knots over all modes (searchsorted right of both ends).
__device__ __forceinline__ void support_of(const double* __restrict__ x, int M, int L, int b,
                                           const double* __restrict__ data_freqs, int N,
                                           int* start, int* len) {
  double lo = 1e300, hi = -1e300;
  for (int t = threadIdx.x; t < M * L; t += blockDim.x) {
    double v = x[(long long)b * M * L + t];
    lo = fmin(lo, v);
    hi = fmax(hi, v);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  __shared__ double slo[32], shi[32];
  int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    slo[w] = lo;
    shi[w] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
      lo = fmin(lo, slo[k]);
      hi = fmax(hi, shi[k]);
    }
    // searchsorted right: number of entries <= v
    int a = 0, c = N;
    while (a < c) {
      int mid = (a + c) >> 1;
      if (data_freqs[mid] <= lo) a = mid + 1; else c = mid;
    }
    int s = a;
    a = s;
    c = N;
    while (a < c) {
      int mid = (a + c) >> 1;
      if (data_freqs[mid] <= hi) a = mid + 1; else c = mid;
    }
    start[b] = s;
    len[b] = a - s;
  }
  __syncthreads();
}

__global__ void k_support(const double* __restrict__ x, int M, int L, int B,
                          const double* __restrict__ data_freqs, int N, int* start, int* len) {
  support_of(x, M, L, blockIdx.x, data_freqs, N, start, len);
}

constexpr int FD_WARPS = 4;
constexpr int FD_K = 4;                          // bins per lane per warp chunk
constexpr int FD_WARP_BINS = 32 * FD_K;          // 128
// data bins per (tile, binary) work item of the single-group kernel: large tiles spread the
// per-item staging, segment table and gate classification over more bins (B = 1024 benchmark:
// 512 -> 104 ms, 1024 -> 88, 2048 -> 80, 4096 -> 78, 8192 -> 79 ms mixed)
constexpr int FD_TILE = 4096;
// spline segments per (tile, mode) staged in shared memory: 8 for the mixed form, 4 for the
// FP64 form, whose slices (FP64 coefficients plus the phase-recurrence state) must stay small
// enough for 3 CTAs per SM
template <typename R>
constexpr int fd_nseg() { return sizeof(R) == 8 ? 4 : 8; }
constexpr int FD_MAXM = 6;    // modes per binary
constexpr int FD_NC = 36;     // 9 quantities x (y, c1, c2, c3) per segment
constexpr int FD_MAXCHUNK = 32;  // 128-bin chunks per tile item (tiles of up to 4096 bins)

struct FusedArgs {
  const double* data_freqs;
  const cplx* data;     // [3, N] noise-weighted data
  const double* noise;  // [3, N] sqrt(df / S)
  int N;
  const double* x;  // [B, M, L]
  const double* y;  // [9, B, M, L]
  const double* c1;
  const double* c2;
  const double* c3;
  const double* t_start;
  const double* t_end;
  const int* sup_start;
  const int* sup_len;
  int B, M, L;
  int ntiles;
  int tile;            // data bins per tile item (multiple of FD_WARP_BINS)
  double* partials;    // [ntiles * B][3]
  const int2* segtab;  // [ntiles][B][M]: segments of the tile's first and last bin
  double* d_h;         // [B] complex outputs
  double* h_h;
  const float2* data32;  // optional FP32 copies of data / noise for the mixed form (or null)
  const float* noise32;
  long long qstride;     // distance between the 9 quantities in y, c1..c3 (B M L of those arrays)
  // optional, FP64 form (gradient chain): d lnL / d h = 4 w (d~ - w h) of every support bin,
  // written at gh[3 (gh_off[b] + i - sup_start[b]) + channel]; null in the likelihood calls
  cplx* gh;
  const long long* gh_off;
  // uniform-grid record of data_freqs (k_grid_detect) enabling the phase recurrence, or null
  const struct GridInfo* grid;
  // work-queue counter, zero at launch: warps claim (tile, binary) items from it in increasing
  // order (claim_item)
  unsigned long long* next;
};

// Data grid of the form f_i = fl((k0 + i) df): numpy's k * df and rfftfreq grids, the form
// BBHx's data streams take.  k_grid_detect verifies the form bit-exactly on the device for
// three candidates of df (the rounded f[N-1] / (k0 + N - 1) and its two neighbours); bit c of
// ok says candidate c reproduces every f_i.  The fused kernel then knows every bin's exact
// frequency k df (as p + pe, an error-free product), which the phase recurrence needs.
struct GridInfo {
  double k0;
  double df[3];
  unsigned ok;
  unsigned pad;
};

// Uniform-grid check of f[0..N) by block bx of nb: every bin against the three candidate
// spacings; block 0 also records k0 and the candidates.
__device__ __forceinline__ void grid_detect_part(const double* __restrict__ f, int N, GridInfo* g,
                                                 long long bx, long long nb) {
  unsigned ok = 0;
  double k0 = 0.0, cand[3] = {0.0, 0.0, 0.0};
  if (N >= 2) {
    const double f0 = f[0], f1 = f[N - 1];
    const double dfa = (f1 - f0) / (double)(N - 1);
    k0 = rint(f0 / dfa);
    const double kN = k0 + (double)(N - 1);
    const double dc = f1 / kN;
    cand[0] = dc;
    cand[1] = nextafter(dc, 0.0);
    cand[2] = nextafter(dc, 1e300);
    ok = (f0 > 0.0 && dfa > 0.0 && k0 >= 1.0 && kN < 4.0e15) ? 7u : 0u;
    for (long long i = bx * blockDim.x + threadIdx.x; ok && i < N; i += nb * blockDim.x) {
      const double kd = k0 + (double)i;
      const double fi = f[i];
#pragma unroll
      for (int c = 0; c < 3; ++c)
        if (__dmul_rn(kd, cand[c]) != fi) ok &= ~(1u << c);
    }
  }
  ok = __reduce_and_sync(0xffffffffu, ok);
  if ((threadIdx.x & 31) == 0) atomicAnd(&g->ok, ok);
  if (bx == 0 && threadIdx.x == 0) {
    g->k0 = k0;
    g->df[0] = cand[0];
    g->df[1] = cand[1];
    g->df[2] = cand[2];
  }
}

__global__ void k_grid_detect(const double* __restrict__ f, int N, GridInfo* g) {
  grid_detect_part(f, N, g, blockIdx.x, gridDim.x);
}

// Launch the grid detection into g (device) on stream s.
inline int detect_grid(const double* f, int N, GridInfo* g, cudaStream_t s) {
  int st = cuda_status(cudaMemsetAsync(&g->ok, 0xff, sizeof(unsigned), s), "grid record init");
  if (st) return st;
  k_grid_detect<<<grid_for(N, 256, sm_count() * 8), 256, 0, s>>>(f, N, g);
  return launch_status("k_grid_detect");
}

// Segment table: for every (tile, binary, mode) the spline segments holding the first and the
// last data bin of the binary's support inside the tile (searchsorted(side='right') - 1 of
// their frequencies), or (1, 0) when the tile misses the support.  One thread per entry.
__device__ __forceinline__ int2 tile_segment_entry(long long t, const double* __restrict__ x,
                                                   const double* __restrict__ data_freqs,
                                                   const int* sup_start, const int* sup_len,
                                                   int B, int M, int L, int tile_bins) {
  const int m = (int)(t % M);
  const long long tb = t / M;
  const int b = (int)(tb % B);
  const int tile = (int)(tb / B);
  const int s0 = sup_start[b], s1 = s0 + sup_len[b];
  const int i0 = max(tile * tile_bins, s0), i1 = min((tile + 1) * tile_bins, s1) - 1;
  if (i0 > i1) return make_int2(1, 0);
  const double* xr = x + ((long long)b * M + m) * L;
  const double f0 = data_freqs[i0], f1 = data_freqs[i1];
  int lo = 0, hi = L;  // count of knots <= f0
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (xr[mid] <= f0) lo = mid + 1; else hi = mid;
  }
  const int ka = lo - 1;
  hi = L;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (xr[mid] <= f1) lo = mid + 1; else hi = mid;
  }
  return make_int2(ka, lo - 1);
}

__global__ void k_tile_segments(int2* tab, const double* __restrict__ x,
                                const double* __restrict__ data_freqs, const int* sup_start,
                                const int* sup_len, int B, int M, int L, int ntiles, int tile_bins) {
  const long long n = (long long)ntiles * B * M;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    tab[t] = tile_segment_entry(t, x, data_freqs, sup_start, sup_len, B, M, L, tile_bins);
}

// Cubic coefficients of one spline segment held by a lane: phase and t(f) always in FP64,
// amplitude and the six transfer components in R (FP32 when mixed).
template <typename R>
struct SegCoef {
  double xk;
  double py[2], p1[2], p2[2], p3[2];
  R ay[7], a1[7], a2[7], a3[7];
  // v(p, c) = coefficient c (y, c1, c2, c3) of quantity p (amp, phase, tf, T1re .. T3im)
  __device__ __forceinline__ void set(int p, double vy, double v1, double v2, double v3) {
    if (p == 1 || p == 2) {
      py[p - 1] = vy; p1[p - 1] = v1; p2[p - 1] = v2; p3[p - 1] = v3;
    } else {
      const int a = (p == 0) ? 0 : p - 2;
      ay[a] = (R)vy; a1[a] = (R)v1; a2[a] = (R)v2; a3[a] = (R)v3;
    }
  }
};

// Add conj(T_c A e^{i phi}) of one (bin, mode) to acc (6 reals: 3 complex channels), behind the
// t(f) gate.
template <bool MIXED, typename R>
__device__ __forceinline__ void accumulate_bin(const SegCoef<R>& c, double f, double ts, double te,
                                               R* acc) {
  const double u = f - c.xk;
  const double tf = fma(fma(fma(c.p3[1], u, c.p2[1]), u, c.p1[1]), u, c.py[1]);
  if (!tf_gate(tf, ts, te)) return;
  const double ph = fma(fma(fma(c.p3[0], u, c.p2[0]), u, c.p1[0]), u, c.py[0]);
  const R ur = (R)u;
  R v[7];
#pragma unroll
  for (int a = 0; a < 7; ++a) v[a] = fma(fma(fma(c.a3[a], ur, c.a2[a]), ur, c.a1[a]), ur, c.ay[a]);
  R sn, cs;
  if (MIXED) {
    float sf, cf;
    sincos_mixed(ph, &sf, &cf);
    sn = (R)sf;
    cs = (R)cf;
  } else {
    double sd, cd;
    sincos_cw(ph, &sd, &cd);
    sn = (R)sd;
    cs = (R)cd;
  }
  const R apr = v[0] * cs, api = v[0] * sn;
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) {
    const R tr = v[1 + 2 * ch], ti = v[2 + 2 * ch];
    acc[2 * ch] += tr * apr - ti * api;
    acc[2 * ch + 1] -= tr * api + ti * apr;
  }
}

// The FD_K bins of one lane inside one segment, branch-free so the bins' evaluation chains
// interleave (G at a time): bins with f < 0 (outside the support) or failing the per-bin t(f)
// gate (evaluated only when the segment straddles the window, CHECK) contribute zero.  The
// channel sums are FMA chains.
template <bool MIXED, typename R, int G, bool CHECK>
__device__ __forceinline__ void accumulate_chunk(const SegCoef<R>& c, const double* f, double ts,
                                                 double te, R (*acc)[6]) {
#pragma unroll
  for (int j0 = 0; j0 < FD_K; j0 += G) {
    double u[G], ph[G];
    bool g[G];
#pragma unroll
    for (int j = 0; j < G; ++j) {
      u[j] = f[j0 + j] - c.xk;
      g[j] = f[j0 + j] >= 0.0;
      if (CHECK) {
        const double tf = fma(fma(fma(c.p3[1], u[j], c.p2[1]), u[j], c.p1[1]), u[j], c.py[1]);
        g[j] = g[j] && tf_gate(tf, ts, te);
      }
      ph[j] = fma(fma(fma(c.p3[0], u[j], c.p2[0]), u[j], c.p1[0]), u[j], c.py[0]);
    }
#pragma unroll
    for (int j = 0; j < G; ++j) {
      const R ur = (R)u[j];
      R v[7];
#pragma unroll
      for (int a = 0; a < 7; ++a) v[a] = fma(fma(fma(c.a3[a], ur, c.a2[a]), ur, c.a1[a]), ur, c.ay[a]);
      R sn, cs;
      if (MIXED) {
        float sf, cf;
        sincos_mixed(ph[j], &sf, &cf);
        sn = (R)sf;
        cs = (R)cf;
      } else {
        double sd, cd;
        sincos_cw(ph[j], &sd, &cd);
        sn = (R)sd;
        cs = (R)cd;
      }
      const R amp = g[j] ? v[0] : R(0);
      const R apr = amp * cs, api = amp * sn;
      R* a = acc[j0 + j];
#pragma unroll
      for (int ch = 0; ch < 3; ++ch) {  // a += conj(T A e^{i phi})
        const R tr = v[1 + 2 * ch], ti = v[2 + 2 * ch];
        a[2 * ch] = fma(tr, apr, a[2 * ch]);
        a[2 * ch] = fma(-ti, api, a[2 * ch]);
        a[2 * ch + 1] = fma(-tr, api, a[2 * ch + 1]);
        a[2 * ch + 1] = fma(-ti, apr, a[2 * ch + 1]);
      }
    }
  }
}

// Per-warp shared-memory copy of the spline segments one (tile, binary) item needs, for every
// mode: x of the segments' knots, the FP64 cubic coefficients of phase and t(f), and those of
// the amplitude and six transfer components in R (FP32 when mixed), each quantity's
// (y, c1, c2, c3) contiguous so a lane reloads a segment with vector loads.
template <typename R>
struct alignas(16) WarpStage {
  static constexpr int NSEG = fd_nseg<R>();
  double x[FD_MAXM][NSEG + 1];
  double pc[FD_MAXM][NSEG][2][4];
  R ac[FD_MAXM][NSEG][7][4];
  int klo[FD_MAXM];
  int nseg[FD_MAXM];
  // modes whose tile spans more than NSEG segments (nseg = -1, FP64 form): the segment of the
  // last chunk's first bin (a forward cursor) and the window of segments staged per chunk
  int kcur[FD_MAXM];
  int kst[FD_MAXM];
  int nst[FD_MAXM];
  int gate[FD_MAXM][NSEG];  // t(f) gate over the whole segment: 0 mixed, 1 all in, 2 all out
  signed char cseg[FD_MAXCHUNK][FD_MAXM];  // staged segment holding a whole 128-bin chunk, or -1
};

// ---------------------------------------------------------------- phase recurrence
// Inside one spline segment the phase is a cubic in the data-bin index, so along a lane's bins
// (stride h = 32 df on a uniform grid) e^{i phi} advances by complex rotations:
//   E_{j+1} = E_j R_j,  R_{j+1} = R_j Q_j,  Q_{j+1} = Q_j P,
// with R = e^{i Delta}, Q = e^{i Delta^2}, P = e^{i Delta^3} the first, second and (constant)
// third differences of the phase cubic.  Three FP64 complex products per bin replace the
// per-bin phase cubic, range reduction and polynomial sine / cosine.  The state is re-anchored
// (rot_anchor) at a mode's first chunk of a work item and wherever the chunk's segment changes;
// an item holds at most kRecChunks chunks, so no lane runs more than kRecChunks * FD_K steps
// from its anchor.  The anchor phase is
// evaluated at the bin's exact frequency k df (error-free product) with a compensated final sum,
// so it carries < 1e-13 rad instead of the ~ulp(phi) ~ 1e-10 - 1e-9 rad of a plain FP64
// evaluation, and the products add ~2e-11 rad over the kRecChunks * FD_K = 128 steps between
// anchors (bounded by the self-test against 50-digit phases: k_selftest_recurrence).
constexpr int kRecChunks = 32;  // chunks (of FD_K steps per lane) between anchors, at most
static_assert(FD_MAXCHUNK <= kRecChunks, "a work item must not run the recurrence longer");

struct Rot {
  double er, ei, rr, ri, qr, qi, pr, pi;
};

// a *= b (complex, FP64)
__device__ __forceinline__ void cmul_inplace(double& ar, double& ai, double br, double bi) {
  const double r = fma(ar, br, -ai * bi);
  const double i = fma(ar, bi, ai * br);
  ar = r;
  ai = i;
}

// Recurrence state at grid bin kd (exact integer k0 + i, as a double) of the segment whose
// phase cubic is pc = (y, c1, c2, c3) about knot xk; h = 32 df.
__device__ __forceinline__ void rot_anchor(Rot& z, const double* pc, double xk, double kd,
                                           double df, double h) {
  const double p = __dmul_rn(kd, df);     // the grid frequency f_i (bit-exact, see GridInfo)
  const double pe = fma(kd, df, -p);      // p + pe = kd * df exactly
  const double u = __dsub_rn(p, xk);      // exact: xk <= p < xk (1 + 1e-2) (Sterbenz)
  const double y = pc[0], c1 = pc[1], c2 = pc[2], c3 = pc[3];
  double t = u * fma(fma(c3, u, c2), u, c1);
  const double d1 = fma(fma(3.0 * c3, u, 2.0 * c2), u, c1);  // phase derivative at u
  t = fma(d1, pe, t);                     // first-order term of the low part of k df
  const double sh = __dadd_rn(y, t);      // y + t = sh + se exactly (TwoSum)
  const double bb = __dsub_rn(sh, y);
  const double se = __dadd_rn(__dsub_rn(y, __dsub_rn(sh, bb)), __dsub_rn(t, bb));
  sincos_cw(sh, &z.ei, &z.er, se);
  const double D1 = h * fma(c3, fma(3.0 * u, u + h, h * h), fma(c2, fma(2.0, u, h), c1));
  const double D2 = 2.0 * h * h * fma(3.0 * c3, u + h, c2);
  const double D3 = 6.0 * c3 * h * h * h;
  sincos_cw(D1, &z.ri, &z.rr);
  sincos_cw(D2, &z.qi, &z.qr);
  sincos_cw(D3, &z.pi, &z.pr);
}

// The FD_K bins of one lane inside staged segment ka of mode m, with the phase from the
// recurrence z (advanced past the last bin on return): conj(T A e^{i phi}) into acc; bins with
// f < 0 (outside the support) or failing the t(f) gate (CHECK) contribute zero.  The cubics
// are evaluated one quantity at a time for all FD_K bins, reading that quantity's four
// coefficients from shared memory, which keeps few coefficients and partial values live.
template <typename R, bool CHECK>
__device__ __forceinline__ void accumulate_chunk_rec(const WarpStage<R>& S, int m, int ka,
                                                     const double* f, double ts, double te,
                                                     R (*acc)[6], Rot& z) {
  const double xk = S.x[m][ka];
  double u[FD_K];
  bool g[FD_K];
#pragma unroll
  for (int j = 0; j < FD_K; ++j) {
    u[j] = f[j] - xk;
    g[j] = f[j] >= 0.0;
  }
  if (CHECK) {
    const double2 lo = *reinterpret_cast<const double2*>(&S.pc[m][ka][1][0]);
    const double2 hi = *reinterpret_cast<const double2*>(&S.pc[m][ka][1][2]);
#pragma unroll
    for (int j = 0; j < FD_K; ++j) {
      const double tf = fma(fma(fma(hi.y, u[j], hi.x), u[j], lo.y), u[j], lo.x);
      g[j] = g[j] && tf_gate(tf, ts, te);
    }
  }
  // e^{i phi} of the FD_K bins from the recurrence
  double er[FD_K], ei[FD_K];
#pragma unroll
  for (int j = 0; j < FD_K; ++j) {
    er[j] = z.er;
    ei[j] = z.ei;
    cmul_inplace(z.er, z.ei, z.rr, z.ri);
    cmul_inplace(z.rr, z.ri, z.qr, z.qi);
    cmul_inplace(z.qr, z.qi, z.pr, z.pi);
  }
  auto cubic4 = [&](int a, R* v) {
    R c[4];
    if (sizeof(R) == 4) {
      const float4 q = *reinterpret_cast<const float4*>(&S.ac[m][ka][a][0]);
      c[0] = (R)q.x; c[1] = (R)q.y; c[2] = (R)q.z; c[3] = (R)q.w;
    } else {
      const double2 lo = *reinterpret_cast<const double2*>(&S.ac[m][ka][a][0]);
      const double2 hi = *reinterpret_cast<const double2*>(&S.ac[m][ka][a][2]);
      c[0] = (R)lo.x; c[1] = (R)lo.y; c[2] = (R)hi.x; c[3] = (R)hi.y;
    }
#pragma unroll
    for (int j = 0; j < FD_K; ++j) {
      const R ur = (R)u[j];
      v[j] = fma(fma(fma(c[3], ur, c[2]), ur, c[1]), ur, c[0]);
    }
  };
  // A e^{i phi}
  R apr[FD_K], api[FD_K];
  {
    R amp[FD_K];
    cubic4(0, amp);
#pragma unroll
    for (int j = 0; j < FD_K; ++j) {
      const R a = g[j] ? amp[j] : R(0);
      apr[j] = a * (R)er[j];
      api[j] = a * (R)ei[j];
    }
  }
  // acc += conj(T_ch A e^{i phi}) channel by channel
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) {
    R tr[FD_K], ti[FD_K];
    cubic4(1 + 2 * ch, tr);
    cubic4(2 + 2 * ch, ti);
#pragma unroll
    for (int j = 0; j < FD_K; ++j) {
      R* a = acc[j];
      a[2 * ch] = fma(tr[j], apr[j], a[2 * ch]);
      a[2 * ch] = fma(-ti[j], api[j], a[2 * ch]);
      a[2 * ch + 1] = fma(-tr[j], api[j], a[2 * ch + 1]);
      a[2 * ch + 1] = fma(-ti[j], apr[j], a[2 * ch + 1]);
    }
  }
}

// Self-test of the phase recurrence (no reference counterpart): thread l anchors at grid bin
// k0 + l of the phase cubic pc = (y, c1, c2, c3) about knot xk (rot_anchor, step h = 32 df) and
// advances `steps` times as the fused kernel does; out[2 (l steps + j) + {0, 1}] =
// (cos, sin) of the phase at bin k0 + l + 32 j.
__global__ void k_selftest_recurrence(const double* pc, double xk, double k0, double df, int lanes,
                                      int steps, double* out) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= lanes) return;
  Rot z;
  rot_anchor(z, pc, xk, k0 + (double)l, df, 32.0 * df);
  for (int j = 0; j < steps; ++j) {
    out[2 * ((size_t)l * steps + j)] = z.er;
    out[2 * ((size_t)l * steps + j) + 1] = z.ei;
    cmul_inplace(z.er, z.ei, z.rr, z.ri);
    cmul_inplace(z.rr, z.ri, z.qr, z.qi);
    cmul_inplace(z.qr, z.qi, z.pr, z.pi);
  }
}

// FP64 form off the recurrence path: one (bin, mode) with each quantity's cubic coefficients
// read where they are used, from a staged segment in shared memory (SmemCoef) or from the
// spline arrays in global memory (GlobalCoef), so these less frequent paths hold no segment in
// registers and stay within the register budget of the recurrence path.
struct SmemCoef {
  const WarpStage<double>& S;
  int m, k;
  __device__ __forceinline__ double xk() const { return S.x[m][k]; }
  // quantity p: 0 amplitude, 1 phase, 2 t(f), 3..8 transfer (Re, Im of three channels)
  __device__ __forceinline__ void get(int p, double* c) const {
    const double* src = (p == 1 || p == 2) ? &S.pc[m][k][p - 1][0] : &S.ac[m][k][p == 0 ? 0 : p - 2][0];
    const double2 lo = *reinterpret_cast<const double2*>(src);
    const double2 hi = *reinterpret_cast<const double2*>(src + 2);
    c[0] = lo.x; c[1] = lo.y; c[2] = hi.x; c[3] = hi.y;
  }
};

struct GlobalCoef {
  const FusedArgs& A;
  long long o;  // offset of (binary, mode, segment) in one quantity's [B, M, L] block
  double x;
  __device__ __forceinline__ double xk() const { return x; }
  __device__ __forceinline__ void get(int p, double* c) const {
    const long long q = p * A.qstride + o;
    c[0] = __ldg(A.y + q); c[1] = __ldg(A.c1 + q); c[2] = __ldg(A.c2 + q); c[3] = __ldg(A.c3 + q);
  }
};

template <typename Src>
__device__ __forceinline__ void accumulate_bin_src(const Src& src, double f, double ts, double te,
                                                   double* acc) {
  const double u = f - src.xk();
  double c[4];
  src.get(2, c);
  if (!tf_gate(fma(fma(fma(c[3], u, c[2]), u, c[1]), u, c[0]), ts, te)) return;
  src.get(1, c);
  double sn, cs;
  sincos_cw(fma(fma(fma(c[3], u, c[2]), u, c[1]), u, c[0]), &sn, &cs);
  src.get(0, c);
  const double amp = fma(fma(fma(c[3], u, c[2]), u, c[1]), u, c[0]);
  const double apr = amp * cs, api = amp * sn;
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) {
    src.get(3 + 2 * ch, c);
    const double tr = fma(fma(fma(c[3], u, c[2]), u, c[1]), u, c[0]);
    src.get(4 + 2 * ch, c);
    const double ti = fma(fma(fma(c[3], u, c[2]), u, c[1]), u, c[0]);
    acc[2 * ch] += tr * apr - ti * api;
    acc[2 * ch + 1] -= tr * api + ti * apr;
  }
}

// Per-warp recurrence state: E, R, Q of every (mode, lane), P per mode and, per mode, the chunk
// and segment the saved state belongs to.
struct alignas(16) RecStage {
  double2 st[FD_MAXM][3][32];  // E, R, Q of every lane
  double2 P[FD_MAXM];          // e^{i Delta^3}: the same for every lane of a segment
  int next_chunk[FD_MAXM];
  int seg[FD_MAXM];
};

// G bins of one lane that lie in the same spline segment: the same arithmetic as
// accumulate_bin, written branch-free (invalid or gated-off bins are dropped by selects) so the
// G independent evaluation chains interleave.
template <bool MIXED, typename R, int G>
__device__ __forceinline__ void accumulate_group(const SegCoef<R>& c, const double* f,
                                                 const bool* ok, double ts, double te,
                                                 R (*acc)[6]) {
  double u[G], ph[G];
  bool g[G];
#pragma unroll
  for (int j = 0; j < G; ++j) {
    u[j] = f[j] - c.xk;
    const double tf = fma(fma(fma(c.p3[1], u[j], c.p2[1]), u[j], c.p1[1]), u[j], c.py[1]);
    g[j] = ok[j] && tf_gate(tf, ts, te);
    ph[j] = fma(fma(fma(c.p3[0], u[j], c.p2[0]), u[j], c.p1[0]), u[j], c.py[0]);
  }
#pragma unroll
  for (int j = 0; j < G; ++j) {
    const R ur = (R)u[j];
    R v[7];
#pragma unroll
    for (int a = 0; a < 7; ++a) v[a] = fma(fma(fma(c.a3[a], ur, c.a2[a]), ur, c.a1[a]), ur, c.ay[a]);
    R sn, cs;
    if (MIXED) {
      float sf, cf;
      sincos_mixed(ph[j], &sf, &cf);
      sn = (R)sf;
      cs = (R)cf;
    } else {
      double sd, cd;
      sincos_cw(ph[j], &sd, &cd);
      sn = (R)sd;
      cs = (R)cd;
    }
    const R amp = g[j] ? v[0] : R(0);
    const R apr = amp * cs, api = amp * sn;
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
      const R tr = v[1 + 2 * ch], ti = v[2 + 2 * ch];
      acc[j][2 * ch] += tr * apr - ti * api;
      acc[j][2 * ch + 1] -= tr * api + ti * apr;
    }
  }
}


// Whole-segment t(f) gate: bound the cubic t(u) = y + c1 u + c2 u^2 + c3 u^3 over
// u in [0, h] (end points and stationary points) and classify the segment as entirely inside
// the observation window (1), entirely outside (2) or straddling it (0, per-bin gate).  A
// margin of 1e-6 s (tf reaches ~1e8 s, so 1e-6 s is ~1e6 times its rounding) keeps the
// classification on the safe side of the per-bin test.
__device__ __forceinline__ int segment_gate(const double* pc, double h, double ts, double te) {
  const double y = pc[0], c1 = pc[1], c2 = pc[2], c3 = pc[3];
  double lo = y, hi = y;
  const double yh = fma(fma(fma(c3, h, c2), h, c1), h, y);
  lo = fmin(lo, yh);
  hi = fmax(hi, yh);
  // stationary points: c1 + 2 c2 u + 3 c3 u^2 = 0
  double r[2];
  int nr = 0;
  if (c3 != 0.0) {
    const double disc = 4.0 * c2 * c2 - 12.0 * c3 * c1;
    if (disc >= 0.0) {
      const double sq = sqrt(disc);
      r[nr++] = (-2.0 * c2 + sq) / (6.0 * c3);
      r[nr++] = (-2.0 * c2 - sq) / (6.0 * c3);
    }
  } else if (c2 != 0.0) {
    r[nr++] = -c1 / (2.0 * c2);
  }
  for (int i = 0; i < nr; ++i) {
    if (r[i] > 0.0 && r[i] < h) {
      const double v = fma(fma(fma(c3, r[i], c2), r[i], c1), r[i], y);
      lo = fmin(lo, v);
      hi = fmax(hi, v);
    }
  }
  const double eps = 1e-6;
  if (!(lo == lo) || !(hi == hi)) return 0;
  if (lo >= ts + eps && (te <= 0.0 || hi <= te - eps)) return 1;
  if (hi < ts - eps || (te > 0.0 && lo > te + eps)) return 2;
  return 0;
}

template <typename R>
__device__ __forceinline__ void load_seg(SegCoef<R>& cf, const WarpStage<R>& S, int m, int kl) {
  cf.xk = S.x[m][kl];
#pragma unroll
  for (int a = 0; a < 2; ++a) {
    const double2 lo = *reinterpret_cast<const double2*>(&S.pc[m][kl][a][0]);
    const double2 hi = *reinterpret_cast<const double2*>(&S.pc[m][kl][a][2]);
    cf.py[a] = lo.x; cf.p1[a] = lo.y; cf.p2[a] = hi.x; cf.p3[a] = hi.y;
  }
#pragma unroll
  for (int a = 0; a < 7; ++a) {
    if (sizeof(R) == 4) {
      const float4 v = *reinterpret_cast<const float4*>(&S.ac[m][kl][a][0]);
      cf.ay[a] = (R)v.x; cf.a1[a] = (R)v.y; cf.a2[a] = (R)v.z; cf.a3[a] = (R)v.w;
    } else {
      const double2 lo = *reinterpret_cast<const double2*>(&S.ac[m][kl][a][0]);
      const double2 hi = *reinterpret_cast<const double2*>(&S.ac[m][kl][a][2]);
      cf.ay[a] = (R)lo.x; cf.a1[a] = (R)lo.y; cf.a2[a] = (R)hi.x; cf.a3[a] = (R)hi.y;
    }
  }
}

// One (chunk, mode) on the phase recurrence: staged segment kl (global segment kg of the mode's
// grid) holds every support bin of the chunk.  The saved state is continued when this mode's
// previous chunk of the item was the one before, in the same segment; otherwise it is
// re-anchored at this lane's first bin.
template <typename R>
__device__ __forceinline__ void rec_chunk_mode(const WarpStage<R>& S, RecStage* RS, int m, int kl,
                                               int kg, int gate, int ck, int c0, int lane,
                                               const double* fbin, double ts, double te,
                                               R (*acc)[6], double gk0, double gdf, double hstep) {
  const bool cont = (RS->next_chunk[m] == ck) && (RS->seg[m] == kg);
  Rot z;
  if (cont) {
    const double2 e = RS->st[m][0][lane], r = RS->st[m][1][lane];
    const double2 qq = RS->st[m][2][lane], pp = RS->P[m];
    z.er = e.x; z.ei = e.y; z.rr = r.x; z.ri = r.y;
    z.qr = qq.x; z.qi = qq.y; z.pr = pp.x; z.pi = pp.y;
  } else {
    rot_anchor(z, &S.pc[m][kl][0][0], S.x[m][kl], gk0 + (double)(c0 + lane), gdf, hstep);
  }
  const double2 pnew = make_double2(z.pr, z.pi);
  if (gate == 1)
    accumulate_chunk_rec<R, false>(S, m, kl, fbin, ts, te, acc, z);
  else
    accumulate_chunk_rec<R, true>(S, m, kl, fbin, ts, te, acc, z);
  RS->st[m][0][lane] = make_double2(z.er, z.ei);
  RS->st[m][1][lane] = make_double2(z.rr, z.ri);
  RS->st[m][2][lane] = make_double2(z.qr, z.qi);
  __syncwarp();
  if (lane == 0) {
    RS->next_chunk[m] = ck + 1;
    RS->seg[m] = kg;
    RS->P[m] = pnew;  // every lane's P of the segment is bitwise the same
  }
  __syncwarp();
}

// Copy segments [k0, k0 + n) of (binary b, mode m) into the mode's shared-memory slot: knots
// x[k0 .. k0 + n], the FP64 phase / t(f) cubics and the amplitude / transfer cubics in R.
template <typename R>
__device__ __forceinline__ void stage_segments(const FusedArgs& A, WarpStage<R>& S, int b, int m,
                                               int k0, int n, int lane) {
  const long long rowo = ((long long)b * A.M + m) * A.L + k0;
  const int total = n * FD_NC + n + 1;
  for (int idx = lane; idx < total; idx += 32) {
    if (idx < n * FD_NC) {
      const int sg = idx / FD_NC, r = idx - sg * FD_NC, p = r >> 2, cc = r & 3;
      const double* src = (cc == 0) ? A.y : (cc == 1) ? A.c1 : (cc == 2) ? A.c2 : A.c3;
      const double v = __ldg(src + p * A.qstride + rowo + sg);
      if (p == 1 || p == 2)
        S.pc[m][sg][p - 1][cc] = v;
      else
        S.ac[m][sg][(p == 0) ? 0 : p - 2][cc] = (R)v;
    } else {
      const int j = idx - n * FD_NC;
      S.x[m][j] = __ldg(A.x + rowo + j);
    }
  }
}

// One WARP item = (data tile of FD_TILE bins, binary).  Items are enumerated tile-major and
// claimed in increasing order (claim_item), so the warps in flight work on the same data tile
// for different binaries and share it through L2.
// The warp stages the tile's segments of every mode (from the segment table) into its slice of
// shared memory, then walks the tile in FD_TILE / FD_WARP_BINS chunks of 128 bins (lane l owns
// bins chunk + l + 32 j, j < FD_K) and keeps the <d|h>, <h|h> partial sums in registers; no
// block-wide barrier is involved.  Modes whose tile spans more than NSEG segments (low
// frequencies) are staged a window of NSEG segments at a time from a forward cursor in the FP64
// form, and walked per lane over global memory in the mixed form.
// MIXED: phase, t(f), the phase reduction and all accumulations in FP64; amplitude, transfer
// functions, sin/cos of the reduced phase and the mode sum (the template) in FP32; the per-bin
// products with data and weights in FP64 when the FP32 copies of data and weights are given
// (the path of Likelihood and UnevenBatch), in FP32 without them.
// GH (FP64 form only): also write d lnL / d h of every support bin to A.gh (gradient chain).
// REC (FP64 form): the phase recurrence in the one-segment chunk path when the data grid is
// uniform (A.grid), with its state in RS.
template <bool MIXED, typename R, bool GH = false, bool REC = false>
__device__ __forceinline__ void fused_item(const FusedArgs& A, long long q, WarpStage<R>& S,
                                           RecStage* RS, int lane) {
  const long long BML = A.qstride;
  const int L = A.L;
  bool uni = false;
  double gk0 = 0.0, gdf = 0.0;
  if (REC && A.grid != nullptr) {
    const unsigned ok = A.grid->ok & 7u;
    if (ok) {
      uni = true;
      gk0 = A.grid->k0;
      gdf = A.grid->df[(ok & 1u) ? 0 : (ok & 2u) ? 1 : 2];
    }
  }
  const double hstep = 32.0 * gdf;
  {
    const int tile = (int)(q / A.B);
    const int b = (int)(q - (long long)tile * A.B);
    const int s0 = __ldg(A.sup_start + b);
    const int s1 = s0 + __ldg(A.sup_len + b);
    const int t0 = tile * A.tile;
    if (t0 >= s1 || t0 + A.tile <= s0) {
      if (lane == 0) {
        double* P = A.partials + 3 * q;
        P[0] = 0.0; P[1] = 0.0; P[2] = 0.0;
      }
      return;
    }
    // ---- stage this tile's segments for every mode
    if (REC && lane < FD_MAXM) RS->next_chunk[lane] = -1;
    if (lane < A.M) {
      const int2 kk = A.segtab[q * A.M + lane];
      const int klo = max(kk.x, 0), khi = min(kk.y, L - 2);
      const int n = (kk.x > kk.y || khi < klo) ? 0 : khi - klo + 1;
      S.klo[lane] = klo;
      S.nseg[lane] = (n > WarpStage<R>::NSEG) ? -1 : n;
      S.kcur[lane] = klo;
      S.nst[lane] = 0;
    }
    __syncwarp();
    for (int m = 0; m < A.M; ++m) {
      const int n = S.nseg[m];
      if (n <= 0) continue;
      const long long rowo = ((long long)b * A.M + m) * L + S.klo[m];
      const int total = n * FD_NC + n + 1;
      for (int idx = lane; idx < total; idx += 32) {
        if (idx < n * FD_NC) {
          const int sg = idx / FD_NC, r = idx - sg * FD_NC, p = r >> 2, cc = r & 3;
          const double* src = (cc == 0) ? A.y : (cc == 1) ? A.c1 : (cc == 2) ? A.c2 : A.c3;
          const double v = __ldg(src + p * BML + rowo + sg);
          if (p == 1 || p == 2)
            S.pc[m][sg][p - 1][cc] = v;
          else
            S.ac[m][sg][(p == 0) ? 0 : p - 2][cc] = (R)v;
        } else {
          const int j = idx - n * FD_NC;
          S.x[m][j] = __ldg(A.x + rowo + j);
        }
      }
    }
    __syncwarp();
    const double ts = __ldg(A.t_start + b), te = __ldg(A.t_end + b);
    constexpr int NSEG = WarpStage<R>::NSEG;
    for (int idx = lane; idx < A.M * NSEG; idx += 32) {
      const int m = idx / NSEG, sg = idx - m * NSEG;
      if (sg < S.nseg[m])
        S.gate[m][sg] = segment_gate(&S.pc[m][sg][1][0], S.x[m][sg + 1] - S.x[m][sg], ts, te);
    }
    const int nchunk = A.tile / FD_WARP_BINS;
    for (int idx = lane; idx < nchunk * A.M; idx += 32) {
      const int ck = idx / A.M, m = idx - ck * A.M;
      const int c0 = t0 + ck * FD_WARP_BINS;
      const int n = S.nseg[m];
      int seg = -1;
      if (n > 0 && c0 < s1 && c0 + FD_WARP_BINS > s0) {
        const double fa = __ldg(A.data_freqs + max(c0, s0));
        const double fb = __ldg(A.data_freqs + min(c0 + FD_WARP_BINS, s1) - 1);
        int ka = -1, kz = -1;
        for (int k = 0; k <= n; ++k) {
          const double xk = S.x[m][k];
          ka = (xk <= fa) ? k : ka;
          kz = (xk <= fb) ? k : kz;
        }
        if (ka == kz && ka >= 0 && ka < n) seg = ka;
      }
      S.cseg[ck][m] = (signed char)seg;
    }
    __syncwarp();
    double dr = 0.0, di = 0.0, hh = 0.0;
    for (int ch0 = 0; ch0 < A.tile; ch0 += FD_WARP_BINS) {
      const int c0 = t0 + ch0;
      if (c0 >= s1 || c0 + FD_WARP_BINS <= s0) continue;
      double fbin[FD_K];
      R acc[FD_K][6];
#pragma unroll
      for (int j = 0; j < FD_K; ++j) {
        const int i = c0 + 32 * j + lane;
        // on a verified uniform grid f_i = fl(k df) is recomputed bit-exactly instead of loaded
        fbin[j] = (i >= s0 && i < s1) ? (uni ? __dmul_rn(gk0 + (double)i, gdf)
                                             : __ldg(A.data_freqs + i))
                                      : -1.0;
#pragma unroll
        for (int c = 0; c < 6; ++c) acc[j][c] = R(0);
      }
      const int ck = ch0 / FD_WARP_BINS;
      for (int m = 0; m < A.M; ++m) {
        const int n = S.nseg[m];
        if (n == 0) continue;
        SegCoef<R> cf;
        if (n > 0) {
          // warp-uniform fast path: the whole chunk lies in one staged segment
          const int ka = S.cseg[ck][m];
          if (ka >= 0) {
            const int gate = S.gate[m][ka];
            if (gate == 2) continue;
            if (REC && uni) {
              rec_chunk_mode(S, RS, m, ka, S.klo[m] + ka, gate, ck, c0, lane, fbin, ts, te, acc,
                             gk0, gdf, hstep);
              continue;
            }
            if constexpr (!MIXED) {
              const SmemCoef src{S, m, ka};
#pragma unroll
              for (int j = 0; j < FD_K; ++j)
                if (fbin[j] >= 0.0) accumulate_bin_src(src, fbin[j], ts, te, acc[j]);
              continue;
            } else {
              load_seg<R>(cf, S, m, ka);
              constexpr int G = 2;  // two interleaved bins: best of 1/2/4 at 4 CTAs per SM
              if (gate == 1)
                accumulate_chunk<MIXED, R, G, false>(cf, fbin, ts, te, acc);
              else
                accumulate_chunk<MIXED, R, G, true>(cf, fbin, ts, te, acc);
              continue;
            }
          }
          // segment of every bin (local index; n = past the last staged segment)
          int kb[FD_K];
          bool ok[FD_K];
          int kl = 0;
#pragma unroll
          for (int j = 0; j < FD_K; ++j) {
            const double f = fbin[j];
            ok[j] = f >= S.x[m][0];  // also false for bins outside the support (f = -1)
            while (ok[j] && kl < n && f >= S.x[m][kl + 1]) ++kl;
            ok[j] = ok[j] && kl < n;
            kb[j] = kl;
          }
          if constexpr (!MIXED) {
#pragma unroll
            for (int j = 0; j < FD_K; ++j)
              if (ok[j]) accumulate_bin_src(SmemCoef{S, m, kb[j]}, fbin[j], ts, te, acc[j]);
            continue;
          }
          constexpr int G = 1;
          int kc = -1;
#pragma unroll
          for (int j0 = 0; j0 < FD_K; j0 += G) {
            // group path when every valid bin of the group sits in one segment
            int kg = -1;
            bool same = true, any = false;
#pragma unroll
            for (int j = j0; j < j0 + G; ++j) {
              if (!ok[j]) continue;
              if (kg < 0) kg = kb[j];
              same = same && (kb[j] == kg);
              any = true;
            }
            if (!any) continue;
            if (same) {
              if (kg != kc) {
                kc = kg;
                load_seg<R>(cf, S, m, kg);
              }
              accumulate_group<MIXED, R, G>(cf, fbin + j0, ok + j0, ts, te, acc + j0);
            } else {
#pragma unroll
              for (int j = j0; j < j0 + G; ++j) {
                if (!ok[j]) continue;
                if (kb[j] != kc) {
                  kc = kb[j];
                  load_seg<R>(cf, S, m, kc);
                }
                accumulate_bin<MIXED, R>(cf, fbin[j], ts, te, acc[j]);
              }
            }
          }
        } else {
          const long long rowi = (long long)b * A.M + m;
          const double* xrow = A.x + rowi * L;
          if constexpr (!MIXED) {
            // the tile spans more segments of this mode than the slot holds (low frequencies):
            // find the chunk's segments from the forward cursor with one warp-wide load of the
            // next 32 knots, and stage a window of NSEG segments from there when the chunk
            // leaves the staged window
            const int ia = max(c0, s0), iz = min(c0 + FD_WARP_BINS, s1) - 1;
            const double fa = uni ? __dmul_rn(gk0 + (double)ia, gdf) : __ldg(A.data_freqs + ia);
            const double fz = uni ? __dmul_rn(gk0 + (double)iz, gdf) : __ldg(A.data_freqs + iz);
            const int kc = S.kcur[m];
            const int kq = kc + lane;
            const double xv = (kq < L) ? __ldg(xrow + kq) : INFINITY;
            const unsigned ma = __ballot_sync(0xffffffffu, xv <= fa);
            const unsigned mz = __ballot_sync(0xffffffffu, xv <= fz);
            int ka, kz;
            if (mz != 0xffffffffu && ma != 0u) {
              ka = kc + __popc(ma) - 1;
              kz = kc + __popc(mz) - 1;
            } else {  // more than 32 segments ahead (or behind): full searches
              ka = warp_segment_search(xrow, L, fa);
              kz = warp_segment_search(xrow, L, fz);
            }
            const int klo = max(ka, 0), khi = min(kz, L - 2);
            const int nc = khi - klo + 1;
            const int kst0 = S.kst[m], nst0 = S.nst[m];
            __syncwarp();
            if (lane == 0) S.kcur[m] = klo;
            if (nc <= 0) {
              __syncwarp();
              continue;  // no bin of the chunk has a valid segment
            }
            constexpr int NSEG = WarpStage<R>::NSEG;
            if (nc <= NSEG) {
              int kst = kst0;
              if (!(nst0 > 0 && klo >= kst0 && khi < kst0 + nst0)) {
                kst = klo;
                const int nst = min(NSEG, L - 1 - klo);
                stage_segments(A, S, b, m, klo, nst, lane);
                __syncwarp();
                // whole-segment t(f) gates of the window, one segment per lane
                if (lane < nst)
                  S.gate[m][lane] = segment_gate(&S.pc[m][lane][1][0],
                                                 S.x[m][lane + 1] - S.x[m][lane], ts, te);
                if (lane == 0) {
                  S.kst[m] = klo;
                  S.nst[m] = nst;
                }
              }
              __syncwarp();
              const int kl0 = klo - kst, kl1 = khi - kst;
              if (ka == kz) {  // one segment holds every bin of the chunk
                const int gate = S.gate[m][kl0];
                if (gate != 2) {
                  if (REC && uni) {
                    rec_chunk_mode(S, RS, m, kl0, klo, gate, ck, c0, lane, fbin, ts, te, acc, gk0,
                                   gdf, hstep);
                  } else {
                    const SmemCoef src{S, m, kl0};
#pragma unroll
                    for (int j = 0; j < FD_K; ++j)
                      if (fbin[j] >= 0.0) accumulate_bin_src(src, fbin[j], ts, te, acc[j]);
                  }
                }
              } else {
                int kb[FD_K];
                bool ok[FD_K];
                int kl = kl0;
#pragma unroll
                for (int j = 0; j < FD_K; ++j) {
                  const double f = fbin[j];
                  ok[j] = f >= S.x[m][kl0];
                  while (ok[j] && kl <= kl1 && f >= S.x[m][kl + 1]) ++kl;
                  ok[j] = ok[j] && kl <= kl1;
                  kb[j] = kl;
                }
#pragma unroll
                for (int j = 0; j < FD_K; ++j)
                  if (ok[j]) accumulate_bin_src(SmemCoef{S, m, kb[j]}, fbin[j], ts, te, acc[j]);
              }
              __syncwarp();
              continue;
            }
          }
          const double ffirst = __ldg(A.data_freqs + max(c0, s0));
          int k = warp_segment_search(xrow, L, ffirst);
          int kc = -2;
          double xk1 = -1.0;
#pragma unroll
          for (int j = 0; j < FD_K; ++j) {
            const double f = fbin[j];
            if (f < 0.0) continue;
            if (!(f < xk1) || k != kc) {
              while (k + 1 < L && __ldg(xrow + k + 1) <= f) ++k;
            }
            if (k < 0 || k >= L - 1) continue;
            if constexpr (!MIXED) {
              if (k != kc) {
                kc = k;
                xk1 = __ldg(xrow + k + 1);
              }
              accumulate_bin_src(GlobalCoef{A, rowi * L + k, __ldg(xrow + k)}, f, ts, te, acc[j]);
              continue;
            }
            if (k != kc) {
              kc = k;
              cf.xk = __ldg(xrow + k);
              xk1 = __ldg(xrow + k + 1);
              const long long o = rowi * L + k;
#pragma unroll
              for (int p = 0; p < 9; ++p)
                cf.set(p, __ldg(A.y + p * BML + o), __ldg(A.c1 + p * BML + o),
                       __ldg(A.c2 + p * BML + o), __ldg(A.c3 + p * BML + o));
            }
            accumulate_bin<MIXED, R>(cf, f, ts, te, acc[j]);
          }
        }
      }
      if (MIXED && A.data32 != nullptr) {
        // FP32 data and weights, FP32 template; the per-bin products w h, conj(d) w h and
        // |w h|^2 in FP64: their FP32 rounding (random per bin, ~1e-7 relative) summed over the
        // loud bins of <h|h> would leave ~1e-2..1e-1 in lnL near the peak of an SNR ~ 5000
        // source, where the FP32 template error itself enters only through d - h
#pragma unroll
        for (int j = 0; j < FD_K; ++j) {
          if (fbin[j] < 0.0) continue;
          const int i = c0 + 32 * j + lane;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const long long gi = (long long)c * A.N + i;
            const double w = (double)__ldg(A.noise32 + gi);
            const float2 d = __ldg(A.data32 + gi);
            const double hr = (double)acc[j][2 * c] * w, hi = (double)acc[j][2 * c + 1] * w;
            const double dx = (double)d.x, dy = (double)d.y;
            dr = fma(dx, hr, fma(dy, hi, dr));
            di = fma(dx, hi, fma(-dy, hr, di));
            hh = fma(hr, hr, fma(hi, hi, hh));
          }
        }
      } else {
#pragma unroll
        for (int j = 0; j < FD_K; ++j) {
          if (fbin[j] < 0.0) continue;
          const int i = c0 + 32 * j + lane;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const long long gi = (long long)c * A.N + i;
            const R w = (R)__ldg(A.noise + gi);
            const double2 d = __ldg(reinterpret_cast<const double2*>(A.data) + gi);
            const R hr = acc[j][2 * c] * w, hi = acc[j][2 * c + 1] * w;
            const R dxr = (R)d.x, dyr = (R)d.y;
            dr += (double)(dxr * hr + dyr * hi);
            di += (double)(dxr * hi - dyr * hr);
            hh += (double)(hr * hr + hi * hi);
            if (GH) {
              const long long o = 3 * (__ldg(A.gh_off + b) + (i - s0)) + c;
              A.gh[o] = mk(4.0 * (double)w * (d.x - (double)hr), 4.0 * (double)w * (d.y - (double)hi));
            }
          }
        }
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      dr += __shfl_xor_sync(0xffffffffu, dr, o);
      di += __shfl_xor_sync(0xffffffffu, di, o);
      hh += __shfl_xor_sync(0xffffffffu, hh, o);
    }
    if (lane == 0) {
      double* P = A.partials + 3 * q;
      P[0] = dr;
      P[1] = di;
      P[2] = hh;
    }
    __syncwarp();
  }
}

// Shared memory of the fused kernels: FD_WARPS WarpStage slices, then (FP64 form, phase
// recurrence) FD_WARPS RecStage slices.
template <bool MIXED>
constexpr size_t fused_smem_bytes() {
  using R = typename std::conditional<MIXED, float, double>::type;
  return FD_WARPS * (sizeof(WarpStage<R>) + (MIXED ? 0 : sizeof(RecStage)));
}

template <bool MIXED, bool GH = false>
__global__ void __launch_bounds__(FD_WARPS * 32, MIXED ? 4 : 3) k_direct_fused(FusedArgs A) {
  static_assert(!(MIXED && GH), "d lnL / d h is written by the FP64 form only");
  using R = typename std::conditional<MIXED, float, double>::type;
  constexpr bool REC = !MIXED;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  WarpStage<R>& S = reinterpret_cast<WarpStage<R>*>(smem_raw)[warp];
  RecStage* RS = REC ? reinterpret_cast<RecStage*>(smem_raw + FD_WARPS * sizeof(WarpStage<R>)) + warp
                     : nullptr;
  const long long nitems = (long long)A.ntiles * A.B;
  for (long long q = claim_item(A.next, lane); q < nitems; q = claim_item(A.next, lane))
    fused_item<MIXED, R, GH, REC>(A, q, S, RS, lane);
}

// Several independent problems (groups: own data stream, grid length L, mode count M,
// binaries) in ONE persistent launch: the items of all groups form one global range that the
// warps stride over; a warp copies the descriptor of its current group into shared memory
// when it moves to another group.  Group descriptors and the item offsets are in device
// memory (written by k_store_groups from kernel parameters, so no host copy is involved).
constexpr int FD_MAXGROUPS = 64;
struct MultiArgs {
  FusedArgs g[FD_MAXGROUPS];
  long long off[FD_MAXGROUPS + 1];   // item offsets; off[ngroups] = total items
  long long boff[FD_MAXGROUPS + 1];  // binary offsets; boff[ngroups] = total binaries
  long long soff[FD_MAXGROUPS + 1];  // segment-table entry offsets (ntiles B M per group)
  int ngroups;
};

__global__ void k_store_groups(MultiArgs M, MultiArgs* dst) {
  const int n = (int)(sizeof(MultiArgs) / sizeof(unsigned long long));
  const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&M);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(dst);
  for (int i = threadIdx.x; i < n; i += blockDim.x) d[i] = src[i];
}

// Heterodyned problems of an uneven batch: their walkers form one item range in front of the
// direct items of k_uneven.  Stored in device memory by k_store_het (from kernel parameters).
struct HetMulti {
  HetArgs g[FD_MAXGROUPS];
  long long woff[FD_MAXGROUPS + 1];  // walker offsets; woff[ngroups] = total walkers
  long long roff[FD_MAXGROUPS + 1];  // (walker, mode) record offsets
  int ngroups;
};

__global__ void k_store_het(HetMulti H, HetMulti* dst) {
  const int n = (int)(sizeof(HetMulti) / sizeof(unsigned long long));
  const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&H);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(dst);
  for (int i = threadIdx.x; i < n; i += blockDim.x) d[i] = src[i];
}

// Last index i in [0, n) with off[i] <= q (off ascending, off[0] = 0 <= q).
__device__ __forceinline__ int group_of(const long long* off, int n, long long q) {
  int lo = 0, hi = n;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= q) lo = mid; else hi = mid;
  }
  return lo;
}

// Response-mode records of every walker of every heterodyned problem (thread per (walker,
// mode) of the concatenated record range).
__global__ void k_het_response_setup_multi(const HetMulti* __restrict__ HM, long long n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int g = group_of(HM->roff, HM->ngroups, t);
    het_response_setup(HM->g[g], t - HM->roff[g]);
  }
}

// An uneven batch in ONE persistent launch: the walkers of every heterodyned problem (one
// warp item each, het_item) followed by the (tile, binary) items of every direct problem
// (fused_item), enumerated as one range from which the warps claim items (claim_item).  Each warp owns a
// shared-memory slot of `slot` bytes that holds either a direct item's staged segments (and
// recurrence state) or a walker's records and residual strip; the problem's argument block is
// copied to shared memory when the warp moves to another problem.  HET = false compiles the
// walker path out (batches without heterodyned problems): the mixed direct items then run
// within 128 registers, 4 CTAs per SM; with walkers the mixed kernel takes the FP64 budget
// (168 registers, 3 CTAs per SM), which the FP32 heterodyne models need without spilling.
template <bool MIXED, bool HET>
__global__ void __launch_bounds__(FD_WARPS * 32, (MIXED && !HET) ? 4 : 3)
    k_uneven(const MultiArgs* __restrict__ MA, const HetMulti* __restrict__ HM, int slot,
             unsigned long long* next) {
  using R = typename std::conditional<MIXED, float, double>::type;
  constexpr bool REC = !MIXED;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ FusedArgs gcur[FD_WARPS];
  __shared__ HetArgs hcur[FD_WARPS];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  unsigned char* mine = smem_raw + (size_t)warp * slot;
  WarpStage<R>& S = *reinterpret_cast<WarpStage<R>*>(mine);
  RecStage* RS = REC ? reinterpret_cast<RecStage*>(mine + sizeof(WarpStage<R>)) : nullptr;
  const long long nh = HM->woff[HM->ngroups];
  const long long total = nh + MA->off[MA->ngroups];
  int g = -1, hg = -1;
  for (long long q = claim_item(next, lane); q < total; q = claim_item(next, lane)) {
    if (HET && q < nh) {
      if (hg < 0 || q >= HM->woff[hg + 1] || q < HM->woff[hg]) {
        hg = group_of(HM->woff, HM->ngroups, q);
        __syncwarp();
        const int n8 = (int)(sizeof(HetArgs) / sizeof(unsigned long long));
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&HM->g[hg]);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(&hcur[warp]);
        for (int i = lane; i < n8; i += 32) dst[i] = src[i];
        __syncwarp();
      }
      const HetArgs& H = hcur[warp];
      het_item<MIXED, false, false>(H, (int)(q - HM->woff[hg]),
                                    HetSlice(mine, HetSmemLayout(H.M, H.L, false)), lane,
                                    &g_nonfinite_likelihood);
    } else {
      const long long qd = q - nh;
      if (g < 0 || qd >= MA->off[g + 1] || qd < MA->off[g]) {
        g = group_of(MA->off, MA->ngroups, qd);
        __syncwarp();
        const int n8 = (int)(sizeof(FusedArgs) / sizeof(unsigned long long));
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&MA->g[g]);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(&gcur[warp]);
        for (int i = lane; i < n8; i += 32) dst[i] = src[i];
        __syncwarp();
      }
      fused_item<MIXED, R, false, REC>(gcur[warp], qd - MA->off[g], S, RS, lane);
    }
  }
}

__global__ void k_fused_reduce_multi(const MultiArgs* __restrict__ MA) {
  const long long* boff = MA->boff;
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  const int ng = MA->ngroups;
  const long long nb = boff[ng];
  for (long long gb = blockIdx.x * (long long)wpb + (threadIdx.x >> 5); gb < nb;
       gb += (long long)gridDim.x * wpb) {
    int lo = 0, hi = ng;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (boff[mid] <= gb) lo = mid; else hi = mid;
    }
    const FusedArgs& A = MA->g[lo];
    const int b = (int)(gb - boff[lo]);
    double a = 0, c = 0, h = 0;
    const int s0 = A.sup_start[b], n = A.sup_len[b];
    if (n > 0) {
      const int tlo = s0 / A.tile, thi = (s0 + n - 1) / A.tile;
      for (int t = tlo + lane; t <= thi; t += 32) {
        const double* P = A.partials + 3 * ((long long)t * A.B + b);
        a += P[0];
        c += P[1];
        h += P[2];
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      c += __shfl_xor_sync(0xffffffffu, c, o);
      h += __shfl_xor_sync(0xffffffffu, h, o);
    }
    if (lane == 0) {
      A.d_h[2 * b] = 4.0 * a;
      A.d_h[2 * b + 1] = 4.0 * c;
      A.h_h[2 * b] = 4.0 * h;
      A.h_h[2 * b + 1] = 0.0;
      note_nonfinite(&g_nonfinite_likelihood, a, c, h, 0.0);
    }
  }
}

// out: d_h[b], h_h[b] complex (device).  One warp per binary: lane l sums tiles l, l+32, ...
// of the binary's support, then a fixed shuffle tree; the order is the same on every run.
__global__ void k_fused_reduce(const double* partials, const int* sup_start, const int* sup_len,
                               int B, double* d_h, double* h_h) {
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  for (int b = blockIdx.x * wpb + (threadIdx.x >> 5); b < B; b += gridDim.x * wpb) {
    double a = 0, c = 0, h = 0;
    int s0 = sup_start[b], n = sup_len[b];
    if (n > 0) {
      int tlo = s0 / FD_TILE, thi = (s0 + n - 1) / FD_TILE;
      for (int t = tlo + lane; t <= thi; t += 32) {
        const double* P = partials + 3 * ((long long)t * B + b);
        a += P[0];
        c += P[1];
        h += P[2];
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      c += __shfl_xor_sync(0xffffffffu, c, o);
      h += __shfl_xor_sync(0xffffffffu, h, o);
    }
    if (lane == 0) {
      d_h[2 * b] = 4.0 * a;
      d_h[2 * b + 1] = 4.0 * c;
      h_h[2 * b] = 4.0 * h;
      h_h[2 * b + 1] = 0.0;
      note_nonfinite(&g_nonfinite_likelihood, a, c, h, 0.0);
    }
  }
}

}  // namespace bbhx

namespace bbhx {

// d lnL / d h of binaries [b0, b0 + nb) of a [B_all, M, L] sparse-buffer / spline set, by the
// FP64 fused kernel (gradient chain, gradient.cu): gh packed by the batch-local support
// offsets gh_off; start / len the support of all B_all binaries (bbhx_template_support);
// d_h, h_h (complex [B_all], may be null) receive the batch's <d|h>, <h|h>.
// Grid of a queue-driven fused kernel: the CTAs (FD_WARPS warps, `smem` bytes of dynamic shared
// memory, its attribute already set) that are resident on the whole GPU at once, fewer when the
// items are fewer.  Every warp then claims items until the queue drains, with no second wave.
template <typename K>
unsigned resident_grid(K kernel, size_t smem, long long nitems) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, FD_WARPS * 32, smem) !=
          cudaSuccess ||
      per_sm < 1) {
    (void)cudaGetLastError();
    per_sm = 1;
  }
  const long long want = (nitems + FD_WARPS - 1) / FD_WARPS;
  return (unsigned)std::max<long long>(1, std::min<long long>(want, (long long)per_sm * sm_count()));
}

int direct_fused_gh(cplx* gh, const long long* gh_off, double* d_h, double* h_h,
                    const int* start, const int* len, const double* data_freqs,
                    const double* data, const double* noise, int N, const double* x,
                    const double* y, const double* c1, const double* c2, const double* c3,
                    const double* t_start, const double* t_end, int M, int L, int B_all, int b0,
                    int nb, cudaStream_t s) {
  if (nb == 0) return OK;
  const int ntiles = (N + FD_TILE - 1) / FD_TILE;
  const long long nitems = (long long)ntiles * nb;
  const long long row0 = (long long)b0 * M * L;
  double* part = nullptr;
  int2* segtab = nullptr;
  GridInfo* grid = nullptr;
  unsigned long long* next = nullptr;
  BBHX_CHECK_CUDA(pool_alloc_all(s, {{(void**)&part, sizeof(double) * 3 * nitems},
                                     {(void**)&segtab, sizeof(int2) * nitems * M},
                                     {(void**)&grid, sizeof(GridInfo)},
                                     {(void**)&next, sizeof(unsigned long long)}}));
  k_tile_segments<<<grid_for(nitems * M, 256, sm_count() * 64), 256, 0, s>>>(
      segtab, x + row0, data_freqs, start + b0, len + b0, nb, M, L, ntiles, FD_TILE);
  int st = launch_status("k_tile_segments");
  if (!st) st = detect_grid(data_freqs, N, grid, s);
  if (!st) {
    FusedArgs A;
    A.data_freqs = data_freqs;
    A.data = (const cplx*)data;
    A.noise = noise;
    A.N = N;
    A.x = x + row0;
    A.y = y + row0;
    A.c1 = c1 + row0;
    A.c2 = c2 + row0;
    A.c3 = c3 + row0;
    A.t_start = t_start + b0;
    A.t_end = t_end + b0;
    A.sup_start = start + b0;
    A.sup_len = len + b0;
    A.B = nb;
    A.M = M;
    A.L = L;
    A.ntiles = ntiles;
    A.tile = FD_TILE;
    A.partials = part;
    A.segtab = segtab;
    A.d_h = nullptr;
    A.h_h = nullptr;
    A.data32 = nullptr;
    A.noise32 = nullptr;
    A.qstride = (long long)B_all * M * L;
    A.gh = gh;
    A.gh_off = gh_off;
    A.grid = grid;
    A.next = next;
    const size_t sm = fused_smem_bytes<false>();
    st = cuda_status(cudaFuncSetAttribute(k_direct_fused<false, true>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm),
                     "cudaFuncSetAttribute(k_direct_fused)");
    if (!st)
      st = cuda_status(cudaMemsetAsync(next, 0, sizeof(unsigned long long), s), "work-queue counter");
    if (!st) {
      const unsigned grid = resident_grid(k_direct_fused<false, true>, sm, nitems);
      k_direct_fused<false, true><<<grid, FD_WARPS * 32, sm, s>>>(A);
      st = launch_status("k_direct_fused (d lnL / d h)");
    }
  }
  if (!st && d_h != nullptr && h_h != nullptr) {
    k_fused_reduce<<<grid_for(32LL * nb, 128), 128, 0, s>>>(part, start + b0, len + b0, nb,
                                                            d_h + 2LL * b0, h_h + 2LL * b0);
    st = launch_status("k_fused_reduce");
  }
  pool_free(part, s);
  pool_free(segtab, s);
  pool_free(grid, s);
  pool_free(next, s);
  return st;
}

}  // namespace bbhx

using namespace bbhx;

extern "C" {

// Likelihood.hh:11.  d_h, h_h: HOST complex128 arrays, accumulated (+=) like the reference;
// template_ptrs / inds_start / ind_lengths: HOST arrays.  Templates are noise-weighted in
// place, as the reference does.
int bbhx_direct_like(double* d_h, double* h_h, const double* data, const double* noise,
                     const int64_t* template_ptrs, const int* inds_start, const int* ind_lengths,
                     int data_stream_length, int num_bin_all, void* stream) {
  BBHX_REQUIRE(num_bin_all <= 65535, "direct_like handles at most 65535 binaries per call");
  if (num_bin_all == 0) return OK;
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<DirectJob> jobs(num_bin_all);
  long long nparts = 0;
  int maxparts = 0;
  for (int b = 0; b < num_bin_all; ++b) {
    BBHX_REQUIRE(ind_lengths[b] >= 0 && inds_start[b] >= 0 &&
                     (long long)inds_start[b] + ind_lengths[b] <= data_stream_length,
                 "binary %d: data range outside the data grid", b);
    jobs[b].tmpl = (cplx*)template_ptrs[b];
    jobs[b].start = inds_start[b];
    jobs[b].len = ind_lengths[b];
    jobs[b].part0 = nparts;
    jobs[b].nparts = (ind_lengths[b] + DL_CHUNK - 1) / DL_CHUNK;
    nparts += jobs[b].nparts;
    if (jobs[b].nparts > maxparts) maxparts = jobs[b].nparts;
  }
  DirectJob* d_jobs = nullptr;
  double* d_part = nullptr;
  double* d_out = nullptr;
  BBHX_CHECK_CUDA(pool_alloc_all(s, {{(void**)&d_jobs, sizeof(DirectJob) * num_bin_all},
                                     {(void**)&d_part, sizeof(double) * 3 * (nparts + 1)},
                                     {(void**)&d_out, sizeof(double) * 4 * num_bin_all}}));
  int st = cuda_status(cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(DirectJob) * num_bin_all,
                                       cudaMemcpyHostToDevice, s),
                       "direct_like job upload");
  if (!st && maxparts > 0) {
    unsigned gx = maxparts > 1024 ? 1024 : maxparts;
    k_direct_like_partials<<<dim3(gx, num_bin_all), 256, 0, s>>>(d_jobs, (const cplx*)data, noise,
                                                                 data_stream_length, d_part);
    st = launch_status("k_direct_like_partials");
  }
  if (!st) {
    k_sum_partials<<<grid_for(num_bin_all, 128), 128, 0, s>>>(d_jobs, d_part, d_out, num_bin_all);
    st = launch_status("k_sum_partials");
  }
  std::vector<double> host(4 * (size_t)num_bin_all);
  if (!st) {
    cudaError_t e = cudaMemcpyAsync(host.data(), d_out, sizeof(double) * 4 * num_bin_all,
                                    cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = cuda_status(e, "direct_like result copy");
  }
  pool_free(d_jobs, s);
  pool_free(d_part, s);
  pool_free(d_out, s);
  if (st) return st;
  bool finite = true;
  for (int b = 0; b < num_bin_all; ++b) {
    d_h[2 * b] += host[4 * b];
    d_h[2 * b + 1] += host[4 * b + 1];
    h_h[2 * b] += host[4 * b + 2];
    h_h[2 * b + 1] += host[4 * b + 3];
    finite = finite && std::isfinite(host[4 * b] + host[4 * b + 1] + host[4 * b + 2]);
  }
  if (!finite) {
    set_error("direct_like: non-finite <d|h> or <h|h> (results written)");
    return ERR_NONFINITE;
  }
  return OK;
}

// Likelihood.hh:6-9 (GPU semantics: every bin j = 1..L-1 contributes)
int bbhx_hdyn(double* d_h, double* h_h, const double* residuals, const double* constants,
              const double* freqs, int num_bin_all, int length, int n_channels, void* stream) {
  BBHX_REQUIRE(length >= 1 && n_channels >= 1, "bad sizes");
  if (num_bin_all == 0) return OK;
  k_hdyn<<<grid_for(num_bin_all, 128), 128, 0, (cudaStream_t)stream>>>(
      (cplx*)d_h, (cplx*)h_h, (const cplx*)residuals, (const cplx*)constants, freqs, num_bin_all,
      length, n_channels);
  return launch_status("k_hdyn");
}

// Phase-recurrence self-test (k_selftest_recurrence); pc [4] and out [2 lanes steps] device.
int bbhx_selftest_recurrence(const double* pc, double xk, double k0, double df, int lanes,
                             int steps, double* out, void* stream) {
  BBHX_REQUIRE(lanes >= 1 && lanes <= 1024 && steps >= 1 && steps <= 4096, "bad sizes");
  k_selftest_recurrence<<<(lanes + 127) / 128, 128, 0, (cudaStream_t)stream>>>(pc, xk, k0, df,
                                                                              lanes, steps, out);
  return launch_status("k_selftest_recurrence");
}

// Support [start, start+len) of each binary on the data grid (device int arrays).
int bbhx_template_support(int* start, int* len, const double* x, int num_modes, int length,
                          int num_bin_all, const double* data_freqs, int data_length,
                          void* stream) {
  if (num_bin_all == 0) return OK;
  k_support<<<num_bin_all, 128, 0, (cudaStream_t)stream>>>(x, num_modes, length, num_bin_all,
                                                           data_freqs, data_length, start, len);
  return launch_status("k_support");
}

}  // extern "C"

namespace bbhx {
HetArgs het_args(void* orbits, void* d_h, void* h_h, const void* coeffs, const int* ells,
                 const int* mms, const double* phi_ref, const double* inc, const double* lam,
                 const double* beta, const double* psi, const double* t_ref, double t_init,
                 const double* t_start, const double* t_end, const double* freqs, const void* h0,
                 const void* consts, int TDItag, int rescaled, int tdi2, int num_modes,
                 int length, int num_bin_all);
int het_check(void* orbits, int TDItag, int num_modes, int length, int precision);
static_assert(sizeof(HetArgs) % 8 == 0 && sizeof(FusedArgs) % 8 == 0,
              "argument blocks are copied in 8-byte words");

// Direct and heterodyned problems in ONE persistent launch of k_uneven (direct groups only:
// the same kernel with an empty walker range).  groups / hgroups: HOST arrays of descriptors
// (device pointers inside).
// The per-problem set-up of an uneven batch as one launch each over all problems: supports
// (block per (problem, binary)), uniform-grid checks (blockIdx.y = problem) and segment tables
// (thread per entry of the concatenated tables).
__global__ void k_support_multi(const MultiArgs* __restrict__ MA) {
  const long long gb = blockIdx.x;
  const int g = group_of(MA->boff, MA->ngroups, gb);
  const FusedArgs& A = MA->g[g];
  support_of(A.x, A.M, A.L, (int)(gb - MA->boff[g]), A.data_freqs, A.N,
             const_cast<int*>(A.sup_start), const_cast<int*>(A.sup_len));
}

__global__ void k_grid_detect_multi(const MultiArgs* __restrict__ MA) {
  const FusedArgs& A = MA->g[blockIdx.y];
  if (A.B == 0 || A.grid == nullptr) return;
  grid_detect_part(A.data_freqs, A.N, const_cast<GridInfo*>(A.grid), blockIdx.x, gridDim.x);
}

__global__ void k_tile_segments_multi(const MultiArgs* __restrict__ MA) {
  const long long n = MA->soff[MA->ngroups];
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int g = group_of(MA->soff, MA->ngroups, t);
    const FusedArgs& A = MA->g[g];
    const_cast<int2*>(A.segtab)[t - MA->soff[g]] = tile_segment_entry(
        t - MA->soff[g], A.x, A.data_freqs, A.sup_start, A.sup_len, A.B, A.M, A.L, A.tile);
  }
}

int uneven_like(const bbhx_direct_group* groups, int num_groups,
                       const bbhx_hdyn_group* hgroups, int num_het, int precision, int tile_bins,
                       int ctas_per_sm, cudaStream_t s) {
  BBHX_REQUIRE(num_groups >= 0 && num_groups <= FD_MAXGROUPS && (groups != nullptr || num_groups == 0),
               "num_direct must be 0..%d", FD_MAXGROUPS);
  BBHX_REQUIRE(num_het >= 0 && num_het <= FD_MAXGROUPS && (hgroups != nullptr || num_het == 0),
               "num_het must be 0..%d", FD_MAXGROUPS);
  BBHX_REQUIRE(num_groups + num_het >= 1, "no problems in the batch");
  BBHX_REQUIRE(precision == 0 || precision == 1, "precision must be 0 (FP64) or 1 (mixed)");
  BBHX_REQUIRE(tile_bins >= FD_WARP_BINS && tile_bins <= FD_WARP_BINS * FD_MAXCHUNK &&
                   tile_bins % FD_WARP_BINS == 0,
               "tile_bins must be a multiple of %d in [%d, %d]", FD_WARP_BINS, FD_WARP_BINS,
               FD_WARP_BINS * FD_MAXCHUNK);
  BBHX_REQUIRE(ctas_per_sm >= 1 && ctas_per_sm <= 32, "ctas_per_sm must be 1..32");
  // heterodyned problems: validated, walker offsets, the largest per-warp slice
  HetMulti HM;
  memset(&HM, 0, sizeof(HM));
  HM.ngroups = num_het;
  long long walkers = 0, records = 0;
  size_t het_slot = 0;
  for (int g = 0; g < num_het; ++g) {
    const bbhx_hdyn_group& H = hgroups[g];
    const int hs = het_check(H.orbits, H.TDItag, H.num_modes, H.length, precision);
    if (hs) return hs;
    BBHX_REQUIRE(H.num_bin_all >= 0, "heterodyned group %d: bad walker count %d", g, H.num_bin_all);
    HM.g[g] = het_args(H.orbits, H.d_h, H.h_h, H.coeffs, H.ells, H.mms, H.phi_ref, H.inc, H.lam,
                       H.beta, H.psi, H.t_ref, H.t_init, H.t_start, H.t_end, H.freqs, H.h0,
                       H.consts, H.TDItag, H.rescaled, H.tdi2, H.num_modes, H.length,
                       H.num_bin_all);
    HM.woff[g] = walkers;
    HM.roff[g] = records;
    walkers += H.num_bin_all;
    records += (long long)H.num_bin_all * H.num_modes;
    het_slot = std::max(het_slot, align16(HetSmemLayout(H.num_modes, H.length, false).total));
  }
  HM.woff[num_het] = walkers;
  HM.roff[num_het] = records;
  MultiArgs MA;
  memset(&MA, 0, sizeof(MA));
  MA.ngroups = num_groups;
  std::vector<void*> scratch;
  int st = OK;
  long long items = 0, bins = 0, entries = 0;
  for (int g = 0; g < num_groups && !st; ++g) {
    const bbhx_direct_group& G = groups[g];
    if (G.num_bin_all < 0 || G.length < 2 || G.num_modes < 1 || G.num_modes > FD_MAXM ||
        G.data_length < 1) {
      set_error("group %d: bad sizes (B=%d M=%d L=%d N=%d)", g, G.num_bin_all, G.num_modes,
                G.length, G.data_length);
      st = ERR_BAD_ARG;
      break;
    }
    FusedArgs& A = MA.g[g];
    A.data_freqs = G.data_freqs;
    A.data = (const cplx*)G.data;
    A.noise = G.noise;
    A.N = G.data_length;
    A.x = G.x;
    A.y = G.y;
    A.c1 = G.c1;
    A.c2 = G.c2;
    A.c3 = G.c3;
    A.t_start = G.t_start;
    A.t_end = G.t_end;
    A.B = G.num_bin_all;
    A.M = G.num_modes;
    A.L = G.length;
    A.tile = tile_bins;
    A.ntiles = (G.data_length + tile_bins - 1) / tile_bins;
    A.d_h = (double*)G.d_h;
    A.h_h = (double*)G.h_h;
    A.data32 = (const float2*)G.data32;
    A.noise32 = G.noise32;
    A.qstride = (long long)A.B * A.M * A.L;
    A.gh = nullptr;
    A.gh_off = nullptr;
    A.grid = nullptr;
    MA.off[g] = items;
    MA.boff[g] = bins;
    MA.soff[g] = entries;
    const long long nit = (long long)A.ntiles * A.B;
    items += nit;
    bins += A.B;
    if (A.B == 0) continue;
    entries += nit * A.M;
    int* sup = nullptr;
    double* part = nullptr;
    int2* segtab = nullptr;
    if (pool_alloc((void**)&sup, sizeof(int) * 2 * A.B, s) != cudaSuccess ||
        pool_alloc((void**)&part, sizeof(double) * 3 * nit, s) != cudaSuccess ||
        pool_alloc((void**)&segtab, sizeof(int2) * nit * A.M, s) != cudaSuccess) {
      set_error("device allocation for group %d failed", g);
      st = ERR_CUDA;
    }
    if (sup) scratch.push_back(sup);
    if (part) scratch.push_back(part);
    if (segtab) scratch.push_back(segtab);
    if (st) break;
    A.sup_start = sup;
    A.sup_len = sup + A.B;
    A.partials = part;
    A.segtab = segtab;
  }
  MA.off[num_groups] = items;
  MA.boff[num_groups] = bins;
  MA.soff[num_groups] = entries;
  // uniform-grid records of all problems in one array (one initialisation)
  GridInfo* grids = nullptr;
  if (!st && num_groups > 0) {
    if (pool_alloc((void**)&grids, sizeof(GridInfo) * num_groups, s) != cudaSuccess) {
      set_error("device allocation of the grid records failed");
      st = ERR_CUDA;
    } else {
      scratch.push_back(grids);
      for (int g = 0; g < num_groups; ++g)
        if (MA.g[g].B > 0) MA.g[g].grid = grids + g;
      st = cuda_status(cudaMemsetAsync(grids, 0xff, sizeof(GridInfo) * num_groups, s),
                       "grid record init");
    }
  }
  MultiArgs* dMA = nullptr;
  HetMulti* dHM = nullptr;
  if (!st) {
    if (pool_alloc((void**)&dMA, sizeof(MultiArgs), s) != cudaSuccess ||
        pool_alloc((void**)&dHM, sizeof(HetMulti), s) != cudaSuccess) {
      set_error("device allocation of the group tables failed");
      st = ERR_CUDA;
    }
    if (dMA) scratch.push_back(dMA);
    if (dHM) scratch.push_back(dHM);
    if (!st) {
      k_store_groups<<<1, 256, 0, s>>>(MA, dMA);
      st = launch_status("k_store_groups");
    }
    if (!st && bins > 0) {
      k_support_multi<<<(unsigned)bins, 128, 0, s>>>(dMA);
      st = launch_status("k_support_multi");
    }
    if (!st && bins > 0) {
      k_grid_detect_multi<<<dim3(std::max(1, sm_count() * 8 / std::max(1, num_groups)),
                                 num_groups), 256, 0, s>>>(dMA);
      st = launch_status("k_grid_detect_multi");
    }
    if (!st && entries > 0) {
      k_tile_segments_multi<<<grid_for(entries, 256, sm_count() * 64), 256, 0, s>>>(dMA);
      st = launch_status("k_tile_segments_multi");
    }
    // response-mode records of all walkers (scratch), then the walker table
    ResponseMode* rm = nullptr;
    if (!st && records > 0) {
      if (pool_alloc((void**)&rm, sizeof(ResponseMode) * records, s) != cudaSuccess) {
        set_error("device allocation of the response records failed");
        st = ERR_CUDA;
      } else {
        scratch.push_back(rm);
        for (int g = 0; g < num_het; ++g) HM.g[g].rmodes = rm + HM.roff[g];
      }
    }
    if (!st) {
      k_store_het<<<1, 256, 0, s>>>(HM, dHM);
      st = launch_status("k_store_het");
    }
    if (!st && records > 0) {
      k_het_response_setup_multi<<<grid_for(records, 128), 128, 0, s>>>(dHM, records);
      st = launch_status("k_het_response_setup_multi");
    }
  }
  if (!st && items + walkers > 0) {
    const int nsm = sm_count();
    const long long want = (items + walkers + FD_WARPS - 1) / FD_WARPS;
    const unsigned grid = (unsigned)std::min<long long>(want, (long long)nsm * ctas_per_sm);
    const size_t dslot = (precision == 1 ? fused_smem_bytes<true>() : fused_smem_bytes<false>()) / FD_WARPS;
    const size_t slot = align16(std::max(dslot, het_slot));
    const size_t sm = slot * FD_WARPS;
    unsigned long long* next = nullptr;
    if (pool_alloc((void**)&next, sizeof(unsigned long long), s) != cudaSuccess) {
      set_error("device allocation of the work-queue counter failed");
      st = ERR_CUDA;
    } else {
      scratch.push_back(next);
      st = cuda_status(cudaMemsetAsync(next, 0, sizeof(unsigned long long), s),
                       "work-queue counter");
    }
    auto launch = [&](auto kernel) {
      int r = cuda_status(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)sm),
                          "cudaFuncSetAttribute(k_uneven)");
      if (!r) kernel<<<grid, FD_WARPS * 32, sm, s>>>(dMA, dHM, (int)slot, next);
      return r;
    };
    if (!st && precision == 1)
      st = walkers > 0 ? launch(k_uneven<true, true>) : launch(k_uneven<true, false>);
    else if (!st)
      st = walkers > 0 ? launch(k_uneven<false, true>) : launch(k_uneven<false, false>);
    if (!st) st = launch_status("k_uneven");
  }
  if (!st && bins > 0) {
    k_fused_reduce_multi<<<grid_for(32LL * bins, 128), 128, 0, s>>>(dMA);
    st = launch_status("k_fused_reduce_multi");
  }
  for (void* p : scratch) pool_free(p, s);
  return st;
}

}  // namespace bbhx

extern "C" {

// Several direct-likelihood problems in one persistent launch of the fused kernel (k_uneven
// with no heterodyned problems).  groups: HOST array of descriptors (device pointers inside);
// tile_bins: data bins per work item (multiple of 128); ctas_per_sm: persistent CTAs per SM.
int bbhx_direct_like_multi(const bbhx_direct_group* groups, int num_groups, int precision,
                           int tile_bins, int ctas_per_sm, void* stream) {
  BBHX_REQUIRE(groups != nullptr && num_groups >= 1 && num_groups <= FD_MAXGROUPS,
               "num_groups must be 1..%d", FD_MAXGROUPS);
  return uneven_like(groups, num_groups, nullptr, 0, precision, tile_bins, ctas_per_sm,
                     (cudaStream_t)stream);
}

// Direct and heterodyned problems (uneven grid lengths, mode sets, observation spans, sparse
// grids) in one persistent launch (k_uneven).
int bbhx_uneven_like(const bbhx_direct_group* direct, int num_direct, const bbhx_hdyn_group* het,
                     int num_het, int precision, int tile_bins, int ctas_per_sm, void* stream) {
  return uneven_like(direct, num_direct, het, num_het, precision, tile_bins, ctas_per_sm,
                     (cudaStream_t)stream);
}

// Fused direct likelihood: d_h, h_h device complex128 [B] (overwritten, scaled by 4 like the
// reference), data [3, N] noise-weighted complex128, noise [3, N] = sqrt(df / S).
int bbhx_direct_like_fused(double* d_h, double* h_h, const double* data_freqs, const double* data,
                           const double* noise, int data_length, const double* x, const double* y,
                           const double* c1, const double* c2, const double* c3,
                           const double* t_start, const double* t_end, int num_modes, int length,
                           int num_bin_all, int precision, const void* data32,
                           const float* noise32, void* stream) {
  BBHX_REQUIRE(length >= 2 && num_modes >= 1 && data_length >= 1, "bad sizes");
  BBHX_REQUIRE(precision == 0 || precision == 1, "precision must be 0 (FP64) or 1 (mixed)");
  BBHX_REQUIRE((data32 == nullptr) == (noise32 == nullptr),
               "data32 and noise32 must be given together");
  BBHX_REQUIRE(num_modes <= FD_MAXM, "num_modes must be <= 6");
  if (num_bin_all == 0) return OK;
  cudaStream_t s = (cudaStream_t)stream;
  int ntiles = (data_length + FD_TILE - 1) / FD_TILE;
  long long nitems = (long long)ntiles * num_bin_all;
  int* sup = nullptr;
  double* part = nullptr;
  int2* segtab = nullptr;
  GridInfo* grid = nullptr;
  unsigned long long* next = nullptr;
  BBHX_CHECK_CUDA(pool_alloc_all(s, {{(void**)&sup, sizeof(int) * 2 * num_bin_all},
                                     {(void**)&part, sizeof(double) * 3 * nitems},
                                     {(void**)&segtab, sizeof(int2) * nitems * num_modes},
                                     {(void**)&grid, sizeof(GridInfo)},
                                     {(void**)&next, sizeof(unsigned long long)}}));
  k_support<<<num_bin_all, 128, 0, s>>>(x, num_modes, length, num_bin_all, data_freqs, data_length,
                                        sup, sup + num_bin_all);
  int st = launch_status("k_support");
  if (!st) st = detect_grid(data_freqs, data_length, grid, s);
  if (!st) {
    k_tile_segments<<<grid_for(nitems * num_modes, 256, sm_count() * 64), 256, 0, s>>>(
        segtab, x, data_freqs, sup, sup + num_bin_all, num_bin_all, num_modes, length, ntiles,
        FD_TILE);
    st = launch_status("k_tile_segments");
  }
  if (!st) {
    FusedArgs A;
    A.data_freqs = data_freqs;
    A.data = (const cplx*)data;
    A.noise = noise;
    A.N = data_length;
    A.x = x;
    A.y = y;
    A.c1 = c1;
    A.c2 = c2;
    A.c3 = c3;
    A.t_start = t_start;
    A.t_end = t_end;
    A.sup_start = sup;
    A.sup_len = sup + num_bin_all;
    A.B = num_bin_all;
    A.M = num_modes;
    A.L = length;
    A.ntiles = ntiles;
    A.tile = FD_TILE;
    A.partials = part;
    A.segtab = segtab;
    A.d_h = d_h;
    A.h_h = h_h;
    A.data32 = (precision == 1) ? (const float2*)data32 : nullptr;
    A.noise32 = (precision == 1) ? noise32 : nullptr;
    A.qstride = (long long)num_bin_all * num_modes * length;
    A.gh = nullptr;
    A.gh_off = nullptr;
    A.grid = grid;
    A.next = next;
    st = cuda_status(cudaMemsetAsync(next, 0, sizeof(unsigned long long), s), "work-queue counter");
    auto launch = [&](auto kernel, size_t sm, const char* what) {
      int r = cuda_status(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)sm),
                          what);
      if (!r) kernel<<<resident_grid(kernel, sm, nitems), FD_WARPS * 32, sm, s>>>(A);
      return r;
    };
    if (!st)
      st = (precision == 1)
               ? launch(k_direct_fused<true>, fused_smem_bytes<true>(),
                        "cudaFuncSetAttribute(k_direct_fused<true>)")
               : launch(k_direct_fused<false>, fused_smem_bytes<false>(),
                        "cudaFuncSetAttribute(k_direct_fused<false>)");
    if (!st) st = launch_status("k_direct_fused");
  }
  if (!st) {
    k_fused_reduce<<<grid_for(32LL * num_bin_all, 128), 128, 0, s>>>(part, sup, sup + num_bin_all,
                                                              num_bin_all, d_h, h_h);
    st = launch_status("k_fused_reduce");
  }
  pool_free(sup, s);
  pool_free(part, s);
  pool_free(segtab, s);
  pool_free(grid, s);
  pool_free(next, s);
  return st;
}

}  // extern "C"
