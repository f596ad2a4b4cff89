// Algorithmic operation count of one heterodyne point evaluation (diagnostic; no counterpart in
// the reference).
//
// The waveform and response models are templated on their scalar type (phenomhm_model.cuh,
// response_model.cuh).  Instantiated here with an op-counting scalar, one thread runs the FP64
// per-point chain of the fused heterodyned kernel -- PhenomHM amplitude, phase and t(f) at one
// frequency of one mode, the TDI transfer at (f, t(f)), the waveform phasor e^{i phase} and the
// three channel products -- and tallies every arithmetic operation and elementary-function
// call.  The per-(binary, mode) set-up (fit coefficients, QNM frequencies, the response mode
// matrix) is excluded: it is amortised over the sparse grid.  bench.py turns the tally into
// the heterodyned path's algorithmic FP64 rate.
#include "capi_internal.cuh"
#include "phenomhm_model.cuh"
#include "response_model.cuh"

namespace bbhx {
namespace opc {

// tallies: 0 add/sub, 1 mul, 2 div, 3 compare, 4 sqrt, 5 cbrt, 6 log, 7 exp, 8 pow,
// 9 atan, 10 sin/cos/sincos, 11 fabs/floor/hypot (other)
constexpr int NCAT = 12;
__device__ unsigned long long g_tally[NCAT];

__device__ __forceinline__ void tick(int k) { g_tally[k] += 1; }

struct Cnt {
  double v;
  __device__ __forceinline__ Cnt() {}
  __device__ __forceinline__ Cnt(double x) : v(x) {}
};

__device__ __forceinline__ Cnt operator+(const Cnt& a, const Cnt& b) { tick(0); return Cnt(a.v + b.v); }
__device__ __forceinline__ Cnt operator-(const Cnt& a, const Cnt& b) { tick(0); return Cnt(a.v - b.v); }
__device__ __forceinline__ Cnt operator*(const Cnt& a, const Cnt& b) { tick(1); return Cnt(a.v * b.v); }
__device__ __forceinline__ Cnt operator/(const Cnt& a, const Cnt& b) { tick(2); return Cnt(a.v / b.v); }
__device__ __forceinline__ Cnt operator-(const Cnt& a) { return Cnt(-a.v); }
__device__ __forceinline__ Cnt operator+(const Cnt& a, double b) { tick(0); return Cnt(a.v + b); }
__device__ __forceinline__ Cnt operator+(double a, const Cnt& b) { tick(0); return Cnt(a + b.v); }
__device__ __forceinline__ Cnt operator-(const Cnt& a, double b) { tick(0); return Cnt(a.v - b); }
__device__ __forceinline__ Cnt operator-(double a, const Cnt& b) { tick(0); return Cnt(a - b.v); }
__device__ __forceinline__ Cnt operator*(const Cnt& a, double b) { tick(1); return Cnt(a.v * b); }
__device__ __forceinline__ Cnt operator*(double a, const Cnt& b) { tick(1); return Cnt(a * b.v); }
__device__ __forceinline__ Cnt operator/(const Cnt& a, double b) { tick(2); return Cnt(a.v / b); }
__device__ __forceinline__ Cnt operator/(double a, const Cnt& b) { tick(2); return Cnt(a / b.v); }
template <typename S>
__device__ __forceinline__ Cnt& operator+=(Cnt& a, const S& b) { a = a + b; return a; }
template <typename S>
__device__ __forceinline__ Cnt& operator-=(Cnt& a, const S& b) { a = a - b; return a; }
template <typename S>
__device__ __forceinline__ Cnt& operator*=(Cnt& a, const S& b) { a = a * b; return a; }
template <typename S>
__device__ __forceinline__ Cnt& operator/=(Cnt& a, const S& b) { a = a / b; return a; }

#define BBHX_CNT_CMP(op)                                                                       \
  __device__ __forceinline__ bool operator op(const Cnt& a, const Cnt& b) { tick(3); return a.v op b.v; } \
  __device__ __forceinline__ bool operator op(const Cnt& a, double b) { tick(3); return a.v op b; }        \
  __device__ __forceinline__ bool operator op(double a, const Cnt& b) { tick(3); return a op b.v; }
BBHX_CNT_CMP(<)
BBHX_CNT_CMP(>)
BBHX_CNT_CMP(<=)
BBHX_CNT_CMP(>=)
BBHX_CNT_CMP(==)
BBHX_CNT_CMP(!=)
#undef BBHX_CNT_CMP

__device__ __forceinline__ Cnt sqrt(const Cnt& x) { tick(4); return Cnt(::sqrt(x.v)); }
__device__ __forceinline__ Cnt cbrt(const Cnt& x) { tick(5); return Cnt(::cbrt(x.v)); }
__device__ __forceinline__ Cnt log(const Cnt& x) { tick(6); return Cnt(::log(x.v)); }
__device__ __forceinline__ Cnt exp(const Cnt& x) { tick(7); return Cnt(::exp(x.v)); }
__device__ __forceinline__ Cnt pow(const Cnt& x, double p) { tick(8); return Cnt(::pow(x.v, p)); }
__device__ __forceinline__ Cnt atan(const Cnt& x) { tick(9); return Cnt(::atan(x.v)); }
__device__ __forceinline__ Cnt sin(const Cnt& x) { tick(10); return Cnt(::sin(x.v)); }
__device__ __forceinline__ Cnt cos(const Cnt& x) { tick(10); return Cnt(::cos(x.v)); }
__device__ __forceinline__ void sincos(const Cnt& x, Cnt* s, Cnt* c) {
  tick(10);
  double sv, cv;
  ::sincos(x.v, &sv, &cv);
  *s = Cnt(sv);
  *c = Cnt(cv);
}
__device__ __forceinline__ Cnt fabs(const Cnt& x) { tick(11); return Cnt(::fabs(x.v)); }
__device__ __forceinline__ Cnt hypot(const Cnt& a, const Cnt& b) { tick(11); return Cnt(::hypot(a.v, b.v)); }
__device__ __forceinline__ double floor(const Cnt& x) { tick(11); return ::floor(x.v); }
// value part (found by argument-dependent lookup from the templated model)
__device__ __forceinline__ double value_of(const Cnt& x) { return x.v; }

}  // namespace opc

// One thread: set up (binary, mode) records from the parameters, then for each of the L
// frequencies of each of the M modes evaluate the point chain and add its tallies to out
// [NCAT] (set-up tallies excluded).  params: m1, m2 [Msun], chi1z, chi2z, distance [m],
// phi_ref, inc, lam, beta, psi, t_ref; ringdown frequencies computed as the forward path does.
__global__ void k_count_point_ops(unsigned long long* out, const double* prm, const int* ells,
                                  const int* mms, int M, const double* freqs, int L,
                                  const double* qnm, int nq, double dspin, OrbitTables orb,
                                  int TDItag, int rescaled, int tdi2) {
  using C = opc::Cnt;
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int k = 0; k < opc::NCAT; ++k) out[k] = 0;
  const C m1(prm[0]), m2(prm[1]), chi1(prm[2]), chi2(prm[3]), dist(prm[4]);
  const C phi_ref(prm[5]), inc(prm[6]), lam(prm[7]), beta(prm[8]), psi(prm[9]);
  const double t_ref = prm[10];
  C fm, fs;
  final_mass_spin(m1, m2, chi1, chi2, &fm, &fs);
  const int ind = int((fs.v + 1.0) / dspin);
  const C x = fs - (dspin * ind - 1.0);
  const C x2 = x * x, x3 = x2 * x;
  const C rd22 = (qnm[ind] + qnm[nq + ind] * x + qnm[2 * nq + ind] * x2 + qnm[3 * nq + ind] * x3) / fm;
  const double* dm = qnm + 4 * (size_t)nq;
  const C dm22 = (dm[ind] + dm[nq + ind] * x + dm[2 * nq + ind] * x2 + dm[3 * nq + ind] * x3) / fm;
  for (int i = 0; i < M; ++i) {
    const cplxT<C> z = qnm_cw(fs, ells[i], mms[i]);
    const C rd = (0.5 / PI) * z.re / fm, dd = (0.5 / PI) * z.im / fm;
    ModeCoeffsT<C> c;
    phm_setup_mode(c, m1 * MSUN_SI, m2 * MSUN_SI, chi1, chi2, dist, ells[i], mms[i], rd, dd, rd22,
                   dm22, 0);
    ResponseModeT<C> r;
    response_mode_setup(r, ells[i], mms[i], phi_ref, inc, lam, beta, psi);
    for (int k = 0; k < opc::NCAT; ++k) opc::g_tally[k] = 0;
    for (int j = 0; j < L; ++j) {
      const double f = freqs[j];
      PointOutT<C> w = phm_eval_point(c, C(f));
      w.phase = w.phase + f * (t_ref - 0.0) * 2 * PI;
      w.tf = w.tf + t_ref;
      const TransferT<C> T = response_point(r, orb, f, w.tf, TDItag, rescaled, tdi2);
      const cplxT<C> ap = w.amp * expi(w.phase + T.phaseRdelay);
      const cplxT<C> Tc[3] = {T.L1, T.L2, T.L3};
      C h[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      for (int ch = 0; ch < 3; ++ch) {
        const cplxT<C> v = Tc[ch] * ap;
        h[2 * ch] += v.re;
        h[2 * ch + 1] -= v.im;
      }
    }
    for (int k = 0; k < opc::NCAT; ++k) out[k] += opc::g_tally[k];
  }
}

}  // namespace bbhx

using namespace bbhx;

extern "C" {

// Diagnostic: tallies of the FP64 heterodyne point chain summed over the M modes and L
// frequencies (out [12] device: add/sub, mul, div, compare, sqrt, cbrt, log, exp, pow, atan,
// sin-cos, other); params [11] device (see k_count_point_ops).  Single thread, for
// measurement only.
int bbhx_count_point_ops(void* orbits, unsigned long long* out, const double* params,
                         const int* ells, const int* mms, int num_modes, const double* freqs,
                         int length, const double* qnm_table, int qnm_n, double dspin, int TDItag,
                         int rescaled, int tdi2, void* stream) {
  BBHX_REQUIRE(orbits && ((OrbitHandle*)orbits)->ready, "orbit information not added");
  BBHX_REQUIRE(num_modes >= 1 && num_modes <= 6 && length >= 1, "bad sizes");
  k_count_point_ops<<<1, 32, 0, (cudaStream_t)stream>>>(out, params, ells, mms, num_modes, freqs,
                                                        length, qnm_table, qnm_n, dspin,
                                                        ((OrbitHandle*)orbits)->tab, TDItag,
                                                        rescaled, tdi2);
  return launch_status("k_count_point_ops");
}

}  // extern "C"
