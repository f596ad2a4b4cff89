// Shared definitions for the bbhx_b200 CUDA kernels (sm_100a).
//
// Constants are the reference's (src/bbhx/cutils/constants.h:6-60); they must match
// bit-for-bit for parity.  Complex numbers are a plain {re, im} pair of doubles (or
// floats) laid out like numpy complex128 / complex64, so caller buffers can be
// reinterpreted without copies.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace bbhx {

constexpr double MSUN_SI = 1.98848e+30;
constexpr double YRSID_SI = 31558149.763545603;
constexpr double AU_SI = 149597870700.0;
constexpr double C_SI = 299792458.;
constexpr double MTSUN_SI = 4.925491025873693e-06;
constexpr double MRSUN_SI = 1476.6250615036158;
constexpr double PC_SI = 3.0856775814913674e+16;
constexpr double PI = 3.141592653589793238462643383279502884;
constexpr double PI_2 = 1.570796326794896619231321691639751442;
constexpr double PI_4 = 0.785398163397448309615660845819875721;
constexpr double TWO_PI = 6.283185307179586476925286766559005768;
constexpr double GAMMA_E = 0.577215664901532860606512090082402431;
constexpr double SQRT2 = 1.414213562373095048801688724209698079;
constexpr double INVSQRT3 = 0.577350269189625764509148780501957455;
constexpr double INVSQRT6 = 0.408248290463863016366214012450981898;
constexpr double Omega0 = 1.9909865927683788e-07;

// status codes returned by every C-ABI entry point (3 is unused: no kernel of the library
// waits on another CTA, stream or device, so nothing can time out)
enum Status : int {
  OK = 0,
  ERR_BAD_ARG = 1,
  ERR_CUDA = 2,
  ERR_NONFINITE = 4,
  ERR_NO_ORBITS = 5,
  ERR_TOO_LARGE = 6,
};

// The calling warp's next work item from a launch's queue counter (zero at launch).  Items are
// handed out in increasing order, so the warps in flight stay on neighbouring items; a warp that
// finishes a cheap item takes the next one at once, so the resident warps stay busy until the
// queue drains however unequal the items are.  Every lane of the warp must call it.
__device__ __forceinline__ long long claim_item(unsigned long long* next, int lane) {
  unsigned long long q = 0;
  if (lane == 0) q = atomicAdd(next, 1ull);
  return (long long)__shfl_sync(0xffffffffu, q, 0);
}

// Set *word when any of the values is NaN or infinite (the sum is non-finite then).
__device__ __forceinline__ void note_nonfinite(unsigned* word, double a, double b, double c,
                                               double d) {
  if (!isfinite(a + b + c + d)) atomicOr(word, 1u);
}

// Complex numbers over any real scalar T (double, float, or the dual numbers of the
// gradient kernels).  In the scalar products the scalar is converted to T, so double
// constants multiply dual-number complexes directly.
template <typename T>
struct cplxT {
  T re, im;
};
using cplx = cplxT<double>;
using cplxf = cplxT<float>;

template <typename T>
struct ident {
  using type = T;
};

__host__ __device__ __forceinline__ cplx mk(double r, double i) { return cplx{r, i}; }
template <typename T>
__host__ __device__ __forceinline__ cplxT<T> cmk(const T& r, const T& i) {
  return cplxT<T>{r, i};
}
template <typename T>
__host__ __device__ __forceinline__ cplxT<T> operator+(const cplxT<T>& a, const cplxT<T>& b) {
  return {a.re + b.re, a.im + b.im};
}
template <typename T>
__host__ __device__ __forceinline__ cplxT<T> operator-(const cplxT<T>& a, const cplxT<T>& b) {
  return {a.re - b.re, a.im - b.im};
}
template <typename T>
__host__ __device__ __forceinline__ cplxT<T> operator*(const cplxT<T>& a, const cplxT<T>& b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename T>
__host__ __device__ __forceinline__ cplxT<T> operator*(typename ident<T>::type s,
                                                       const cplxT<T>& a) {
  return {s * a.re, s * a.im};
}
template <typename T>
__host__ __device__ __forceinline__ cplxT<T> operator*(const cplxT<T>& a,
                                                       typename ident<T>::type s) {
  return {s * a.re, s * a.im};
}
template <typename T>
__host__ __device__ __forceinline__ cplxT<T> conj(const cplxT<T>& a) {
  return {a.re, -a.im};
}
template <typename T>
__host__ __device__ __forceinline__ cplxT<T> times_i(const cplxT<T>& a) {
  return {-a.im, a.re};
}
template <typename T>
__device__ __forceinline__ cplxT<T> expi(const T& x) {
  T s, c;
  sincos(x, &s, &c);
  return {c, s};
}
__device__ __forceinline__ double cabs(cplx a) { return hypot(a.re, a.im); }

// Phase reduction to [-pi, pi]: k = rint(x / 2pi), then x - k*2pi with 2pi split into a
// double (hi) and its residual (lo); each FMA forms k*part exactly before its single
// rounding, so the reduced angle is good to a few ulp of pi for |x| far beyond the
// 1e7 rad that waveform phases reach.
__device__ __forceinline__ double reduce_2pi(double x) {
  const double INV2PI = 0.15915494309189533577;
  const double TWO_PI_HI = 6.28318530717958623200e+00;   // 2*pi rounded to double
  const double TWO_PI_LO = 2.44929359829470635446e-16;   // 2*pi - TWO_PI_HI
  double k = rint(x * INV2PI);
  double r = fma(-k, TWO_PI_HI, x);
  r = fma(-k, TWO_PI_LO, r);
  return r;
}

// sin and cos of an FP64 angle of any size met here (|x| up to ~1e9 rad) for the hot loops.
// Method: Cody-Waite reduction by pi/2 with pi/2 split into three doubles P1 + P2 + P3 (each
// FMA forms k*P_i exactly before its one rounding), k from the exact product x * 2/pi rounded
// by adding 1.5 * 2^52 (its low bits give k mod 4), then the Taylor series of sin and cos on
// the reduced angle |y| <= pi/4 (+ half an ulp of k), truncated after the y^17 / y^18 terms (truncation below
// 3e-19), evaluated by Horner's rule, and the quadrant k mod 4 applied by swapping / negating.
// Accuracy ~1e-16 absolute; checked against CUDA's sincos in tests/test_gpu_kernels.py.
__device__ __forceinline__ void sincos_cw(double x, double* s, double* c, double x_lo = 0.0) {
  const double TWO_OVER_PI = 0.6366197723675814;
  const double P1 = 1.5707963267948966;
  const double P2 = 6.123233995736766e-17;
  const double P3 = -1.4973849048591698e-33;
  const double MAGIC = 6755399441055744.0;  // 1.5 * 2^52: rounds to an integer, |x| < 2^50
  const double t = fma(x, TWO_OVER_PI, MAGIC);
  const double k = t - MAGIC;
  double y = fma(-k, P1, x);
  y = fma(-k, P2, y);
  y = fma(-k, P3, y);
  y += x_lo;  // angle given as x + x_lo (|x_lo| <= a few ulp of x): folded in after the reduction
  double y2 = y * y;
  double ps = 2.8114572543455206e-15;
  ps = fma(ps, y2, -7.647163731819816e-13);
  ps = fma(ps, y2, 1.6059043836821613e-10);
  ps = fma(ps, y2, -2.505210838544172e-08);
  ps = fma(ps, y2, 2.7557319223985893e-06);
  ps = fma(ps, y2, -0.0001984126984126984);
  ps = fma(ps, y2, 0.008333333333333333);
  ps = fma(ps, y2, -0.16666666666666666);
  double sy = fma(ps * y2, y, y);
  double pc = -1.5619206968586225e-16;
  pc = fma(pc, y2, 4.779477332387385e-14);
  pc = fma(pc, y2, -1.1470745597729725e-11);
  pc = fma(pc, y2, 2.08767569878681e-09);
  pc = fma(pc, y2, -2.755731922398589e-07);
  pc = fma(pc, y2, 2.48015873015873e-05);
  pc = fma(pc, y2, -0.001388888888888889);
  pc = fma(pc, y2, 0.041666666666666664);
  pc = fma(pc, y2, -0.5);
  double cy = fma(pc, y2, 1.0);
  const int q = __double2loint(t) & 3;
  double ss = (q & 1) ? cy : sy;
  double cc = (q & 1) ? sy : cy;
  *s = (q & 2) ? -ss : ss;
  *c = ((q + 1) & 2) ? -cc : cc;
}

// sin / cos in FP32 of an FP64 angle: the quadrant reduction by pi/2 stays in FP64 (the
// angle reaches ~1e7 rad), the reduced |y| <= pi/4 goes to FP32 Taylor polynomials
// (through y^9 and y^10; truncation < 2e-9).
__device__ __forceinline__ void sincos_mixed(double x, float* s, float* c) {
  const double TWO_OVER_PI = 0.6366197723675814;
  // k = nearest integer to x * 2/pi by adding 1.5 * 2^52 (valid for |x| < 2^50); the quadrant
  // k mod 4 is then the low bits of the sum (no float-to-integer conversion needed)
  const double MAGIC = 6755399441055744.0;
  const double t = fma(x, TWO_OVER_PI, MAGIC);
  const double k = t - MAGIC;
  double yd = fma(-k, 1.5707963267948966, x);
  yd = fma(-k, 6.123233995736766e-17, yd);
  float y = (float)yd;
  float y2 = y * y;
  float ps = fmaf(fmaf(fmaf(2.7557319e-06f, y2, -1.9841270e-04f), y2, 8.3333333e-03f), y2,
                  -1.6666667e-01f);
  float sy = fmaf(ps * y2, y, y);
  float pc = fmaf(fmaf(fmaf(fmaf(-2.7557319e-07f, y2, 2.4801587e-05f), y2, -1.3888889e-03f), y2,
                       4.1666667e-02f), y2, -0.5f);
  float cy = fmaf(pc, y2, 1.0f);
  const int q = __double2loint(t) & 3;
  float ss = (q & 1) ? cy : sy;
  float cc = (q & 1) ? sy : cy;
  *s = (q & 2) ? -ss : ss;
  *c = ((q + 1) & 2) ? -cc : cc;
}

}  // namespace bbhx
