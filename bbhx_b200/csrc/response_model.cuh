// Fast frequency-domain LISA TDI response (device side).
//
// Follows the reference's response (src/bbhx/cutils/Response.cu), i.e. the
// Marsat & Baker fast FD response (arXiv:1806.10734, 2003.00357):
//   * per (binary, mode): wave vector k, polarisation tensors H+ / Hx rotated into the
//     SSB frame, and the complex mode matrix H = Y+ H+ + Yx Hx from the spin-weighted
//     spherical harmonics (Response.cu:468-608);
//   * per (binary, mode, frequency): single-link transfer functions G_slr at the
//     spacecraft positions for time t = t(f) (Response.cu:54-194), combined into
//     XYZ or AET (optionally 2nd-generation) TDI (Response.cu:197-261), plus the
//     orbital Roemer delay 2 pi f k.R / c added to the phase (Response.cu:264-314).
// The per-(binary, mode) part is computed once (ResponseMode) instead of by thread 0 of
// every block; the orbit tables are read through the __ldg path.
//
// Orbit tables (bbhx_b200/orbits.py): x_arr[N][3][3], n_arr[N][6][3], link order
// links[6]; sample k at t = k dt; linear interpolation for 0 <= floor(t/dt) < N-1, zero
// vector outside.  The window and its fraction are found once per time and shared by the six
// vectors read there.
#pragma once

#include "bbhx_common.cuh"
#include "dual.cuh"

namespace bbhx {

struct OrbitTables {
  const double* x_arr;  // [N][3][3]
  const double* n_arr;  // [N][6][3]
  double dt;
  double inv_dt;  // 1 / dt
  int N;
  int link_index[3];  // table slots of links 12, 23, 31
  double armlength;
  double inv_armlength;  // 1 / armlength
  double pi_L_over_c;    // pi armlength / c
};

// Device-resident orbit tables owned by the C-ABI orbit handle (bbhx_orbits_*).
struct OrbitHandle {
  double* d_x = nullptr;
  double* d_n = nullptr;
  OrbitTables tab{};
  bool ready = false;
};

template <typename T>
struct ResponseModeT {
  cplxT<T> H[9];  // complex mode matrix, row-major
  T k[3];         // propagation direction
};
using ResponseMode = ResponseModeT<double>;


template <typename T>
struct V3T {
  T x, y, z;
};

// Table window of time t: w = floor(t / dt) (the lookup rule), valid for 0 <= w < N - 1, and the
// interpolation fraction (t - w dt) / dt shared by all vectors read at that time.
template <typename T>
struct OrbitWindow {
  const double* x_lo;  // first x row of the window (nullptr when outside the table)
  const double* n_lo;
  T frac;
};

template <typename T>
__device__ __forceinline__ OrbitWindow<T> orbit_window(const OrbitTables& orb, const T& t) {
  OrbitWindow<T> w;
  const double f = floor(value_of(t) / orb.dt);
  if (!(f >= 0.0) || f >= (double)(orb.N - 1)) {
    w.x_lo = nullptr;
    w.n_lo = nullptr;
    w.frac = T(0.0);
    return w;
  }
  const int wi = (int)f;
  w.x_lo = orb.x_arr + (size_t)wi * 9;
  w.n_lo = orb.n_arr + (size_t)wi * 18;
  w.frac = (t - wi * orb.dt) * orb.inv_dt;
  return w;
}

// lo + (hi - lo) * frac of the 3-vector at `offset` of rows lo and lo + stride; zero vector
// outside the table.
template <typename T>
__device__ __forceinline__ V3T<T> orbit_lerp(const double* lo, int stride, int offset,
                                             const T& frac) {
  if (lo == nullptr) return V3T<T>{T(0.0), T(0.0), T(0.0)};
  lo += offset;
  const double* hi = lo + stride;
  V3T<T> r;
  r.x = __ldg(lo + 0) + (__ldg(hi + 0) - __ldg(lo + 0)) * frac;
  r.y = __ldg(lo + 1) + (__ldg(hi + 1) - __ldg(lo + 1)) * frac;
  r.z = __ldg(lo + 2) + (__ldg(hi + 2) - __ldg(lo + 2)) * frac;
  return r;
}
// spin-weight -2 spherical harmonics for l = 2..4 (Response.cu:383-424)
template <typename T>
__device__ inline cplxT<T> sylm_m2(int l, int m, const T& theta, const T& phi) {
  T fac = 0.0;
  T ct = cos(theta), st = sin(theta);
  T c2 = cos(theta / 2.0), s2 = sin(theta / 2.0);
  if (l == 2) {
    if (m == -2) fac = sqrt(5.0 / (64.0 * PI)) * (1.0 - ct) * (1.0 - ct);
    else if (m == -1) fac = sqrt(5.0 / (16.0 * PI)) * st * (1.0 - ct);
    else if (m == 1) fac = sqrt(5.0 / (16.0 * PI)) * st * (1.0 + ct);
    else if (m == 2) fac = sqrt(5.0 / (64.0 * PI)) * (1.0 + ct) * (1.0 + ct);
  } else if (l == 3) {
    if (m == -3) fac = sqrt(21.0 / (2.0 * PI)) * c2 * pow(s2, 5.0);
    else if (m == -2) fac = sqrt(7.0 / (4.0 * PI)) * (2.0 + 3.0 * ct) * pow(s2, 4.0);
    else if (m == 2) fac = sqrt(7.0 / PI) * pow(c2, 4.0) * (-2.0 + 3.0 * ct) / 2.0;
    else if (m == 3) fac = -sqrt(21.0 / (2.0 * PI)) * pow(c2, 5.0) * s2;
  } else if (l == 4) {
    if (m == -4) fac = 3.0 * sqrt(7.0 / PI) * pow(c2, 2.0) * pow(s2, 6.0);
    else if (m == -3) fac = 3.0 * sqrt(7.0 / (2.0 * PI)) * c2 * (1.0 + 2.0 * ct) * pow(s2, 5.0);
    else if (m == 3) fac = -3.0 * sqrt(7.0 / (2.0 * PI)) * pow(c2, 5.0) * (-1.0 + 2.0 * ct) * s2;
    else if (m == 4) fac = 3.0 * sqrt(7.0 / PI) * pow(c2, 6.0) * pow(s2, 2.0);
  }
  if (m == 0) return cmk(fac, T(0.0));
  T s, c;
  sincos(m * phi, &s, &c);
  return cmk(fac * c, fac * s);
}

template <typename T>
__device__ inline void response_mode_setup(ResponseModeT<T>& r, int ell, int mm, const T& phi_ref,
                                           const T& inc, const T& lam, const T& beta,
                                           const T& psi) {
  T cl = cos(lam), sl = sin(lam), cb = cos(beta), sb = sin(beta), cp = cos(psi), sp = sin(psi);
  r.k[0] = -cb * cl;
  r.k[1] = -cb * sl;
  r.k[2] = -sb;
  // rotation from the wave frame to the SSB frame and its inverse
  T O[9] = {cp * sl - cl * sb * sp, -cl * cp * sb - sl * sp, -cb * cl,
            -cl * cp - sb * sl * sp, -cp * sb * sl + cl * sp, -cb * sl,
            cb * sp, cb * cp, -sb};
  T Oi[9] = {O[0], O[3], O[6], O[1], O[4], O[7], O[2], O[5], O[8]};
  // H+ = O diag(1,-1,0) O^-1, Hx = O offdiag(1,1) O^-1
  T Hp[9], Hc[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      // (HS+ O^-1)_{kj} = s_k Oi[k][j] with s = (1,-1,0); (HSx O^-1)_{0j} = Oi[1][j], _{1j} = Oi[0][j]
      T p = O[i * 3 + 0] * Oi[0 * 3 + j] - O[i * 3 + 1] * Oi[1 * 3 + j];
      T x = O[i * 3 + 0] * Oi[1 * 3 + j] + O[i * 3 + 1] * Oi[0 * 3 + j];
      Hp[i * 3 + j] = p;
      Hc[i * 3 + j] = x;
    }
  cplxT<T> Ylm = sylm_m2(ell, mm, inc, phi_ref);
  cplxT<T> Ylmm = sylm_m2(ell, -mm, inc, phi_ref);
  double sgn = (ell % 2 == 0) ? 1.0 : -1.0;
  cplxT<T> Yl_m = sgn * conj(Ylmm);
  cplxT<T> Yp = 0.5 * (Ylm + Yl_m);
  cplxT<T> Yc = times_i(0.5 * (Ylm - Yl_m));
  for (int q = 0; q < 9; ++q) r.H[q] = Yp * Hp[q] + Yc * Hc[q];
}

template <typename T>
struct TransferT {
  cplxT<T> L1, L2, L3;
  T phaseRdelay;
};
using Transfer = TransferT<double>;

template <typename T>
__device__ __forceinline__ cplxT<T> nHn(const cplxT<T>* H, const V3T<T>& n) {
  T v[3] = {n.x, n.y, n.z};
  cplxT<T> out = cmk(T(0.0), T(0.0));
  for (int i = 0; i < 3; ++i) {
    cplxT<T> t = cmk(T(0.0), T(0.0));
    for (int j = 0; j < 3; ++j) t = t + H[i * 3 + j] * v[j];
    out = out + v[i] * t;
  }
  return out;
}

template <typename T>
__device__ __forceinline__ T sinc(const T& x) { return x == 0.0 ? T(1.0) : sin(x) / x; }

// TDItag: 1 = XYZ, 2 = AET.  f in Hz, t in s.  The frequency has its own type F: double, or
// the dual type T when the frequency itself carries tangents (knots that move with theta).
template <typename T, typename F = double>
__device__ inline TransferT<T> response_point(const ResponseModeT<T>& r, const OrbitTables& orb,
                                              const F& f, const T& t, int TDItag, int rescaled,
                                              int tdi2) {
  const T* k = r.k;
  // Roemer delay relative to the SSB (circular 1 AU orbit of the guiding centre)
  T al = Omega0 * t;
  T sa, ca;
  sincos(al, &sa, &ca);
  T kR = k[0] * (AU_SI * ca) + k[1] * (AU_SI * sa) + k[2] * (0.0 * t);
  TransferT<T> out;
  out.phaseRdelay = 2. * PI / C_SI * f * kR;

  const OrbitWindow<T> win = orbit_window(orb, t);
  V3T<T> p1 = orbit_lerp(win.x_lo, 9, 0, win.frac);
  V3T<T> p2 = orbit_lerp(win.x_lo, 9, 3, win.frac);
  V3T<T> p3 = orbit_lerp(win.x_lo, 9, 6, win.frac);
  V3T<T> n1 = orbit_lerp(win.n_lo, 18, orb.link_index[0] * 3, win.frac);
  V3T<T> n2 = orbit_lerp(win.n_lo, 18, orb.link_index[1] * 3, win.frac);
  V3T<T> n3 = orbit_lerp(win.n_lo, 18, orb.link_index[2] * 3, win.frac);
  T kn1 = k[0] * n1.x + k[1] * n1.y + k[2] * n1.z;
  T kn2 = k[0] * n2.x + k[1] * n2.y + k[2] * n2.z;
  T kn3 = k[0] * n3.x + k[1] * n3.y + k[2] * n3.z;
  cplxT<T> n1H = nHn(r.H, n1), n2H = nHn(r.H, n2), n3H = nHn(r.H, n3);
  T k12 = k[0] * (p1.x + p2.x) + k[1] * (p1.y + p2.y) + k[2] * (p1.z + p2.z);
  T k23 = k[0] * (p2.x + p3.x) + k[1] * (p2.y + p3.y) + k[2] * (p2.z + p3.z);
  T k31 = k[0] * (p3.x + p1.x) + k[1] * (p3.y + p1.y) + k[2] * (p3.z + p1.z);
  const double invL = orb.inv_armlength;
  T pre = f * orb.pi_L_over_c;
  cplxT<T> e12 = expi(pre * (1. + k12 * invL));
  cplxT<T> e23 = expi(pre * (1. + k23 * invL));
  cplxT<T> e31 = expi(pre * (1. + k31 * invL));
  // The constellation-centre phase factor exp(+i 2 pi f k.p0 / c) of the full response and
  // the Roemer-delay factor exp(-i phaseRdelay) cancel identically (Response.cu:166,304-309).
  cplxT<T> common = cmk(T(0.0), pre);
  cplxT<T> c3 = common * n3H, c1 = common * n1H, c2 = common * n2H;
  cplxT<T> G12 = c3 * (sinc(pre * (1. - kn3)) * e12);
  cplxT<T> G21 = c3 * (sinc(pre * (1. + kn3)) * e12);
  cplxT<T> G23 = c1 * (sinc(pre * (1. - kn1)) * e23);
  cplxT<T> G32 = c1 * (sinc(pre * (1. + kn1)) * e23);
  cplxT<T> G31 = c2 * (sinc(pre * (1. - kn2)) * e31);
  cplxT<T> G13 = c2 * (sinc(pre * (1. + kn2)) * e31);

  // e^{ix}, x = pre, and its powers / sines from one sincos
  const cplxT<T> e1 = expi(pre);
  const cplxT<T> z = e1 * e1;  // e^{2ix}
  const T s2x = 2. * e1.im * e1.re;
  if (TDItag == 1) {
    cplxT<T> fac = rescaled ? cmk(T(1.0), T(0.0)) : times_i(2. * s2x * z);
    cplxT<T> X = G21 + z * G12 - G31 - z * G13;
    cplxT<T> Y = G32 + z * G23 - G12 - z * G21;
    cplxT<T> Z = G13 + z * G31 - G23 - z * G32;
    out.L1 = fac * X;
    out.L2 = fac * Y;
    out.L3 = fac * Z;
    return out;
  }
  cplxT<T> fAE, fT;
  if (rescaled) {
    fAE = cmk(T(1.0), T(0.0));
    fT = cmk(T(1.0), T(0.0));
  } else {
    fAE = times_i(SQRT2 * s2x * z);
    fT = (2. * SQRT2 * s2x * e1.im) * (z * e1);
  }
  cplxT<T> one = cmk(T(1.0), T(0.0));
  cplxT<T> A = 0.5 * ((one + z) * (G31 + G13) - G23 - z * G32 - G21 - z * G12);
  cplxT<T> E = (0.5 * INVSQRT3) * ((one - z) * (G13 - G31) + (cmk(T(2.0), T(0.0)) + z) * (G12 - G32) +
                              (one + 2. * z) * (G21 - G23));
  cplxT<T> Tc = INVSQRT6 * (G21 - G12 + G32 - G23 + G13 - G31);
  cplxT<T> f2 = cmk(T(2.0), T(0.0));
  if (tdi2) f2 = 2.0 * times_i((-2. * (2. * s2x * z.re)) * (z * z));  // -2i sin4x e^{4ix}
  out.L1 = f2 * (fAE * A);
  out.L2 = f2 * (fAE * E);
  out.L3 = f2 * (fT * Tc);
  return out;
}

}  // namespace bbhx
