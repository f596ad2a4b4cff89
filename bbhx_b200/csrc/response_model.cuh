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
// vector outside.
#pragma once

#include "bbhx_common.cuh"

namespace bbhx {

struct OrbitTables {
  const double* x_arr;  // [N][3][3]
  const double* n_arr;  // [N][6][3]
  double dt;
  int N;
  int link_index[3];  // table slots of links 12, 23, 31
  double armlength;
};

// Device-resident orbit tables owned by the C-ABI orbit handle (bbhx_orbits_*).
struct OrbitHandle {
  double* d_x = nullptr;
  double* d_n = nullptr;
  OrbitTables tab{};
  bool ready = false;
};

struct ResponseMode {
  cplx H[9];     // complex mode matrix, row-major
  double k[3];   // propagation direction
};

struct V3 {
  double x, y, z;
};

__device__ __forceinline__ V3 orbit_lerp(const double* tab, int stride, int offset, double dt,
                                         int N, double t) {
  double w = floor(t / dt);
  if (!(w >= 0.0) || w >= (double)(N - 1)) return V3{0.0, 0.0, 0.0};
  int wi = (int)w;
  const double* lo = tab + (size_t)wi * stride + offset;
  const double* hi = lo + stride;
  double tt = t - wi * dt;
  V3 r;
  r.x = __ldg(lo + 0) + (__ldg(hi + 0) - __ldg(lo + 0)) / dt * tt;
  r.y = __ldg(lo + 1) + (__ldg(hi + 1) - __ldg(lo + 1)) / dt * tt;
  r.z = __ldg(lo + 2) + (__ldg(hi + 2) - __ldg(lo + 2)) / dt * tt;
  return r;
}

// spin-weight -2 spherical harmonics for l = 2..4 (Response.cu:383-424)
__device__ inline cplx sylm_m2(int l, int m, double theta, double phi) {
  double fac = 0.0;
  double ct = cos(theta), st = sin(theta);
  double c2 = cos(theta / 2.0), s2 = sin(theta / 2.0);
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
  if (m == 0) return mk(fac, 0.0);
  double s, c;
  sincos(m * phi, &s, &c);
  return mk(fac * c, fac * s);
}

__device__ inline void response_mode_setup(ResponseMode& r, int ell, int mm, double phi_ref,
                                           double inc, double lam, double beta, double psi) {
  double cl = cos(lam), sl = sin(lam), cb = cos(beta), sb = sin(beta), cp = cos(psi), sp = sin(psi);
  r.k[0] = -cb * cl;
  r.k[1] = -cb * sl;
  r.k[2] = -sb;
  // rotation from the wave frame to the SSB frame and its inverse
  double O[9] = {cp * sl - cl * sb * sp, -cl * cp * sb - sl * sp, -cb * cl,
                 -cl * cp - sb * sl * sp, -cp * sb * sl + cl * sp, -cb * sl,
                 cb * sp, cb * cp, -sb};
  double Oi[9] = {O[0], O[3], O[6], O[1], O[4], O[7], O[2], O[5], O[8]};
  // H+ = O diag(1,-1,0) O^-1, Hx = O offdiag(1,1) O^-1
  double Hp[9], Hc[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      // (HS+ O^-1)_{kj} = s_k Oi[k][j] with s = (1,-1,0); (HSx O^-1)_{0j} = Oi[1][j], _{1j} = Oi[0][j]
      double p = O[i * 3 + 0] * Oi[0 * 3 + j] - O[i * 3 + 1] * Oi[1 * 3 + j];
      double x = O[i * 3 + 0] * Oi[1 * 3 + j] + O[i * 3 + 1] * Oi[0 * 3 + j];
      Hp[i * 3 + j] = p;
      Hc[i * 3 + j] = x;
    }
  cplx Ylm = sylm_m2(ell, mm, inc, phi_ref);
  cplx Ylmm = sylm_m2(ell, -mm, inc, phi_ref);
  double sgn = (ell % 2 == 0) ? 1.0 : -1.0;
  cplx Yl_m = sgn * conj(Ylmm);
  cplx Yp = 0.5 * (Ylm + Yl_m);
  cplx Yc = times_i(0.5 * (Ylm - Yl_m));
  for (int q = 0; q < 9; ++q) r.H[q] = Yp * Hp[q] + Yc * Hc[q];
}

struct Transfer {
  cplx L1, L2, L3;
  double phaseRdelay;
};

__device__ __forceinline__ cplx nHn(const cplx* H, V3 n) {
  double v[3] = {n.x, n.y, n.z};
  cplx out = mk(0.0, 0.0);
  for (int i = 0; i < 3; ++i) {
    cplx t = mk(0.0, 0.0);
    for (int j = 0; j < 3; ++j) t = t + H[i * 3 + j] * v[j];
    out = out + v[i] * t;
  }
  return out;
}

__device__ __forceinline__ double sinc(double x) { return x == 0.0 ? 1.0 : sin(x) / x; }

// TDItag: 1 = XYZ, 2 = AET.  f in Hz, t in s.
__device__ inline Transfer response_point(const ResponseMode& r, const OrbitTables& orb, double f,
                                          double t, int TDItag, int rescaled, int tdi2) {
  const double* k = r.k;
  // Roemer delay relative to the SSB (circular 1 AU orbit of the guiding centre)
  double al = Omega0 * t;
  double sa, ca;
  sincos(al, &sa, &ca);
  double kR = k[0] * (AU_SI * ca) + k[1] * (AU_SI * sa) + k[2] * (0.0 * t);
  Transfer out;
  out.phaseRdelay = 2. * PI / C_SI * f * kR;

  V3 p1 = orbit_lerp(orb.x_arr, 9, 0, orb.dt, orb.N, t);
  V3 p2 = orbit_lerp(orb.x_arr, 9, 3, orb.dt, orb.N, t);
  V3 p3 = orbit_lerp(orb.x_arr, 9, 6, orb.dt, orb.N, t);
  V3 n1 = orbit_lerp(orb.n_arr, 18, orb.link_index[0] * 3, orb.dt, orb.N, t);
  V3 n2 = orbit_lerp(orb.n_arr, 18, orb.link_index[1] * 3, orb.dt, orb.N, t);
  V3 n3 = orbit_lerp(orb.n_arr, 18, orb.link_index[2] * 3, orb.dt, orb.N, t);
  double kn1 = k[0] * n1.x + k[1] * n1.y + k[2] * n1.z;
  double kn2 = k[0] * n2.x + k[1] * n2.y + k[2] * n2.z;
  double kn3 = k[0] * n3.x + k[1] * n3.y + k[2] * n3.z;
  cplx n1H = nHn(r.H, n1), n2H = nHn(r.H, n2), n3H = nHn(r.H, n3);
  double k12 = k[0] * (p1.x + p2.x) + k[1] * (p1.y + p2.y) + k[2] * (p1.z + p2.z);
  double k23 = k[0] * (p2.x + p3.x) + k[1] * (p2.y + p3.y) + k[2] * (p2.z + p3.z);
  double k31 = k[0] * (p3.x + p1.x) + k[1] * (p3.y + p1.y) + k[2] * (p3.z + p1.z);
  const double L = orb.armlength;
  double pre = PI * f * L / C_SI;
  cplx e12 = expi(pre * (1. + k12 / L));
  cplx e23 = expi(pre * (1. + k23 / L));
  cplx e31 = expi(pre * (1. + k31 / L));
  // The constellation-centre phase factor exp(+i 2 pi f k.p0 / c) of the full response and
  // the Roemer-delay factor exp(-i phaseRdelay) cancel identically (Response.cu:166,304-309).
  cplx common = mk(0.0, pre);
  cplx c3 = common * n3H, c1 = common * n1H, c2 = common * n2H;
  cplx G12 = c3 * (sinc(pre * (1. - kn3)) * e12);
  cplx G21 = c3 * (sinc(pre * (1. + kn3)) * e12);
  cplx G23 = c1 * (sinc(pre * (1. - kn1)) * e23);
  cplx G32 = c1 * (sinc(pre * (1. + kn1)) * e23);
  cplx G31 = c2 * (sinc(pre * (1. - kn2)) * e31);
  cplx G13 = c2 * (sinc(pre * (1. + kn2)) * e31);

  // e^{ix}, x = pre, and its powers / sines from one sincos
  const cplx e1 = expi(pre);
  const cplx z = e1 * e1;  // e^{2ix}
  const double s2x = 2. * e1.im * e1.re;
  if (TDItag == 1) {
    cplx fac = rescaled ? mk(1.0, 0.0) : times_i(2. * s2x * z);
    cplx X = G21 + z * G12 - G31 - z * G13;
    cplx Y = G32 + z * G23 - G12 - z * G21;
    cplx Z = G13 + z * G31 - G23 - z * G32;
    out.L1 = fac * X;
    out.L2 = fac * Y;
    out.L3 = fac * Z;
    return out;
  }
  cplx fAE, fT;
  if (rescaled) {
    fAE = mk(1.0, 0.0);
    fT = mk(1.0, 0.0);
  } else {
    fAE = times_i(SQRT2 * s2x * z);
    fT = (2. * SQRT2 * s2x * e1.im) * (z * e1);
  }
  cplx one = mk(1.0, 0.0);
  cplx A = 0.5 * ((one + z) * (G31 + G13) - G23 - z * G32 - G21 - z * G12);
  cplx E = (0.5 * INVSQRT3) * ((one - z) * (G13 - G31) + (mk(2.0, 0.0) + z) * (G12 - G32) +
                              (one + 2. * z) * (G21 - G23));
  cplx T = INVSQRT6 * (G21 - G12 + G32 - G23 + G13 - G31);
  cplx f2 = mk(2.0, 0.0);
  if (tdi2) f2 = 2.0 * times_i((-2. * (2. * s2x * z.re)) * (z * z));  // -2i sin4x e^{4ix}
  out.L1 = f2 * (fAE * A);
  out.L2 = f2 * (fAE * E);
  out.L3 = f2 * (fT * T);
  return out;
}

}  // namespace bbhx
