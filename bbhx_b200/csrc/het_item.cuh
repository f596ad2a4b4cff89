// Per-walker body of the fused heterodyned (relative-binning) likelihood, shared by the
// single-problem kernel (heterodyne.cu, k_het_fused) and the uneven-batch persistent kernel
// (likelihood.cu, k_uneven): one warp evaluates one walker from its own slice of shared memory.
//
// Precision variants (template flag MIXED):
//   FP64  : everything in FP64 (phm_eval_point / response_point of the direct path).
//   mixed : phase, t(f), the Roemer delay, the orbit positions, the arguments of the
//           transfer phasors, the waveform phasor e^{i phase}, the distance / mass scale and
//           the channel products in FP64; the shape of the amplitude (PhenomD ansatz and PN
//           ratios), the sinc factors and the transfer algebra in FP32; r = h / h0 and the
//           bin sums in FP64.
#pragma once

#include "bbhx_common.cuh"
#include "phenomhm_model.cuh"
#include "response_model.cuh"
#include "spline_eval.cuh"

namespace bbhx {

// ------------------------------------------------------------------ FP32 amplitude model
// Amplitude coefficients of one (binary, mode) in FP32 (built once per CTA from ModeCoeffs).
struct __align__(16) AmpModeF {
  float amp0, ains[8], g1, g2, g3, fRD, fDM, fpeak;
  float hf1, hf2, hf3, hc0, hc1, hc2, hc3, hc4;
  float am_fi, am_fr, am_ai, am_am, am_bm, am_br;
  // PN amplitude |H_lm(v)| (IMRPhenomHMOnePointFiveSpinPN, PhenomHMWaveform.cu:2375-2455)
  float eta, delta, Xs, Xa, two_pi_over_m, four_pi_over_m2, pn_k;
  int pn_case;  // 0: (2,2) or PhenomD only; 1: 21; 2: 33; 3: 32; 4: 44; 5: 43; 6: none
};

__device__ inline void build_amp_f(AmpModeF& a, const ModeCoeffs& c) {
  const PhenomD& d = c.d;
  a.amp0 = (float)d.amp0;
  for (int k = 0; k < 8; ++k) a.ains[k] = (float)d.ains[k];
  a.g1 = (float)d.g1;
  a.g2 = (float)d.g2;
  a.g3 = (float)d.g3;
  a.fRD = (float)d.fRD;
  a.fDM = (float)d.fDM;
  a.fpeak = (float)d.fpeak;
  a.hf1 = (float)d.hf1;
  a.hf2 = (float)d.hf2;
  a.hf3 = (float)d.hf3;
  a.hc0 = (float)d.hc0;
  a.hc1 = (float)d.hc1;
  a.hc2 = (float)d.hc2;
  a.hc3 = (float)d.hc3;
  a.hc4 = (float)d.hc4;
  a.am_fi = (float)c.am_fi;
  a.am_fr = (float)c.am_fr;
  a.am_ai = (float)c.am_ai;
  a.am_am = (float)c.am_am;
  a.am_bm = (float)c.am_bm;
  a.am_br = (float)c.am_br;
  a.eta = (float)c.pn_eta;
  a.delta = (float)c.pn_delta;
  a.Xs = (float)c.pn_Xs;
  a.Xa = (float)c.pn_Xa;
  a.two_pi_over_m = (float)c.pn_2pi_m;
  a.four_pi_over_m2 = (float)c.pn_4pi_m2;
  a.pn_k = (float)c.pn_k;
  a.pn_case = c.pn_case;
}

// |H_lm(v)| of the 1.5PN spinning amplitude for the non-22 cases.
__device__ __forceinline__ float pn_habs_f(const AmpModeF& a, float v) {
  const float v2 = v * v, v3 = v2 * v;
  switch (a.pn_case) {
    case 1: {
      const float v4 = v3 * v;
      const float re = a.pn_k * (v * a.delta - v2 * 1.5f * (a.Xa + a.delta * a.Xs) +
                                 v3 * a.delta * (335.0f / 672.0f + a.eta * (117.0f / 56.0f)) +
                                 v4 * (a.Xa * (3427.0f / 1344.0f - a.eta * (2101.0f / 336.0f)) +
                                       a.delta * a.Xs * (3427.0f / 1344.0f - a.eta * (965.0f / 336.0f)) -
                                       a.delta * (float)PI));
      const float im = a.pn_k * v4 * a.delta * (-0.5f - 2.0f * 0.69314718056f);
      return sqrtf(re * re + im * im);
    }
    case 2: return fabsf(a.pn_k * v * a.delta);
    case 3: return fabsf(a.pn_k * v2 * (1.0f - 3.0f * a.eta));
    case 4: return fabsf(a.pn_k * v2 * (1.0f - 3.0f * a.eta));
    case 5: return fabsf(a.pn_k * v3 * a.delta * (1.0f - 2.0f * a.eta));
    default: return 0.0f;
  }
}


// PhenomD amplitude without the distance / mass scale (PhenomHMWaveform.cu:1508-1537).
__device__ __forceinline__ float phenomd_amp_f(const AmpModeF& a, float Mf) {
  const float third = cbrtf(Mf);
  const float sixth = sqrtf(third);
  const float pre = a.amp0 / (Mf * sixth);
  if (Mf < (float)AMP_FJOIN_INS) {
    const float two_thirds = Mf / third, four_thirds = Mf * third;
    const float five_thirds = four_thirds * third, two = Mf * Mf;
    const float seven_thirds = third * two, eight_thirds = two_thirds * two;
    const float ins = 1.0f + two_thirds * a.ains[0] + Mf * a.ains[1] + four_thirds * a.ains[2] +
                      five_thirds * a.ains[3] + two * a.ains[4] + seven_thirds * a.ains[5] +
                      eight_thirds * a.ains[6] + Mf * two * a.ains[7];
    return pre * ins;
  }
  if (Mf >= a.fpeak) {
    const float s = a.fDM * a.g3;
    const float x = Mf - a.fRD;
    return pre * expf(-x * a.g2 / s) * (s * a.g1) / (x * x + s * s);
  }
  const float u = Mf - a.hf1;
  return pre * (a.hc0 + u * (a.hc1 + u * (a.hc2 + (Mf - a.hf2) * (a.hc3 + (Mf - a.hf3) * a.hc4))));
}

// Mode amplitude at geometric frequency Mf without the distance / mass scale: PhenomD at the
// mapped frequency times the PN ratio (get_amp, PhenomHMWaveform.cu:2461-2514).  With v_lm(x) = (2 pi x / m)^(1/3), the
// four v^-3.5 |H| factors of the reference reduce to |H(v(Mf))| |H(v(Mfa))| / |H(v(2Mf/m))|
// because the v^-3.5 powers cancel exactly: v(2Mf/m) / v(Mf) = (2/m)^(1/3) and
// v_22(Mfa) / v_lm(Mfa) = (m/2)^(1/3).
__device__ __forceinline__ float mode_amp_f(const AmpModeF& a, float Mf) {
  float Mfa;
  if (Mf > a.am_fi) Mfa = (Mf > a.am_fr) ? Mf + a.am_br : fmaf(a.am_am, Mf, a.am_bm);
  else Mfa = a.am_ai * Mf;
  const float amp = phenomd_amp_f(a, Mfa);
  if (a.pn_case == 0) return amp;
  const float t1 = pn_habs_f(a, cbrtf(a.two_pi_over_m * Mf));
  if (t1 == 0.0f) return 0.0f;
  const float t2 = pn_habs_f(a, cbrtf(a.four_pi_over_m2 * Mf));
  const float h1 = pn_habs_f(a, cbrtf(a.two_pi_over_m * Mfa));
  return amp * (t1 / t2) * h1;
}

// ------------------------------------------------------------------ FP32 response algebra
struct __align__(16) RespModeF {
  cplxf H[9];
  double k[3];
};

__device__ inline void build_resp_f(RespModeF& o, const ResponseMode& r) {
  for (int q = 0; q < 9; ++q) o.H[q] = cplxf{(float)r.H[q].re, (float)r.H[q].im};
  for (int q = 0; q < 3; ++q) o.k[q] = r.k[q];
}

struct TransferF {
  cplxf L1, L2, L3;
  double phaseRdelay;
};

__device__ __forceinline__ cplxf nHn_f(const cplxf* H, float n0, float n1, float n2) {
  const float v[3] = {n0, n1, n2};
  cplxf out{0.f, 0.f};
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    cplxf t{0.f, 0.f};
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      t.re = fmaf(H[i * 3 + j].re, v[j], t.re);
      t.im = fmaf(H[i * 3 + j].im, v[j], t.im);
    }
    out.re = fmaf(v[i], t.re, out.re);
    out.im = fmaf(v[i], t.im, out.im);
  }
  return out;
}

__device__ __forceinline__ float sinc_f(float x) { return x == 0.0f ? 1.0f : __fdividef(sinf(x), x); }
__device__ __forceinline__ cplxf cf(float r, float i) { return cplxf{r, i}; }
__device__ __forceinline__ cplxf ti_f(cplxf a) { return {-a.im, a.re}; }
__device__ __forceinline__ cplxf ephase(double x) {
  float s, c;
  sincos_mixed(x, &s, &c);
  return cplxf{c, s};
}

// Same transfer as response_point (Response.cu:54-314) with the split described above.
__device__ inline TransferF response_point_mixed(const RespModeF& r, const OrbitTables& orb,
                                                 double f, double t, int TDItag, int rescaled,
                                                 int tdi2) {
  const double* k = r.k;
  double sa, ca;
  sincos_cw(Omega0 * t, &sa, &ca);
  TransferF out;
  out.phaseRdelay = 2. * PI / C_SI * f * (k[0] * (AU_SI * ca) + k[1] * (AU_SI * sa));

  const OrbitWindow<double> win = orbit_window(orb, t);
  V3T<double> p1 = orbit_lerp(win.x_lo, 9, 0, win.frac);
  V3T<double> p2 = orbit_lerp(win.x_lo, 9, 3, win.frac);
  V3T<double> p3 = orbit_lerp(win.x_lo, 9, 6, win.frac);
  V3T<double> n1 = orbit_lerp(win.n_lo, 18, orb.link_index[0] * 3, win.frac);
  V3T<double> n2 = orbit_lerp(win.n_lo, 18, orb.link_index[1] * 3, win.frac);
  V3T<double> n3 = orbit_lerp(win.n_lo, 18, orb.link_index[2] * 3, win.frac);
  const float kn1 = (float)(k[0] * n1.x + k[1] * n1.y + k[2] * n1.z);
  const float kn2 = (float)(k[0] * n2.x + k[1] * n2.y + k[2] * n2.z);
  const float kn3 = (float)(k[0] * n3.x + k[1] * n3.y + k[2] * n3.z);
  const cplxf n1H = nHn_f(r.H, (float)n1.x, (float)n1.y, (float)n1.z);
  const cplxf n2H = nHn_f(r.H, (float)n2.x, (float)n2.y, (float)n2.z);
  const cplxf n3H = nHn_f(r.H, (float)n3.x, (float)n3.y, (float)n3.z);
  const double k12 = k[0] * (p1.x + p2.x) + k[1] * (p1.y + p2.y) + k[2] * (p1.z + p2.z);
  const double k23 = k[0] * (p2.x + p3.x) + k[1] * (p2.y + p3.y) + k[2] * (p2.z + p3.z);
  const double k31 = k[0] * (p3.x + p1.x) + k[1] * (p3.y + p1.y) + k[2] * (p3.z + p1.z);
  const double invL = orb.inv_armlength;
  const double pre = f * orb.pi_L_over_c;
  const cplxf e12 = ephase(pre * (1. + k12 * invL));
  const cplxf e23 = ephase(pre * (1. + k23 * invL));
  const cplxf e31 = ephase(pre * (1. + k31 * invL));
  const float pf = (float)pre;
  const cplxf c3 = pf * ti_f(n3H), c1 = pf * ti_f(n1H), c2 = pf * ti_f(n2H);
  const cplxf G12 = sinc_f(pf * (1.f - kn3)) * (c3 * e12);
  const cplxf G21 = sinc_f(pf * (1.f + kn3)) * (c3 * e12);
  const cplxf G23 = sinc_f(pf * (1.f - kn1)) * (c1 * e23);
  const cplxf G32 = sinc_f(pf * (1.f + kn1)) * (c1 * e23);
  const cplxf G31 = sinc_f(pf * (1.f - kn2)) * (c2 * e31);
  const cplxf G13 = sinc_f(pf * (1.f + kn2)) * (c2 * e31);

  // powers of e^{ix}, x = pre, from one reduction
  const cplxf e1 = ephase(pre);
  const cplxf z = e1 * e1;  // e^{2ix}
  const float s1 = e1.im, s2x = 2.f * e1.im * e1.re;
  if (TDItag == 1) {
    const cplxf fac = rescaled ? cf(1.f, 0.f) : ti_f((2.f * s2x) * z);
    const cplxf X = G21 + z * G12 - G31 - z * G13;
    const cplxf Y = G32 + z * G23 - G12 - z * G21;
    const cplxf Z = G13 + z * G31 - G23 - z * G32;
    out.L1 = fac * X;
    out.L2 = fac * Y;
    out.L3 = fac * Z;
    return out;
  }
  cplxf fAE, fT;
  if (rescaled) {
    fAE = cf(1.f, 0.f);
    fT = cf(1.f, 0.f);
  } else {
    fAE = ti_f((float)SQRT2 * s2x * z);
    fT = (2.f * (float)SQRT2 * s2x * s1) * (z * e1);
  }
  const cplxf one = cf(1.f, 0.f);
  const cplxf A = 0.5f * ((one + z) * (G31 + G13) - G23 - z * G32 - G21 - z * G12);
  const cplxf E = (0.5f * (float)INVSQRT3) *
                  ((one - z) * (G13 - G31) + (cf(2.f, 0.f) + z) * (G12 - G32) +
                   (one + 2.f * z) * (G21 - G23));
  const cplxf T = (float)INVSQRT6 * (G21 - G12 + G32 - G23 + G13 - G31);
  cplxf f2 = cf(2.f, 0.f);
  if (tdi2) {
    const cplxf z2 = z * z;                                // e^{4ix}
    const float s4x = 2.f * s2x * (e1.re * e1.re - e1.im * e1.im);  // sin 4x
    f2 = 2.f * ti_f((-2.f * s4x) * z2);
  }
  out.L1 = f2 * (fAE * A);
  out.L2 = f2 * (fAE * E);
  out.L3 = f2 * (fT * T);
  return out;
}

// ------------------------------------------------------------------ one walker
constexpr int HET_THREADS = 128;
constexpr int HET_STRIP = 128;  // sparse frequencies whose residuals r are held at a time

struct HetArgs {
  cplx* d_h;
  cplx* h_h;
  const ModeCoeffs* coeffs;    // [B, M]
  const ResponseMode* rmodes;  // [B, M] (k_het_response_setup)
  const int* ells;             // [M]
  const int* mms;              // [M]
  const double* phi_ref;       // [B] each: the response-mode inputs
  const double* inc;
  const double* lam;
  const double* beta;
  const double* psi;
  OrbitTables orb;
  const double* t_ref;
  double t_init;
  const double* t_start;
  const double* t_end;
  const double* freqs;  // [L]
  const cplx* h0;       // [3, L]
  const cplx* consts;   // [4, 3, L]: A0, A1, B0, B1
  int TDItag, rescaled, tdi2;
  int M, L, B;
  cplx* gh;  // optional [B, 3, L]: d lnL / d h (adjoint of the bin sums and of r = h / h0)
};

__host__ __device__ __forceinline__ size_t align16(size_t n) { return (n + 15) & ~(size_t)15; }

// Shared memory of one warp (walker): ModeCoeffs[M] | ResponseMode[M] | AmpModeF[M] |
// RespModeF[M] | residuals r, each region starting on a 16-byte boundary.  r holds
// r = h / h0 of all L frequencies [3][L] (FULL), or one strip of HET_STRIP frequencies plus the
// previous strip's last one [3][HET_STRIP + 1], which bounds the slice for any L.
struct HetSmemLayout {
  size_t sr, sa, sf, rr, total;
  __host__ __device__ HetSmemLayout(int M, int L, bool full_r) {
    sr = align16(sizeof(ModeCoeffs) * M);
    sa = sr + align16(sizeof(ResponseMode) * M);
    sf = sa + align16(sizeof(AmpModeF) * M);
    rr = sf + align16(sizeof(RespModeF) * M);
    total = rr + sizeof(cplx) * 3 * (size_t)(full_r ? L : HET_STRIP + 1);
  }
};

// Typed views of one warp's slice (shared memory).
struct HetSlice {
  ModeCoeffs* sc;
  ResponseMode* sr;
  AmpModeF* sa;
  RespModeF* sf;
  cplx* rr;
  __device__ __forceinline__ HetSlice(unsigned char* base, const HetSmemLayout& lay)
      : sc((ModeCoeffs*)base), sr((ResponseMode*)(base + lay.sr)), sa((AmpModeF*)(base + lay.sa)),
        sf((RespModeF*)(base + lay.sf)), rr((cplx*)(base + lay.rr)) {}
};

// r = h / h0 of walker b at sparse frequency index j (h: the conjugated mode sum in the three
// channels), written to dst[0], dst[stride], dst[2 stride].
template <bool MIXED>
__device__ __forceinline__ void het_point(const HetArgs& A, const HetSlice& W, double tr,
                                          double ts, double te, int j, cplx* dst, int stride) {
  const double f = A.freqs[j];
  double h[6] = {0, 0, 0, 0, 0, 0};
  for (int m = 0; m < A.M; ++m) {
    if (MIXED) {
      const ModeCoeffs& c = W.sc[m];
      const double Mf = f * c.M_sec;
      double ph, tf;
      mode_phase_tf(c, Mf, &ph, &tf);  // FP64
      ph += f * (tr - A.t_init) * 2 * PI;
      tf += tr;
      if (!tf_gate(tf, ts, te)) continue;
      const float ampf = c.phenomd_only ? phenomd_amp_f(W.sa[m], (float)Mf)
                                        : mode_amp_f(W.sa[m], (float)Mf);
      const TransferF T = response_point_mixed(W.sf[m], A.orb, f, tf, A.TDItag, A.rescaled, A.tdi2);
      // phasor and channel products in FP64 (the scale factor stays FP64 as well)
      double sn, cs;
      sincos_cw(ph + T.phaseRdelay, &sn, &cs);
      const double amp = (double)ampf * c.amp_scale;
      const double apr = amp * cs, api = amp * sn;
      const cplxf Tc[3] = {T.L1, T.L2, T.L3};
#pragma unroll
      for (int ch = 0; ch < 3; ++ch) {
        const double trr = Tc[ch].re, tii = Tc[ch].im;
        h[2 * ch] += trr * apr - tii * api;
        h[2 * ch + 1] -= trr * api + tii * apr;
      }
    } else {
      PointOut o = phm_eval_point(W.sc[m], f);
      o.phase += f * (tr - A.t_init) * 2 * PI;
      o.tf += tr;
      if (!tf_gate(o.tf, ts, te)) continue;
      const Transfer T = response_point(W.sr[m], A.orb, f, o.tf, A.TDItag, A.rescaled, A.tdi2);
      const cplx ap = o.amp * expi(o.phase + T.phaseRdelay);
      const cplx Tc[3] = {T.L1, T.L2, T.L3};
#pragma unroll
      for (int ch = 0; ch < 3; ++ch) {
        const cplx v = Tc[ch] * ap;
        h[2 * ch] += v.re;
        h[2 * ch + 1] -= v.im;
      }
    }
  }
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) {
    const cplx d = A.h0[(size_t)ch * A.L + j];
    const double den = d.re * d.re + d.im * d.im;
    dst[ch * stride] = mk((h[2 * ch] * d.re + h[2 * ch + 1] * d.im) / den,
                          (h[2 * ch + 1] * d.re - h[2 * ch] * d.im) / den);
  }
}

// Relative-binning term of bin j >= 1 (hdynLikelihood, Likelihood.cu:20-123) from r_j (cur)
// and r_{j-1} (prv), added to the four sums.
__device__ __forceinline__ void het_bin(const HetArgs& A, int j, int ch, cplx cur, cplx prv,
                                        double& dre, double& dim, double& hre, double& him) {
  const double fj = A.freqs[j], fp = A.freqs[j - 1];
  if (fp == 0.0) return;
  const double df = fj - fp;
  const double fm = (fj + fp) / 2.0;
  const cplx r1 = mk((cur.re - prv.re) / df, (cur.im - prv.im) / df);
  const cplx r0 = cur - r1 * (fj - fm);
  const cplx A0 = A.consts[((size_t)0 * 3 + ch) * A.L + j];
  const cplx A1 = A.consts[((size_t)1 * 3 + ch) * A.L + j];
  const cplx B0 = A.consts[((size_t)2 * 3 + ch) * A.L + j];
  const cplx B1 = A.consts[((size_t)3 * 3 + ch) * A.L + j];
  const cplx t = A0 * conj(r0) + A1 * conj(r1);
  dre += t.re;
  dim += t.im;
  const double mag2 = r0.re * r0.re + r0.im * r0.im;
  const double re01 = r0.re * r1.re + r0.im * r1.im;
  hre += B0.re * mag2 + 2.0 * B1.re * re01;
  him += B0.im * mag2 + 2.0 * B1.im * re01;
}

// Response-mode records of walkers [0, B) of A into A.rmodes (one thread per (walker, mode)),
// set up once per evaluation outside the walker loop: inlined there, the set-up's code and
// registers slow the per-point loop down.
__device__ __forceinline__ ResponseMode het_response_record(const HetArgs& A, long long t) {
  const int b = (int)(t / A.M), i = (int)(t % A.M);
  ResponseMode r;
  response_mode_setup(r, A.ells[i], A.mms[i], A.phi_ref[b], A.inc[b], A.lam[b], A.beta[b],
                      A.psi[b]);
  return r;
}
__device__ __forceinline__ void het_response_setup(const HetArgs& A, long long t) {
  const_cast<ResponseMode*>(A.rmodes)[t] = het_response_record(A, t);
}

// Walker b of A by one warp in its slice W (HetSmemLayout(M, L, FULL)): records staged
// (PhenomHM and response modes copied), then the points and the bin sums; lane 0 writes
// d_h[b], h_h[b] and flags a non-finite result in *nonfinite.  Bin j is summed by lane
// (j - 1) mod 32 in increasing j in both residual layouts, so both give the same sums.
// GH (FP64, FULL): d lnL / d h is written to A.gh as well.
template <bool MIXED, bool FULL, bool GH>
__device__ __forceinline__ void het_item(const HetArgs& A, int b, const HetSlice& W, int lane,
                                         unsigned* nonfinite) {
  static_assert(!(MIXED && GH), "d lnL / d h is written by the FP64 form only");
  static_assert(FULL || !GH, "the adjoint needs all residuals");
  __syncwarp();  // the previous walker's shared data is no longer in use
  {
    const unsigned long long* src = (const unsigned long long*)(A.coeffs + (size_t)b * A.M);
    unsigned long long* dst = (unsigned long long*)W.sc;
    const int n = (int)(sizeof(ModeCoeffs) * A.M / 8);
    for (int i = lane; i < n; i += 32) dst[i] = src[i];
    src = (const unsigned long long*)(A.rmodes + (size_t)b * A.M);
    dst = (unsigned long long*)W.sr;
    const int n2 = (int)(sizeof(ResponseMode) * A.M / 8);
    for (int i = lane; i < n2; i += 32) dst[i] = src[i];
  }
  __syncwarp();
  if (MIXED) {
    if (lane < A.M) build_amp_f(W.sa[lane], W.sc[lane]);
    else if (lane >= 16 && lane < 16 + A.M) build_resp_f(W.sf[lane - 16], W.sr[lane - 16]);
    __syncwarp();
  }
  const double tr = A.t_ref[b];
  const double ts = A.t_start[b], te = A.t_end[b];
  cplx* rr = W.rr;
  double dre = 0, dim = 0, hre = 0, him = 0;
  if (FULL) {
    for (int j = lane; j < A.L; j += 32) het_point<MIXED>(A, W, tr, ts, te, j, rr + j, A.L);
    __syncwarp();
    for (int j = 1 + lane; j < A.L; j += 32) {
#pragma unroll
      for (int ch = 0; ch < 3; ++ch)
        het_bin(A, j, ch, rr[ch * A.L + j], rr[ch * A.L + j - 1], dre, dim, hre, him);
    }
  } else {
    // strips of HET_STRIP frequencies; rr[ch][0] carries r of the previous strip's last one
    constexpr int SW = HET_STRIP + 1;
    for (int j0 = 0; j0 < A.L; j0 += HET_STRIP) {
      const int jn = min(HET_STRIP, A.L - j0);
      for (int jj = lane; jj < jn; jj += 32)
        het_point<MIXED>(A, W, tr, ts, te, j0 + jj, rr + 1 + jj, SW);
      __syncwarp();
      // bin j = j0 + jj (lane (j - 1) mod 32, as with all residuals held)
      for (int jj = (j0 + lane + 1) & 31; jj < jn; jj += 32) {
        const int j = j0 + jj;
        if (j < 1) continue;
#pragma unroll
        for (int ch = 0; ch < 3; ++ch)
          het_bin(A, j, ch, rr[ch * SW + 1 + jj], rr[ch * SW + jj], dre, dim, hre, him);
      }
      __syncwarp();
      if (lane < 3) rr[lane * SW] = rr[lane * SW + jn];
      __syncwarp();
    }
  }
  if (GH && A.gh) {
    // Adjoint of lnL = Re d_h - (d_d + Re h_h) / 2 through the bin terms: per bin
    // g_r0 = A0 - Re(B0) r0 - Re(B1) r1, g_r1 = A1 - Re(B1) r0, carried to r_j / r_{j-1}
    // with the same coefficients as the forward r0, r1; then g_h = g_r / conj(h0).
    for (int j = lane; j < A.L; j += 32) {
#pragma unroll
      for (int ch = 0; ch < 3; ++ch) {
        cplx g = mk(0.0, 0.0);
        for (int side = 0; side < 2; ++side) {
          const int jj = j + side;  // bin jj has cur = r_jj, prv = r_{jj-1}
          if (jj < 1 || jj >= A.L) continue;
          const double fj = A.freqs[jj], fp = A.freqs[jj - 1];
          if (fp == 0.0) continue;
          const double df = fj - fp;
          const double fm = (fj + fp) / 2.0;
          const double a = (fj - fm) / df;
          const cplx cur = rr[ch * A.L + jj], prv = rr[ch * A.L + jj - 1];
          const cplx r1 = mk((cur.re - prv.re) / df, (cur.im - prv.im) / df);
          const cplx r0 = cur - r1 * (fj - fm);
          const cplx A0 = A.consts[((size_t)0 * 3 + ch) * A.L + jj];
          const cplx A1 = A.consts[((size_t)1 * 3 + ch) * A.L + jj];
          const double B0 = A.consts[((size_t)2 * 3 + ch) * A.L + jj].re;
          const double B1 = A.consts[((size_t)3 * 3 + ch) * A.L + jj].re;
          const cplx g0 = A0 - B0 * r0 - B1 * r1;
          const cplx g1 = A1 - B1 * r0;
          if (side == 0) g = g + (1.0 - a) * g0 + (1.0 / df) * g1;  // r_j is cur of bin j
          else g = g + a * g0 - (1.0 / df) * g1;                    // r_j is prv of bin j+1
        }
        const cplx d = A.h0[(size_t)ch * A.L + j];
        const double den = d.re * d.re + d.im * d.im;  // g / conj(d) = g d / |d|^2
        A.gh[((size_t)b * 3 + ch) * A.L + j] =
            mk((g.re * d.re - g.im * d.im) / den, (g.re * d.im + g.im * d.re) / den);
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    dre += __shfl_xor_sync(0xffffffffu, dre, o);
    dim += __shfl_xor_sync(0xffffffffu, dim, o);
    hre += __shfl_xor_sync(0xffffffffu, hre, o);
    him += __shfl_xor_sync(0xffffffffu, him, o);
  }
  if (lane == 0) {
    A.d_h[b] = mk(dre, dim);
    A.h_h[b] = mk(hre, him);
    note_nonfinite(nonfinite, dre, dim, hre, him);
  }
}

}  // namespace bbhx
