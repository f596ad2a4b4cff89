// Device forms of the reference drivers' per-binary bookkeeping and of its frame transforms,
// so that a likelihood step launches no framework elementwise kernels:
//   parameter checks and mass ordering     phenomhm.py:175-199
//   SSB observation limits                 waveformbuild.py:477-484 (tSSBfromLframe,
//                                          utils/transform.py:75-105)
//   orbit-table coverage of t(f)           fastfdresponse.py:427-433
//   lnL = -(d_d + h_h - 2 d_h) / 2         likelihood.py:204-225
//   LISA <-> SSB frame, sky modes          utils/transform.py:136-426
#include <cmath>

#include "capi_internal.cuh"
#include "frames.cuh"
#include "sparse_stages.cuh"

namespace bbhx {

constexpr double ZETA = PI / 3.0;                // inclination of the constellation plane

// numpy's float modulo (result has the sign of the divisor)
__device__ __forceinline__ double py_mod(double a, double b) {
  double r = fmod(a, b);
  if (r != 0.0 && ((r < 0.0) != (b < 0.0))) r += b;
  return r;
}

__device__ __forceinline__ double modpi_dev(double x) { return x - floor(x / PI) * PI; }

__device__ __forceinline__ double tl_from_ssb(double tS, double lam, double beta, double t0) {
  const double phase = CONST_OMEGA * tS + CONST_OMEGA * t0 - lam;
  return tS - ORBIT_R / C_SI * cos(beta) * cos(phase);
}

// (lambda', beta') of (lambda, beta) rotated by Rz(alpha) Ry(-zeta) Rz(-alpha), and the angle
// between the two frames' polarisation references
__device__ __forceinline__ void rotate_sky(double lam, double beta, double alpha, double zeta,
                                           double* lam_out, double* beta_out, double* dpsi) {
  const double d = lam - alpha;
  const double cb = cos(beta), sb = sin(beta), cd = cos(d), sd = sin(d);
  const double cz = cos(zeta), sz = sin(zeta);
  const double x1 = cb * cd * cz - sb * sz;
  const double y1 = cb * sd;
  const double z1 = cb * cd * sz + sb * cz;
  const double ca = cos(alpha), sa = sin(alpha);
  *lam_out = atan2(x1 * sa + y1 * ca, x1 * ca - y1 * sa);
  *beta_out = asin(z1);
  *dpsi = atan2(sz * sd, cb * cz - sb * sz * cd);
}

// Parameter front end of a step: m1 >= m2 ordering (swapping the spins with the masses), the
// SI masses, the |chi| <= 1 checks (flags[2] bit 1: chi1z, bit 2: chi2z), the SSB observation limits and, per
// (binary, mode), the observation span the window regrid reads.  The step's status flags are
// cleared by k_clear_flags, launched before on the same stream.
__global__ void k_step_front(double* __restrict__ out, double* __restrict__ t_start,
                             double* __restrict__ t_end, double* __restrict__ tobs_rows,
                             const double* __restrict__ m1, const double* __restrict__ m2,
                             const double* __restrict__ chi1, const double* __restrict__ chi2,
                             const double* __restrict__ lam, const double* __restrict__ beta,
                             int B, int M, double tL_start, double tL_end, int* flags) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B; b += gridDim.x * blockDim.x) {
    const double x1 = chi1[b], x2 = chi2[b];
    const FrontMasses fr = front_masses(m1[b], m2[b], x1, x2);
    out[0 * (long long)B + b] = fr.m1;
    out[1 * (long long)B + b] = fr.m2;
    out[2 * (long long)B + b] = fr.chi1;
    out[3 * (long long)B + b] = fr.chi2;
    out[4 * (long long)B + b] = fr.m1_SI;
    out[5 * (long long)B + b] = fr.m2_SI;
    if (flags != nullptr && fabs(x1) > 1.0) atomicOr(flags + 2, 1);  // chi1z out of range
    if (flags != nullptr && fabs(x2) > 1.0) atomicOr(flags + 2, 2);  // chi2z out of range
    if (t_start != nullptr) {
      const double ts = tssb_from_l(tL_start, lam[b], beta[b], 0.0);
      const double te = tssb_from_l(tL_end, lam[b], beta[b], 0.0);
      t_start[b] = ts;
      t_end[b] = te;
      if (tobs_rows != nullptr)
        for (int m = 0; m < M; ++m) tobs_rows[(long long)b * M + m] = te - ts;
    }
  }
}

__global__ void k_clear_flags(int* flags, int n) {
  if (threadIdx.x < n) flags[threadIdx.x] = 0;
}

// flag = 1 if any t(f) lies outside [tmin, tmax] (NaN does not count, as in the reference's
// min / max comparison)
__global__ void k_tf_range(const double* __restrict__ tf, long long n, double tmin, double tmax,
                           int* flag) {
  bool bad = false;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double v = tf[i];
    bad = bad || (v < tmin) || (v > tmax);
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

// packed = [lnL (B) | Re d_h' (B) | Re h_h (B) | flags (nflags)], d_h' = |d_h| when phase
// marginalised, lnL = -(d_d + Re h_h - 2 Re d_h') / 2
__global__ void k_pack_lnl(double* __restrict__ packed, const cplx* __restrict__ d_h,
                           const cplx* __restrict__ h_h, double d_d, int B, int phase_marg,
                           const int* __restrict__ flags, int nflags) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B + nflags;
       b += gridDim.x * blockDim.x) {
    if (b < B) {
      const double dh = phase_marg ? hypot(d_h[b].re, d_h[b].im) : d_h[b].re;
      const double hh = h_h[b].re;
      packed[b] = -1.0 / 2.0 * ((d_d + hh) - 2.0 * dh);
      packed[B + b] = dh;
      packed[2LL * B + b] = hh;
    } else {
      packed[3LL * B + (b - B)] = (double)flags[b - B];
    }
  }
}

__global__ void k_tssb(double* out, const double* t, const double* lam, const double* beta,
                       int n, double t0, int inverse) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = inverse ? tl_from_ssb(t[i], lam[i], beta[i], t0) : tssb_from_l(t[i], lam[i], beta[i], t0);
}

// LISA_to_SSB (to_ssb = 1; transform.py:136-231: three fixed-point passes for the SSB time in
// the orbital phase) and SSB_to_LISA (to_ssb = 0; :233-294); t0 in seconds
__global__ void k_frame(double* __restrict__ t_out, double* __restrict__ lam_out,
                        double* __restrict__ beta_out, double* __restrict__ psi_out,
                        const double* __restrict__ t_in, const double* __restrict__ lam_in,
                        const double* __restrict__ beta_in, const double* __restrict__ psi_in,
                        int n, double t0, int to_ssb) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double tin = t_in[i], lin = lam_in[i], bin = beta_in[i], pin = psi_in[i];
    double lam, beta, dpsi;
    if (to_ssb) {
      double tS = tin;
      for (int it = 0; it < 3; ++it) {
        const double alpha = CONST_OMEGA * tS + CONST_OMEGA * t0;
        rotate_sky(lin, bin, alpha, ZETA, &lam, &beta, &dpsi);
        tS = tssb_from_l(tin, lam, beta, t0);
      }
      t_out[i] = tS;
      lam_out[i] = py_mod(lam, 2.0 * PI);
    } else {
      const double alpha = CONST_OMEGA * tin + CONST_OMEGA * t0;
      rotate_sky(lin, bin, alpha, -ZETA, &lam, &beta, &dpsi);
      t_out[i] = tl_from_ssb(tin, lin, bin, t0);
      lam_out[i] = lam;
    }
    beta_out[i] = beta;
    psi_out[i] = modpi_dev(pin + dpsi);
  }
}

// mbh_sky_mode_transform on rows already tiled by the mode count (transform.py:296-426):
// row r is sky mode r % factor; latitudinal mirror on odd modes ("both", "lat"); longitudinal
// quarter turns lambda + i pi/2 (mod 2 pi), psi + i pi/2 (mod pi)
__global__ void k_sky_modes(double* __restrict__ c, int rows, int ndim, int inc, int lam,
                            int beta, int psi, int kind, int cos_i) {
  const int factor = kind == 0 ? 8 : (kind == 1 ? 4 : 2);  // 0 both, 1 long, 2 lat
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
    double* row = c + (long long)r * ndim;
    const int mode = r % factor;
    if ((kind == 0 || kind == 2) && (mode & 1)) {
      row[inc] = cos_i ? -row[inc] : PI - row[inc];
      row[beta] = -row[beta];
      row[psi] = PI - row[psi];
    }
    const int q = kind == 0 ? mode / 2 : (kind == 1 ? mode : 0);
    if (q > 0) {
      row[lam] = py_mod(row[lam] + PI / 2 * q, 2.0 * PI);
      row[psi] = py_mod(row[psi] + PI / 2 * q, PI);
    }
  }
}

}  // namespace bbhx

using namespace bbhx;

extern "C" {

// Front end of a likelihood step (phenomhm.py:175-199 + waveformbuild.py:477-484).
// out [6, B]: m1, m2 (ordered, Msun), chi1, chi2 (swapped with the masses), m1, m2 in kg;
// t_start, t_end [B] (may be null: not computed), tobs_rows [B, M] = t_end - t_start (may be
// null); flags: device int[nflags] cleared, then flags[2] |= 1 if some |chi1z| > 1 and |= 2 if some
// |chi2z| > 1 (may be null).
int bbhx_step_front(double* out, double* t_start, double* t_end, double* tobs_rows,
                    const double* m1, const double* m2, const double* chi1z, const double* chi2z,
                    const double* lam, const double* beta, int num_bin_all, int num_modes,
                    double t_obs_start_L, double t_obs_end_L, int* flags, int nflags,
                    void* stream) {
  BBHX_REQUIRE(num_bin_all >= 0 && num_modes >= 1, "bad sizes");
  BBHX_REQUIRE(flags == nullptr || (nflags >= 3 && nflags <= 32), "nflags must be 3..32");
  cudaStream_t s = (cudaStream_t)stream;
  if (flags != nullptr) {
    k_clear_flags<<<1, 32, 0, s>>>(flags, nflags);
    int st = launch_status("k_clear_flags");
    if (st) return st;
  }
  if (num_bin_all == 0) return OK;
  k_step_front<<<grid_for(num_bin_all, 128), 128, 0, s>>>(out, t_start, t_end, tobs_rows, m1, m2,
                                                          chi1z, chi2z, lam, beta, num_bin_all,
                                                          num_modes, t_obs_start_L, t_obs_end_L,
                                                          flags);
  return launch_status("k_step_front");
}

// orbit-table coverage (fastfdresponse.py:427-433): *flag = 1 if any of tf[0..n) lies outside
// [tmin, tmax]; *flag is only ever set, never cleared
int bbhx_tf_range_check(const double* tf, long long n, double tmin, double tmax, int* flag,
                        void* stream) {
  if (n <= 0) return OK;
  k_tf_range<<<grid_for(n, 256, sm_count() * 4), 256, 0, (cudaStream_t)stream>>>(tf, n, tmin, tmax,
                                                                                flag);
  return launch_status("k_tf_range");
}

// lnL and the values get_ll returns (likelihood.py:204-225) in one device buffer for one copy:
// packed [3 B + nflags] = lnL | Re d_h' | Re h_h | flags; d_h, h_h complex [B]
int bbhx_pack_lnl(double* packed, const void* d_h, const void* h_h, double d_d, int num_bin_all,
                  int phase_marginalize, const int* flags, int nflags, void* stream) {
  BBHX_REQUIRE(num_bin_all >= 0 && nflags >= 0, "bad sizes");
  const int n = num_bin_all + nflags;
  if (n == 0) return OK;
  k_pack_lnl<<<grid_for(n, 128), 128, 0, (cudaStream_t)stream>>>(
      packed, (const cplx*)d_h, (const cplx*)h_h, d_d, num_bin_all, phase_marginalize, flags,
      nflags);
  return launch_status("k_pack_lnl");
}

// tSSBfromLframe (inverse = 0) / tLfromSSBframe (inverse = 1), transform.py:75-135; t0 in s
int bbhx_tssb_from_lframe(double* out, const double* t, const double* lam, const double* beta,
                          int n, double t0, int inverse, void* stream) {
  if (n <= 0) return OK;
  k_tssb<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(out, t, lam, beta, n, t0, inverse);
  return launch_status("k_tssb");
}

// LISA_to_SSB (to_ssb = 1) / SSB_to_LISA (to_ssb = 0), transform.py:136-294; t0 in seconds
int bbhx_frame_transform(double* t_out, double* lam_out, double* beta_out, double* psi_out,
                         const double* t_in, const double* lam_in, const double* beta_in,
                         const double* psi_in, int n, double t0, int to_ssb, void* stream) {
  if (n <= 0) return OK;
  k_frame<<<grid_for(n, 128), 128, 0, (cudaStream_t)stream>>>(t_out, lam_out, beta_out, psi_out,
                                                              t_in, lam_in, beta_in, psi_in, n, t0,
                                                              to_ssb);
  return launch_status("k_frame");
}

// mbh_sky_mode_transform in place on coords [rows, ndim] already tiled by the mode count
// (transform.py:296-426); kind 0 = both (8 modes), 1 = long (4), 2 = lat (2)
int bbhx_sky_mode_transform(double* coords, int rows, int ndim, int inc, int lam, int beta,
                            int psi, int kind, int cos_i, void* stream) {
  BBHX_REQUIRE(kind >= 0 && kind <= 2, "kind must be 0 (both), 1 (long) or 2 (lat)");
  BBHX_REQUIRE(inc >= 0 && inc < ndim && lam >= 0 && lam < ndim && beta >= 0 && beta < ndim &&
                   psi >= 0 && psi < ndim,
               "parameter indices outside [0, ndim)");
  if (rows <= 0) return OK;
  k_sky_modes<<<grid_for(rows, 128), 128, 0, (cudaStream_t)stream>>>(coords, rows, ndim, inc, lam,
                                                                     beta, psi, kind, cos_i);
  return launch_status("k_sky_modes");
}

}  // extern "C"
