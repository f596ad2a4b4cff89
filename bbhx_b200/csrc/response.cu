// LISA TDI response kernels, the orbit-table handle, and the fused
// waveform -> response kernel.
//
// Reference interfaces replaced:
//   FastLISAResponse::LISA_response (src/bbhx/cutils/Response.hh:27-41, Response.cu:671-746)
//   AddOrbits::add_orbit_information / dealloc (lisaresponse.pyx:12-13,73-76)
// The reference copies the Orbits object to the device on every call (Response.cu:700-725);
// here the tables live on the device for the lifetime of the handle.
#include <new>

#include "capi_internal.cuh"
#include "phenomhm_model.cuh"
#include "response_model.cuh"
#include "sparse_stages.cuh"

namespace bbhx {

__global__ void k_response_setup(ResponseMode* out, const int* ells, const int* mms,
                                 const double* phi_ref, const double* inc, const double* lam,
                                 const double* beta, const double* psi, int M, int B) {
  long long n = (long long)B * M;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    int b = (int)(t / M), i = (int)(t % M);
    ResponseMode r;
    response_mode_setup(r, ells[i], mms[i], phi_ref[b], inc[b], lam[b], beta[b], psi[b]);
    out[t] = r;
  }
}

// API form: reads phase (slot s0) and t(f) (slot s0+1) of buf, writes the six transfer
// slots and adds the Roemer delay to the phase (Response.cu:321-377).
__global__ void k_response_points(double* buf, const double* freqs, const ResponseMode* rmodes,
                                  OrbitTables orb, int M, int L, int B, int s0, int TDItag,
                                  int rescaled, int tdi2) {
  long long n = (long long)B * M * L;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    long long bm = t / L;
    double f = freqs[t];
    double tf = buf[(long long)(s0 + 1) * n + t];
    Transfer r = response_point(rmodes[bm], orb, f, tf, TDItag, rescaled, tdi2);
    double* tr = buf + (long long)(s0 + 2) * n;
    tr[t] = r.L1.re;
    tr[n + t] = r.L1.im;
    tr[2 * n + t] = r.L2.re;
    tr[3 * n + t] = r.L2.im;
    tr[4 * n + t] = r.L3.re;
    tr[5 * n + t] = r.L3.im;
    buf[(long long)s0 * n + t] += r.phaseRdelay;
  }
}

// Fused: amplitude, phase, t(f) (+ t_ref shift) then the transfer at (f, t(f)); all nine
// slots of the [9, B, M, L] buffer in one pass.
__global__ void k_phm_response(double* buf, const double* freqs, const ModeCoeffs* coeffs,
                               const ResponseMode* rmodes, OrbitTables orb, int M, int L, int B,
                               const double* t_ref, double t_init, int TDItag, int rescaled,
                               int tdi2) {
  long long n = (long long)B * M * L;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    long long bm = t / L;
    int b = (int)(bm / M);
    phm_response_point(buf, n, t, freqs[t], coeffs[bm], rmodes[bm], orb, t_ref[b], t_init,
                       TDItag, rescaled, tdi2);
  }
}

int find_link_slots(const int* links, int out[3]) {
  const int want[3] = {12, 23, 31};
  for (int k = 0; k < 3; ++k) {
    out[k] = -1;
    for (int i = 0; i < 6; ++i)
      if (links[i] == want[k]) out[k] = i;
    if (out[k] < 0) return ERR_BAD_ARG;
  }
  return OK;
}

}  // namespace bbhx

using namespace bbhx;

extern "C" {

size_t bbhx_response_mode_bytes(void) { return sizeof(ResponseMode); }

int bbhx_orbits_create(void** handle) {
  BBHX_REQUIRE(handle != nullptr, "null handle pointer");
  *handle = new (std::nothrow) OrbitHandle();
  if (!*handle) {
    set_error("out of host memory");
    return ERR_BAD_ARG;
  }
  return OK;
}

// lisaresponse.pyx:12 argument order; array arguments are HOST arrays and are copied to
// the device (x_arr [N,3,3], n_arr [N,6,3]; L_arr, sc_r, sc_e are accepted for interface
// compatibility and not needed by the response).
int bbhx_orbits_add_orbit_information(void* handle, double dt, int N, const double* n_arr,
                                      const double* L_arr, const double* x_arr, const int* links,
                                      const int* sc_r, const int* sc_e, double armlength) {
  (void)L_arr;
  (void)sc_r;
  (void)sc_e;
  BBHX_REQUIRE(handle != nullptr, "null orbit handle");
  BBHX_REQUIRE(N >= 2 && dt > 0.0 && armlength > 0.0, "bad orbit table (N=%d dt=%g L=%g)", N, dt,
               armlength);
  OrbitHandle* h = (OrbitHandle*)handle;
  int slots[3];
  BBHX_REQUIRE(find_link_slots(links, slots) == OK, "links must contain 12, 23 and 31");
  if (h->d_x) cudaFree(h->d_x);
  if (h->d_n) cudaFree(h->d_n);
  h->d_x = h->d_n = nullptr;
  h->ready = false;
  BBHX_CHECK_CUDA(cudaMalloc((void**)&h->d_x, sizeof(double) * 9 * (size_t)N));
  BBHX_CHECK_CUDA(cudaMalloc((void**)&h->d_n, sizeof(double) * 18 * (size_t)N));
  BBHX_CHECK_CUDA(cudaMemcpy(h->d_x, x_arr, sizeof(double) * 9 * (size_t)N, cudaMemcpyHostToDevice));
  BBHX_CHECK_CUDA(cudaMemcpy(h->d_n, n_arr, sizeof(double) * 18 * (size_t)N, cudaMemcpyHostToDevice));
  h->tab.x_arr = h->d_x;
  h->tab.n_arr = h->d_n;
  h->tab.dt = dt;
  h->tab.inv_dt = 1.0 / dt;
  h->tab.N = N;
  for (int k = 0; k < 3; ++k) h->tab.link_index[k] = slots[k];
  h->tab.armlength = armlength;
  h->tab.inv_armlength = 1.0 / armlength;
  h->tab.pi_L_over_c = PI * armlength / C_SI;
  h->ready = true;
  return OK;
}

int bbhx_orbits_destroy(void* handle) {
  if (!handle) return OK;
  OrbitHandle* h = (OrbitHandle*)handle;
  if (h->d_x) cudaFree(h->d_x);
  if (h->d_n) cudaFree(h->d_n);
  delete h;
  return OK;
}

// Response.hh:27-41; buf is [(8|9), B, M, L] with slots (amp,) phase, tf, 6 transfers.
int bbhx_LISA_response(void* orbits, double* response_out, const int* ells, const int* mms,
                       const double* freqs, const double* phi_ref, const double* inc,
                       const double* lam, const double* beta, const double* psi, int TDItag,
                       int rescaled, int tdi2, int order_fresnel_stencil, int num_modes,
                       int length, int num_bin_all, int includes_amps, void* stream) {
  BBHX_REQUIRE(orbits && ((OrbitHandle*)orbits)->ready, "orbit information not added");
  BBHX_REQUIRE(order_fresnel_stencil == 0, "order_fresnel_stencil > 0 is not implemented");
  BBHX_REQUIRE(TDItag == 1 || TDItag == 2, "TDItag must be 1 (XYZ) or 2 (AET)");
  BBHX_REQUIRE(num_modes > 0 && num_modes <= MAX_MODES, "num_modes must be 1..6");
  BBHX_REQUIRE(includes_amps == 0 || includes_amps == 1, "includes_amps must be 0 or 1");
  if (num_bin_all == 0 || length == 0) return OK;
  cudaStream_t s = (cudaStream_t)stream;
  long long nbm = (long long)num_bin_all * num_modes;
  ResponseMode* rm = nullptr;
  BBHX_CHECK_CUDA(pool_alloc((void**)&rm, sizeof(ResponseMode) * nbm, s));
  k_response_setup<<<grid_for(nbm, 128), 128, 0, s>>>(rm, ells, mms, phi_ref, inc, lam, beta, psi,
                                                      num_modes, num_bin_all);
  int st = launch_status("k_response_setup");
  if (!st) {
    long long n = nbm * length;
    k_response_points<<<grid_for(n, 128), 128, 0, s>>>(response_out, freqs, rm,
                                                       ((OrbitHandle*)orbits)->tab, num_modes,
                                                       length, num_bin_all, includes_amps,
                                                       TDItag, rescaled, tdi2);
    st = launch_status("k_response_points");
  }
  pool_free(rm, s);
  return st;
}

// Fused PhenomHM + response into a [9, B, M, L] buffer.  `coeffs` from bbhx_phenomhm_setup.
int bbhx_waveform_response_fused(void* orbits, double* buf, const double* freqs,
                                 const void* coeffs, const int* ells, const int* mms,
                                 const double* phi_ref, const double* inc, const double* lam,
                                 const double* beta, const double* psi, const double* t_ref,
                                 double t_init, int TDItag, int rescaled, int tdi2, int num_modes,
                                 int length, int num_bin_all, void* stream) {
  BBHX_REQUIRE(orbits && ((OrbitHandle*)orbits)->ready, "orbit information not added");
  BBHX_REQUIRE(TDItag == 1 || TDItag == 2, "TDItag must be 1 (XYZ) or 2 (AET)");
  BBHX_REQUIRE(num_modes > 0 && num_modes <= MAX_MODES, "num_modes must be 1..6");
  if (num_bin_all == 0 || length == 0) return OK;
  cudaStream_t s = (cudaStream_t)stream;
  long long nbm = (long long)num_bin_all * num_modes;
  ResponseMode* rm = nullptr;
  BBHX_CHECK_CUDA(pool_alloc((void**)&rm, sizeof(ResponseMode) * nbm, s));
  k_response_setup<<<grid_for(nbm, 128), 128, 0, s>>>(rm, ells, mms, phi_ref, inc, lam, beta, psi,
                                                      num_modes, num_bin_all);
  int st = launch_status("k_response_setup");
  if (!st) {
    long long n = nbm * length;
    k_phm_response<<<grid_for(n, 128), 128, 0, s>>>(
        buf, freqs, (const ModeCoeffs*)coeffs, rm, ((OrbitHandle*)orbits)->tab, num_modes, length,
        num_bin_all, t_ref, t_init, TDItag, rescaled, tdi2);
    st = launch_status("k_phm_response");
  }
  pool_free(rm, s);
  return st;
}

}  // extern "C"
