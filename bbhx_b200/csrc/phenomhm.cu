// PhenomHM kernels and their C-ABI entry points.
//
// Reference interfaces replaced (src/bbhx/cutils/PhenomHMWaveform.hh:322-371):
//   get_phenomhm_ringdown_frequencies_wrap, get_phenomd_ringdown_frequencies_wrap,
//   waveform_amp_phase.
// Layout of the waveform buffer (phenomhm.py:201-249): flat [nparams, B, M, L] with
// slot 0 = amplitude, 1 = phase, 2 = t(f); freqs flat [B, M, L].
#include <algorithm>
#include <mutex>

#include "capi_internal.cuh"
#include "phenomhm_model.cuh"
#include "sparse_stages.cuh"

namespace bbhx {

// ------------------------------------------------------------------ ringdown frequencies
// thread per (binary, mode); output index b*M + mode (PhenomHMWaveform.cu:1816-1877)
__global__ void k_ringdown_hm(double* fring, double* fdamp, const double* m1, const double* m2,
                              const double* chi1, const double* chi2, const int* ells,
                              const int* mms, int M, int B, int out_stride) {
  long long n = (long long)B * M;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    int b = (int)(t / M), i = (int)(t % M);
    long long o = (long long)b * out_stride + i;
    ringdown_hm(m1[b], m2[b], chi1[b], chi2[b], ells[i], mms[i], &fring[o], &fdamp[o]);
  }
}

__global__ void k_ringdown_d(double* fring, double* fdamp, const double* m1, const double* m2,
                             const double* chi1, const double* chi2, int B, const double* y_rd,
                             const double* c1_rd, const double* c2_rd, const double* c3_rd,
                             const double* y_dm, const double* c1_dm, const double* c2_dm,
                             const double* c3_dm, double dspin, int out_stride, int out_offset) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B; b += gridDim.x * blockDim.x) {
    double fm, fs;
    final_mass_spin(m1[b], m2[b], chi1[b], chi2[b], &fm, &fs);
    double fr, fd;
    phenomd_qnm_lookup(fs, fm, y_rd, c1_rd, c2_rd, c3_rd, y_dm, c1_dm, c2_dm, c3_dm, dspin, &fr,
                       &fd);
    fring[(long long)b * out_stride + out_offset] = fr;
    fdamp[(long long)b * out_stride + out_offset] = fd;
  }
}

// ------------------------------------------------------------------ per-mode setup
// The records of a block's threads are staged in shared memory and written out as one
// contiguous run with 16-byte stores: written straight from each thread, the 848-byte records
// at an 848-byte stride made every warp store touch 32 cache lines.
constexpr int kSetupThreads = 32;
static_assert(sizeof(ModeCoeffs) % 16 == 0, "records are copied in 16-byte words");
__global__ void __launch_bounds__(kSetupThreads)
    k_phm_setup(ModeCoeffs* coeffs, const int* ells, const int* mms, const double* m1_SI,
                const double* m2_SI, const double* chi1, const double* chi2, const double* dist,
                const double* Mf_RD_lm, const double* Mf_DM_lm, int M, int B, int run_phenomd) {
  __shared__ __align__(16) ModeCoeffs stage[kSetupThreads];
  const long long n = (long long)B * M;
  const int add = run_phenomd ? 0 : 1;
  for (long long base = (long long)blockIdx.x * kSetupThreads; base < n;
       base += (long long)gridDim.x * kSetupThreads) {
    const long long t = base + threadIdx.x;
    if (t < n) {
      const int b = (int)(t / M), i = (int)(t % M);
      const double* rd = Mf_RD_lm + (long long)b * (M + add);
      const double* dm = Mf_DM_lm + (long long)b * (M + add);
      const double rd22 = run_phenomd ? rd[0] : rd[M];
      const double dm22 = run_phenomd ? dm[0] : dm[M];
      const int ell = run_phenomd ? 2 : ells[i];
      const int mm = run_phenomd ? 2 : mms[i];
      ModeCoeffs c;
      phm_setup_mode(c, m1_SI[b], m2_SI[b], chi1[b], chi2[b], dist[b], ell, mm, rd[i], dm[i],
                     rd22, dm22, run_phenomd);
      stage[threadIdx.x] = c;
    }
    __syncthreads();
    const int cnt = (int)min((long long)kSetupThreads, n - base);
    const int words = cnt * (int)(sizeof(ModeCoeffs) / 16);
    const uint4* src = reinterpret_cast<const uint4*>(stage);
    uint4* dst = reinterpret_cast<uint4*>(coeffs + base);
    for (int w = threadIdx.x; w < words; w += kSetupThreads) dst[w] = src[w];
    __syncthreads();
  }
}

// ------------------------------------------------------------------ per-point evaluation
// thread per (binary, mode, frequency).  t_ref (optional) adds 2 pi f (t_ref - t_init) to the
// phase and t_ref to t(f), the driver-side shift of phenomhm.py:485-507.
__global__ void k_phm_points(double* out, const double* freqs, const ModeCoeffs* coeffs, int M,
                             int L, int B, const double* t_ref, double t_init) {
  long long n = (long long)B * M * L;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    long long bm = t / L;
    const ModeCoeffs& c = coeffs[bm];
    double f = freqs[t];
    PointOut o = phm_eval_point(c, f);
    if (t_ref) {
      int b = (int)(bm / M);
      double tr = t_ref[b];
      o.phase += f * (tr - t_init) * 2 * PI;
      o.tf += tr;
    }
    out[t] = o.amp;
    out[n + t] = o.phase;
    out[2 * n + t] = o.tf;
  }
}

// t(f) only (first pass of the observation-window regrid)
__global__ void k_phm_tf(double* tf_out, const double* freqs, const ModeCoeffs* coeffs, int M,
                         int L, int B, const double* t_ref) {
  long long n = (long long)B * M * L;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    long long bm = t / L;
    const double tf = phm_tf_value(coeffs[bm], freqs[t]);
    tf_out[t] = tf + (t_ref ? t_ref[bm / M] : 0.0);
  }
}

// ------------------------------------------------------------------ observation window
// One thread per (binary, mode): the linear-interpolation crossing search of
// phenomhm.py:520-606 followed by the log-spaced regrid of :608-610.
//   freqs_in/tf: [BM, L]; Tobs [BM]; writes freqs_out [BM, L] and fminmax [BM, 2].
// err[0] is set to 1 (lower edge) or 2 (upper edge) when a row that needs clipping does not
// have exactly one crossing (the reference raises ValueError there).
// One CTA per row: the edges by block reductions (the same results as the sequential scan),
// then the row's knots by all threads.
__global__ void k_tf_window(double* freqs_out, double* fminmax, const double* freqs_in,
                            const double* tf, const double* Tobs, int L, long long BM, int* err) {
  for (long long r = blockIdx.x; r < BM; r += gridDim.x) {
    const WindowEdges w = tf_window_edges_block(freqs_in + r * L, tf + r * L, L, Tobs[r]);
    if (threadIdx.x == 0) {
      if (w.err) atomicCAS(err, 0, w.err);
      fminmax[2 * r] = w.flo;
      fminmax[2 * r + 1] = w.fhi;
    }
    double* o = freqs_out + r * L;
    for (int k = threadIdx.x; k < L; k += blockDim.x) o[k] = window_knot(k, L, w.flo, w.fhi);
  }
}

// default sparse grid (phenomhm.py:208-224): logspace(mf_min, mf_max, L) / M_sec * m / 2
__global__ void k_default_freqs(double* freqs, const double* m1, const double* m2, const int* mms,
                                double mf_min, double mf_max, int M, int L, int B) {
  long long n = (long long)B * M * L;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    int k = (int)(t % L);
    int i = (int)((t / L) % M);
    int b = (int)(t / ((long long)L * M));
    freqs[t] = default_freq(k, L, mf_min, mf_max, m1[b], m2[b], mms[i]);
  }
}

// ------------------------------------------------------------------ allocation-free variant
// Scratch of bbhx_waveform_amp_phase_noalloc: the per-(binary, mode) model records live in
// this file-scope device array instead of memory obtained with cudaMalloc / cudaMallocAsync.
// It is part of the library's device image, so every GPU that loads the library holds it
// (kNoAllocMaxRecords * sizeof(ModeCoeffs) = 8192 * 848 B, about 6.9 MB) until the process
// exits.  All calls share it.
constexpr long long kNoAllocMaxRecords = 8192;
static_assert(sizeof(ModeCoeffs) == 848, "the documented footprint of the no-alloc array assumes 848-byte records");
static __device__ __align__(256) ModeCoeffs g_noalloc_records[kNoAllocMaxRecords];

}  // namespace bbhx

using namespace bbhx;

namespace {
constexpr int kThreads = 256;

// Device address of g_noalloc_records for the current device, looked up once per device.
// In host code the array's name is only a host-side stand-in, not a device address, so the
// kernels are given the address that cudaGetSymbolAddress returns.  The address is valid for
// the life of the device's primary context: a cudaDeviceReset (which unloads the module) while
// the library is in use is not supported.
std::mutex g_noalloc_mutex;
void* g_noalloc_addr[256] = {};

int noalloc_records(ModeCoeffs** out) {
  int dev = 0;
  BBHX_CHECK_CUDA(cudaGetDevice(&dev));
  BBHX_REQUIRE(dev >= 0 && dev < 256, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (g_noalloc_addr[dev] == nullptr) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_records);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_noalloc_records)");
    g_noalloc_addr[dev] = p;
  }
  *out = (ModeCoeffs*)g_noalloc_addr[dev];
  return OK;
}

int alloc_coeffs(ModeCoeffs** p, long long n, cudaStream_t s) {
  BBHX_CHECK_CUDA(pool_alloc((void**)p, sizeof(ModeCoeffs) * (size_t)n, s));
  return OK;
}
}  // namespace

extern "C" {

size_t bbhx_mode_coeffs_bytes(void) { return sizeof(ModeCoeffs); }

// PhenomHMWaveform.hh:322-333
int bbhx_get_phenomhm_ringdown_frequencies(double* fringdown, double* fdamp, const double* m1,
                                           const double* m2, const double* chi1z,
                                           const double* chi2z, const int* ells, const int* mms,
                                           int num_modes, int num_bin_all, void* stream) {
  BBHX_REQUIRE(num_modes > 0 && num_modes <= MAX_MODES, "num_modes must be 1..6");
  BBHX_REQUIRE(num_bin_all >= 0, "num_bin_all < 0");
  if (num_bin_all == 0) return OK;
  long long n = (long long)num_bin_all * num_modes;
  k_ringdown_hm<<<grid_for(n, kThreads), kThreads, 0, (cudaStream_t)stream>>>(
      fringdown, fdamp, m1, m2, chi1z, chi2z, ells, mms, num_modes, num_bin_all, num_modes);
  return launch_status("k_ringdown_hm");
}

// PhenomHMWaveform.hh:335-352
int bbhx_get_phenomd_ringdown_frequencies(double* fringdown, double* fdamp, const double* m1,
                                          const double* m2, const double* chi1z,
                                          const double* chi2z, int num_bin_all,
                                          const double* y_rd, const double* c1_rd,
                                          const double* c2_rd, const double* c3_rd,
                                          const double* y_dm, const double* c1_dm,
                                          const double* c2_dm, const double* c3_dm, double dspin,
                                          void* stream) {
  BBHX_REQUIRE(num_bin_all >= 0, "num_bin_all < 0");
  BBHX_REQUIRE(dspin > 0.0, "dspin must be positive");
  if (num_bin_all == 0) return OK;
  k_ringdown_d<<<grid_for(num_bin_all, kThreads), kThreads, 0, (cudaStream_t)stream>>>(
      fringdown, fdamp, m1, m2, chi1z, chi2z, num_bin_all, y_rd, c1_rd, c2_rd, c3_rd, y_dm, c1_dm,
      c2_dm, c3_dm, dspin, 1, 0);
  return launch_status("k_ringdown_d");
}

// Both ringdown sets in the [B, M+1] layout that waveform_amp_phase consumes
// (phenomhm.py:397-463 builds it with two calls and a concatenation).  With run_phenomd the
// layout is [B, 1] holding the PhenomD values.
int bbhx_ringdown_frequencies_all(double* fringdown, double* fdamp, const double* m1,
                                  const double* m2, const double* chi1z, const double* chi2z,
                                  const int* ells, const int* mms, int num_modes, int num_bin_all,
                                  const double* qnm_table /* 8 x 1001: y,c1,c2,c3 rd; y,c1,c2,c3 dm */,
                                  int table_len, double dspin, int run_phenomd, void* stream) {
  BBHX_REQUIRE(num_modes > 0 && num_modes <= MAX_MODES, "num_modes must be 1..6");
  BBHX_REQUIRE(table_len > 0 && dspin > 0.0, "bad QNM table");
  if (num_bin_all == 0) return OK;
  cudaStream_t s = (cudaStream_t)stream;
  const double* T = qnm_table;
  int stride = run_phenomd ? 1 : num_modes + 1;
  int off = run_phenomd ? 0 : num_modes;
  if (!run_phenomd) {
    long long n = (long long)num_bin_all * num_modes;
    k_ringdown_hm<<<grid_for(n, kThreads), kThreads, 0, s>>>(
        fringdown, fdamp, m1, m2, chi1z, chi2z, ells, mms, num_modes, num_bin_all, num_modes + 1);
    int st = launch_status("k_ringdown_hm");
    if (st) return st;
  }
  k_ringdown_d<<<grid_for(num_bin_all, kThreads), kThreads, 0, s>>>(
      fringdown, fdamp, m1, m2, chi1z, chi2z, num_bin_all, T, T + table_len, T + 2 * table_len,
      T + 3 * table_len, T + 4 * table_len, T + 5 * table_len, T + 6 * table_len,
      T + 7 * table_len, dspin, stride, off);
  return launch_status("k_ringdown_d");
}

// PhenomHMWaveform.hh:354-371.  waveform_out [3 or more, B, M, L] (amp, phase, tf slots).
int bbhx_waveform_amp_phase(double* waveform_out, const int* ells, const int* mms,
                            const double* freqs, const double* m1_SI, const double* m2_SI,
                            const double* chi1z, const double* chi2z, const double* distance,
                            const double* f_ref, int num_modes, int length, int num_bin_all,
                            const double* Mf_RD_lm, const double* Mf_DM_lm, int run_phenomd,
                            void* stream) {
  (void)f_ref;  // the reference always sets f_ref to the 22 amplitude peak (PhenomHMWaveform.cu:2767)
  BBHX_REQUIRE(num_modes > 0 && num_modes <= MAX_MODES, "num_modes must be 1..6");
  BBHX_REQUIRE(length >= 1 && num_bin_all >= 0, "bad length / num_bin_all");
  if (run_phenomd) BBHX_REQUIRE(num_modes == 1, "run_phenomd requires one mode");
  if (num_bin_all == 0) return OK;
  cudaStream_t s = (cudaStream_t)stream;
  long long nbm = (long long)num_bin_all * num_modes;
  ModeCoeffs* c = nullptr;
  int st = alloc_coeffs(&c, nbm, s);
  if (st) return st;
  k_phm_setup<<<grid_for(nbm, kSetupThreads), kSetupThreads, 0, s>>>(
      c, ells, mms, m1_SI, m2_SI, chi1z, chi2z, distance, Mf_RD_lm, Mf_DM_lm, num_modes,
      num_bin_all, run_phenomd);
  st = launch_status("k_phm_setup");
  if (!st) {
    long long n = nbm * length;
    k_phm_points<<<grid_for(n, kThreads), kThreads, 0, s>>>(waveform_out, freqs, c, num_modes,
                                                            length, num_bin_all, nullptr, 0.0);
    st = launch_status("k_phm_points");
  }
  pool_free(c, s);
  return st;
}

// Allocation-free form of bbhx_waveform_amp_phase, for callers that must not allocate
// device memory: hosts whose own memory pool owns the whole GPU and forbids allocations made
// behind its back, latency-critical loops in which cudaMalloc's implicit device-wide
// synchronisation would stall work on other streams, and deployments without the
// stream-ordered allocator that cudaMallocAsync needs.  Same arguments, layout and results
// as bbhx_waveform_amp_phase; the per-(binary, mode) records go to the library's static
// device array (at most 8192 records, i.e. num_bin_all * num_modes <= 8192; larger requests
// return status 6 without launching anything).
//   * Nothing is allocated or freed: no cudaMalloc / cudaFree / cudaMallocAsync, no library
//     routine that allocates.
//   * The first call on a device looks up the array's device address once for that device
//     (cudaGetSymbolAddress, which may also load the library's device code); make that first
//     call before any stream capture.
//   * Every call uses the same array and it keeps the last call's records.  Each call
//     overwrites every record it reads before reading it, so nothing needs clearing, but calls
//     that overlap on the GPU (different streams, or different host threads, without ordering
//     between them) race on the array: serialise them.
int bbhx_waveform_amp_phase_noalloc(double* waveform_out, const int* ells, const int* mms,
                                    const double* freqs, const double* m1_SI, const double* m2_SI,
                                    const double* chi1z, const double* chi2z,
                                    const double* distance, const double* f_ref, int num_modes,
                                    int length, int num_bin_all, const double* Mf_RD_lm,
                                    const double* Mf_DM_lm, int run_phenomd, void* stream) {
  (void)f_ref;
  BBHX_REQUIRE(num_modes > 0 && num_modes <= MAX_MODES, "num_modes must be 1..6");
  BBHX_REQUIRE(length >= 1 && num_bin_all >= 0, "bad length / num_bin_all");
  if (run_phenomd) BBHX_REQUIRE(num_modes == 1, "run_phenomd requires one mode");
  long long nbm = (long long)num_bin_all * num_modes;
  if (nbm > kNoAllocMaxRecords) {
    set_error("bbhx_waveform_amp_phase_noalloc: num_bin_all * num_modes = %lld exceeds the "
              "static scratch capacity of %lld (binary, mode) records; split the batch or use "
              "bbhx_waveform_amp_phase", nbm, kNoAllocMaxRecords);
    return ERR_TOO_LARGE;
  }
  if (num_bin_all == 0) return OK;
  ModeCoeffs* c = nullptr;
  int st = noalloc_records(&c);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  k_phm_setup<<<grid_for(nbm, kSetupThreads), kSetupThreads, 0, s>>>(
      c, ells, mms, m1_SI, m2_SI, chi1z, chi2z, distance, Mf_RD_lm, Mf_DM_lm, num_modes,
      num_bin_all, run_phenomd);
  st = launch_status("k_phm_setup");
  if (st) return st;
  long long n = nbm * length;
  k_phm_points<<<grid_for(n, kThreads), kThreads, 0, s>>>(waveform_out, freqs, c, num_modes,
                                                          length, num_bin_all, nullptr, 0.0);
  return launch_status("k_phm_points");
}

// Setup records for later fused kernels (caller owns `coeffs`, B*M records of
// bbhx_mode_coeffs_bytes() bytes each).
int bbhx_phenomhm_setup(void* coeffs, const int* ells, const int* mms, const double* m1_SI,
                        const double* m2_SI, const double* chi1z, const double* chi2z,
                        const double* distance, const double* Mf_RD_lm, const double* Mf_DM_lm,
                        int num_modes, int num_bin_all, int run_phenomd, void* stream) {
  BBHX_REQUIRE(num_modes > 0 && num_modes <= MAX_MODES, "num_modes must be 1..6");
  if (num_bin_all == 0) return OK;
  BBHX_REQUIRE(((uintptr_t)coeffs & 15) == 0, "coeffs must be 16-byte aligned");
  long long nbm = (long long)num_bin_all * num_modes;
  k_phm_setup<<<grid_for(nbm, kSetupThreads), kSetupThreads, 0, (cudaStream_t)stream>>>(
      (ModeCoeffs*)coeffs, ells, mms, m1_SI, m2_SI, chi1z, chi2z, distance, Mf_RD_lm, Mf_DM_lm,
      num_modes, num_bin_all, run_phenomd);
  return launch_status("k_phm_setup");
}

// amplitude/phase/t(f) from prepared records, with the t_ref shift fused (t_ref may be null)
int bbhx_phenomhm_points(double* waveform_out, const double* freqs, const void* coeffs,
                         const double* t_ref, double t_init, int num_modes, int length,
                         int num_bin_all, void* stream) {
  if (num_bin_all == 0) return OK;
  long long n = (long long)num_bin_all * num_modes * length;
  k_phm_points<<<grid_for(n, kThreads), kThreads, 0, (cudaStream_t)stream>>>(
      waveform_out, freqs, (const ModeCoeffs*)coeffs, num_modes, length, num_bin_all, t_ref,
      t_init);
  return launch_status("k_phm_points");
}

int bbhx_phenomhm_tf(double* tf_out, const double* freqs, const void* coeffs, const double* t_ref,
                     int num_modes, int length, int num_bin_all, void* stream) {
  if (num_bin_all == 0) return OK;
  long long n = (long long)num_bin_all * num_modes * length;
  k_phm_tf<<<grid_for(n, kThreads), kThreads, 0, (cudaStream_t)stream>>>(
      tf_out, freqs, (const ModeCoeffs*)coeffs, num_modes, length, num_bin_all, t_ref);
  return launch_status("k_phm_tf");
}

int bbhx_default_freqs(double* freqs, const double* m1, const double* m2, const int* mms,
                       double mf_min, double mf_max, int num_modes, int length, int num_bin_all,
                       void* stream) {
  BBHX_REQUIRE(length >= 2, "length must be >= 2");
  if (num_bin_all == 0) return OK;
  long long n = (long long)num_bin_all * num_modes * length;
  k_default_freqs<<<grid_for(n, kThreads), kThreads, 0, (cudaStream_t)stream>>>(
      freqs, m1, m2, mms, mf_min, mf_max, num_modes, length, num_bin_all);
  return launch_status("k_default_freqs");
}

// Observation-window regrid.  `err_dev` is a device int (zeroed by the caller); after the
// stream completes it holds 0, 1 (lower crossing search failed) or 2 (upper).
int bbhx_tf_window_regrid(double* freqs_out, double* fminmax, const double* freqs_in,
                          const double* tf, const double* Tobs, int length, long long num_rows,
                          int* err_dev, void* stream) {
  BBHX_REQUIRE(length >= 2, "length must be >= 2");
  if (num_rows == 0) return OK;
  const unsigned grid = (unsigned)std::min<long long>(num_rows, (long long)sm_count() * 16);
  k_tf_window<<<grid, 128, 0, (cudaStream_t)stream>>>(freqs_out, fminmax, freqs_in, tf, Tobs,
                                                      length, num_rows, err_dev);
  return launch_status("k_tf_window");
}

}  // extern "C"
