// Fused heterodyned (relative-binning) likelihood.
//
// Replaces, for the heterodyned path, the chain the reference runs per call
// (likelihood.py:550-648):
//   PhenomHM on the sparse grid   waveform_amp_phase  (PhenomHMWaveform.cu:2891-3060)
//   TDI response                  LISA_response       (Response.cu:671-746)
//   mode sum                      direct_sum          (WaveformBuild.cu:193-296)
//   r = h / h0, layout transpose  (likelihood.py:606-616, host-side numpy/cupy)
//   relative-binning sums         hdyn                (Likelihood.cu:20-201)
// with ONE kernel: a warp owns one walker, stages its per-mode PhenomHM and response records
// in its own slice of shared memory, evaluates amplitude, phase, t(f) and the three TDI transfers at every
// sparse frequency, sums the modes, forms r = h / h0 and reduces the bin terms.  The
// [9, B, M, L] buffer, the [B, 3, L] templates and the transposed residuals are never
// written.
//
// Precision variants (FP64, mixed): het_item.cuh.
#include <algorithm>

#include "capi_internal.cuh"
#include "gradient_model.cuh"
#include "het_item.cuh"

namespace bbhx {

// set when a walker's <d|h> or <h|h> is not finite (read by bbhx_take_status)
static __device__ unsigned g_nonfinite_heterodyne = 0;

int take_nonfinite_heterodyne(cudaStream_t s, unsigned* any) {
  static const unsigned zero = 0;
  unsigned v = 0;
  BBHX_CHECK_CUDA(cudaMemcpyFromSymbolAsync(&v, g_nonfinite_heterodyne, sizeof(v), 0,
                                            cudaMemcpyDeviceToHost, s));
  BBHX_CHECK_CUDA(cudaMemcpyToSymbolAsync(g_nonfinite_heterodyne, &zero, sizeof(zero), 0,
                                          cudaMemcpyHostToDevice, s));
  BBHX_CHECK_CUDA(cudaStreamSynchronize(s));
  *any |= v;
  return OK;
}

// ------------------------------------------------------------------ fused kernel
// Response-mode records of the walkers (thread per (walker, mode)), staged in shared memory
// per block of 32 and written out as one contiguous run of 8-byte words (each thread's 168-byte
// record stored directly made every warp store touch ~40 cache lines).
constexpr int kRespSetupThreads = 32;
__global__ void __launch_bounds__(kRespSetupThreads) k_het_response_setup(HetArgs A) {
  __shared__ ResponseMode stage[kRespSetupThreads];
  const long long n = (long long)A.B * A.M;
  for (long long base = (long long)blockIdx.x * kRespSetupThreads; base < n;
       base += (long long)gridDim.x * kRespSetupThreads) {
    const long long t = base + threadIdx.x;
    if (t < n) stage[threadIdx.x] = het_response_record(A, t);
    __syncwarp();
    const int cnt = (int)min((long long)kRespSetupThreads, n - base);
    const int words = cnt * (int)(sizeof(ResponseMode) / 8);
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(stage);
    unsigned long long* dst =
        reinterpret_cast<unsigned long long*>(const_cast<ResponseMode*>(A.rmodes) + base);
    for (int w = threadIdx.x; w < words; w += kRespSetupThreads) dst[w] = src[w];
    __syncwarp();
  }
}

// One WARP per walker (het_item, het_item.cuh), each warp with its own slice of shared memory:
// no block-wide barrier, so a warp never waits for another walker's slower points or for the
// serial per-walker set-up of the others.  All L residuals of the sparse grid are held in the
// slice (the layout the adjoint needs; the strip layout of the uneven-batch kernel ran this
// kernel ~20 % slower in the mixed form).
template <bool MIXED, bool GH>
__global__ void __launch_bounds__(HET_THREADS, 4) k_het_fused(HetArgs A, unsigned long long* next) {
  extern __shared__ __align__(16) unsigned char het_smem[];
  const HetSmemLayout lay(A.M, A.L, true);
  const int lane = threadIdx.x & 31;
  const HetSlice W(het_smem + (size_t)(threadIdx.x >> 5) * align16(lay.total), lay);
  for (long long b = claim_item(next, lane); b < A.B; b = claim_item(next, lane))
    het_item<MIXED, true, GH>(A, (int)b, W, lane, &g_nonfinite_heterodyne);
}

// Warps (walkers) per CTA of k_het_fused and its dynamic shared memory: up to
// HET_THREADS / 32 warps, as many slices as fit in the opt-in per-block shared memory.
inline int het_launch_shape(int M, int L, bool full_r, int* threads, size_t* smem) {
  const size_t slice = align16(HetSmemLayout(M, L, full_r).total);
  int dev = 0, limit = 48 * 1024;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&limit, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const int w = std::min<int>(HET_THREADS / 32, (int)((size_t)limit / slice));
  if (w < 1) {
    set_error("heterodyne length %d needs %zu B of shared memory per walker (limit %d)", L,
              slice, limit);
    return ERR_TOO_LARGE;
  }
  *threads = 32 * w;
  *smem = slice * w;
  return OK;
}

// Response-mode set-up into scratch, then the walkers; A.rmodes is set here.
template <bool MIXED, bool GH>
int launch_het(HetArgs A, cudaStream_t s) {
  int threads = HET_THREADS;
  size_t smem = 0;
  int st = het_launch_shape(A.M, A.L, true, &threads, &smem);
  if (st) return st;
  ResponseMode* rm = nullptr;
  unsigned long long* next = nullptr;
  BBHX_CHECK_CUDA(pool_alloc_all(s, {{(void**)&rm, sizeof(ResponseMode) * (size_t)A.B * A.M},
                                     {(void**)&next, sizeof(unsigned long long)}}));
  A.rmodes = rm;
  k_het_response_setup<<<grid_for((long long)A.B * A.M, kRespSetupThreads), kRespSetupThreads,
                         0, s>>>(A);
  st = launch_status("k_het_response_setup");
  if (!st)
    st = cuda_status(cudaFuncSetAttribute(k_het_fused<MIXED, GH>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                     "cudaFuncSetAttribute(k_het_fused)");
  if (!st)
    st = cuda_status(cudaMemsetAsync(next, 0, sizeof(unsigned long long), s), "work-queue counter");
  if (!st) {
    // resident CTAs only: every warp claims walkers until the queue drains
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_het_fused<MIXED, GH>, threads,
                                                      smem) != cudaSuccess ||
        per_sm < 1) {
      (void)cudaGetLastError();
      per_sm = 1;
    }
    const long long wpc = threads / 32;
    const unsigned grid =
        (unsigned)std::min<long long>((A.B + wpc - 1) / wpc, (long long)sm_count() * per_sm);
    k_het_fused<MIXED, GH><<<grid, threads, smem, s>>>(A, next);
    st = launch_status("k_het_fused");
  }
  pool_free(rm, s);
  pool_free(next, s);
  return st;
}

}  // namespace bbhx

using namespace bbhx;

namespace {
constexpr int kHetMaxL = 2048;
constexpr int kGradChunk = 4096;  // walkers per dual-number setup / contraction batch
}

namespace bbhx {

// Walker description of one heterodyned problem (validated by the caller).
HetArgs het_args(void* orbits, void* d_h, void* h_h, const void* coeffs, const int* ells,
                 const int* mms, const double* phi_ref, const double* inc, const double* lam,
                 const double* beta, const double* psi, const double* t_ref, double t_init,
                 const double* t_start, const double* t_end, const double* freqs, const void* h0,
                 const void* consts, int TDItag, int rescaled, int tdi2, int num_modes,
                 int length, int num_bin_all) {
  HetArgs A;
  A.d_h = (cplx*)d_h;
  A.h_h = (cplx*)h_h;
  A.coeffs = (const ModeCoeffs*)coeffs;
  A.rmodes = nullptr;
  A.ells = ells;
  A.mms = mms;
  A.phi_ref = phi_ref;
  A.inc = inc;
  A.lam = lam;
  A.beta = beta;
  A.psi = psi;
  A.orb = ((OrbitHandle*)orbits)->tab;
  A.t_ref = t_ref;
  A.t_init = t_init;
  A.t_start = t_start;
  A.t_end = t_end;
  A.freqs = freqs;
  A.h0 = (const cplx*)h0;
  A.consts = (const cplx*)consts;
  A.TDItag = TDItag;
  A.rescaled = rescaled;
  A.tdi2 = tdi2;
  A.gh = nullptr;
  A.M = num_modes;
  A.L = length;
  A.B = num_bin_all;
  return A;
}

int het_check(void* orbits, int TDItag, int num_modes, int length, int precision) {
  BBHX_REQUIRE(orbits && ((OrbitHandle*)orbits)->ready, "orbit information not added");
  BBHX_REQUIRE(TDItag == 1 || TDItag == 2, "TDItag must be 1 (XYZ) or 2 (AET)");
  BBHX_REQUIRE(num_modes > 0 && num_modes <= MAX_MODES, "num_modes must be 1..6");
  BBHX_REQUIRE(length >= 2 && length <= kHetMaxL, "heterodyne length must be 2..%d", kHetMaxL);
  BBHX_REQUIRE(precision == 0 || precision == 1, "precision must be 0 (fp64) or 1 (mixed)");
  return OK;
}

}  // namespace bbhx

extern "C" {

// Heterodyned log-likelihood terms for B walkers in one fused kernel (no reference
// counterpart as one call; same result as waveform_amp_phase + LISA_response + direct_sum +
// r = h / h0 + hdyn, GPU form of hdyn: every bin j >= 1).
int bbhx_hdyn_fused(void* orbits, void* d_h, void* h_h, const void* coeffs, const int* ells,
                    const int* mms, const double* phi_ref, const double* inc, const double* lam,
                    const double* beta, const double* psi, const double* t_ref, double t_init,
                    const double* t_start, const double* t_end, const double* freqs,
                    const void* h0, const void* consts, int TDItag, int rescaled, int tdi2,
                    int num_modes, int length, int num_bin_all, int precision, void* stream) {
  int st = het_check(orbits, TDItag, num_modes, length, precision);
  if (st) return st;
  if (num_bin_all == 0) return OK;
  const HetArgs A = het_args(orbits, d_h, h_h, coeffs, ells, mms, phi_ref, inc, lam, beta, psi,
                             t_ref, t_init, t_start, t_end, freqs, h0, consts, TDItag, rescaled,
                             tdi2, num_modes, length, num_bin_all);
  cudaStream_t s = (cudaStream_t)stream;
  return precision == 1 ? launch_het<true, false>(A, s) : launch_het<false, false>(A, s);
}

// Heterodyned lnL and its gradient d lnL / d theta for the 11 parameters (order in
// gradient_model.cuh) of B walkers: FP64 forward pass that also emits d lnL / d h at the
// sparse grid (reverse part), then dual-number tangents of the waveform + response at every
// (mode, frequency), contracted with those weights (forward part).  params: [12, B] device.
int bbhx_hdyn_grad(void* orbits, void* d_h, void* h_h, double* grad, const void* coeffs,
                   const double* params, const int* ells, const int* mms, const double* qnm_table,
                   int qnm_n, double dspin, double t_init, const double* t_start,
                   const double* t_end, const double* freqs, const void* h0, const void* consts,
                   int TDItag, int rescaled, int tdi2, int run_phenomd, int num_modes, int length,
                   int num_bin_all, void* stream) {
  int st = het_check(orbits, TDItag, num_modes, length, 0);
  if (st) return st;
  BBHX_REQUIRE(qnm_n >= 2 && dspin > 0.0, "bad QNM table");
  if (num_bin_all == 0) return OK;
  cudaStream_t s = (cudaStream_t)stream;
  cplx* gh = nullptr;
  ModeCoeffsT<GD>* cD = nullptr;
  ResponseModeT<GD>* rD = nullptr;
  const int chunk = std::min(num_bin_all, kGradChunk);
  const int nsm = sm_count();
  if (pool_alloc((void**)&gh, sizeof(cplx) * 3 * (size_t)length * num_bin_all, s) != cudaSuccess ||
      pool_alloc((void**)&cD, sizeof(ModeCoeffsT<GD>) * (size_t)chunk * num_modes, s) != cudaSuccess ||
      pool_alloc((void**)&rD, sizeof(ResponseModeT<GD>) * (size_t)chunk * num_modes, s) != cudaSuccess) {
    set_error("device allocation of the gradient scratch failed");
    st = ERR_CUDA;
  }
  if (!st) {
    const size_t B = (size_t)num_bin_all;
    HetArgs A = het_args(orbits, d_h, h_h, coeffs, ells, mms, params + 5 * B, params + 7 * B,
                         params + 8 * B, params + 9 * B, params + 10 * B, params + 11 * B, t_init,
                         t_start, t_end, freqs, h0, consts, TDItag, rescaled, tdi2, num_modes,
                         length, num_bin_all);
    A.gh = gh;
    st = launch_het<false, true>(A, s);
    for (int b0 = 0; !st && b0 < num_bin_all; b0 += chunk) {
      const int nb = std::min(chunk, num_bin_all - b0);
      const long long n = (long long)nb * num_modes;
      for (int k0 = 0; !st && k0 < NGRAD; k0 += GRAD_CHUNK) {
        k_grad_setup<<<grid_for(n, 64), 64, 0, s>>>(cD, rD, params, num_bin_all, b0, nb, ells,
                                                    mms, num_modes, qnm_table, qnm_n, dspin,
                                                    run_phenomd, k0);
        st = launch_status("k_grad_setup");
        if (st) break;
        k_contract_het<<<(unsigned)std::min(nb, nsm * 8), 128, 0, s>>>(
            grad, cD, rD, A.orb, params, num_bin_all, b0, nb, t_start, t_end, t_init, freqs, gh,
            TDItag, rescaled, tdi2, num_modes, length, k0);
        st = launch_status("k_contract_het");
      }
    }
  }
  if (rD) pool_free(rD, s);
  if (cD) pool_free(cD, s);
  if (gh) pool_free(gh, s);
  return st;
}

}  // extern "C"
