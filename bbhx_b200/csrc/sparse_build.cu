// Sparse-grid build of many direct-likelihood problems in one launch (uneven batches).
//
// Replaces, for every (binary, mode) row of every problem, the chain the single-problem path
// runs as separate launches (the reference's phenomhm.py:270-614 + fastfdresponse.py:278-531 +
// interpolate.py:77-211): mass ordering and SSB observation limits, ringdown frequencies,
// PhenomHM record, default grid and its t(f), observation-window regrid, waveform + TDI
// response at the new knots, orbit-coverage check and the not-a-knot spline of the nine
// quantities.  A first launch sets up every row's records (thread per row); then one CTA owns
// one row: it stages the row's records, evaluates the default grid, finds the window edges by
// block reductions, evaluates the knots and solves the spline in shared memory.  The steps are the same device functions as the separate kernels
// (sparse_stages.cuh), so the outputs are the same numbers.
#include <algorithm>
#include <cstring>
#include <vector>

#include "capi_internal.cuh"
#include "sparse_stages.cuh"

namespace bbhx {

constexpr int SB_MAXGROUPS = 64;
constexpr int SB_THREADS = 256;
constexpr size_t kBuildSmemMax = 200 * 1024;

// One problem's build, in device memory (from bbhx_direct_source).
struct BuildArgs {
  const double* params;  // [12, B]
  const int* ells;
  const int* mms;
  const double* qnm;  // [8, nq]
  OrbitTables orb;
  double dspin, mf_min, mf_max, t_init, tL_start, tL_end, orb_tmin, orb_tmax;
  double *x, *y, *c1, *c2, *c3, *t_start, *t_end;
  double* scratch;  // (4 + 9) L doubles per CTA when a row does not fit in shared memory
  ModeCoeffs* coeffs_out;  // heterodyned problems: the walkers' PhenomHM records (no build)
  int* flags;
  int nq, TDItag, rescaled, tdi2, run_phenomd, M, L, B;
};

struct BuildMulti {
  BuildArgs g[2 * SB_MAXGROUPS];  // direct problems, then heterodyned ones
  long long roff[2 * SB_MAXGROUPS + 1];  // row offsets; roff[ngroups] = total rows
  int ngroups;     // direct + heterodyned problems
  int ndirect;     // the first ndirect are built; the rest only get records
  int max_length;  // work-area stride of one CTA in `scratch`
};

// A host struct copied to device memory through kernel parameters, 24 KB per launch (no host
// copy is involved, so the copy is part of a captured graph like any launch).
struct WordChunk {
  unsigned long long w[3072];
};
__global__ void k_store_words(WordChunk c, unsigned long long* dst, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = c.w[i];
}
static_assert(sizeof(BuildMulti) % 8 == 0, "the build table is stored in 8-byte words");

int store_struct(const void* host, size_t bytes, void* dev, cudaStream_t s) {
  const unsigned long long* src = static_cast<const unsigned long long*>(host);
  unsigned long long* dst = static_cast<unsigned long long*>(dev);
  const size_t n = bytes / 8;
  for (size_t o = 0; o < n; o += 3072) {
    WordChunk c;
    const int m = (int)std::min<size_t>(3072, n - o);
    memcpy(c.w, src + o, 8 * (size_t)m);
    k_store_words<<<1, 256, 0, s>>>(c, dst + o, m);
    const int st = launch_status("k_store_words");
    if (st) return st;
  }
  return OK;
}

// Per-row set-up, made by k_row_records (thread per row) and staged into the row's CTA.
struct RowRec {
  ModeCoeffs c;    // PhenomHM record (k_phm_setup)
  ResponseMode r;  // response-mode record (k_response_setup)
  double m1, m2;   // ordered masses [Msun] (the default grid's total mass)
  double To;       // SSB observation span (the regrid's upper edge)
  double t_ref;
};
static_assert(sizeof(RowRec) % 8 == 0, "row records are staged in 8-byte words");

__device__ __forceinline__ int build_group(const BuildMulti* H, long long row) {
  int lo = 0, hi = H->ngroups;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (H->roff[mid] <= row) lo = mid; else hi = mid;
  }
  return lo;
}

// Thread per (problem, binary, mode) row: front end (k_step_front: mass ordering, SSB
// observation limits, |chi| checks), ringdown frequencies (k_ringdown_hm / k_ringdown_d), the
// PhenomHM record (k_phm_setup) and the response-mode record.
__global__ void k_row_records(const BuildMulti* __restrict__ H, RowRec* recs) {
  const long long total = H->roff[H->ngroups];
  for (long long row = blockIdx.x * (long long)blockDim.x + threadIdx.x; row < total;
       row += (long long)gridDim.x * blockDim.x) {
    const int g = build_group(H, row);
    const BuildArgs& A = H->g[g];
    const long long r = row - H->roff[g];
    const int b = (int)(r / A.M), m = (int)(r % A.M);
    const int B = A.B;
    const double* P = A.params;
    const int ell = A.run_phenomd ? 2 : A.ells[m];
    const int mm = A.run_phenomd ? 2 : A.mms[m];
    const double x1 = P[2 * (size_t)B + b], x2 = P[3 * (size_t)B + b];
    const FrontMasses fr = front_masses(P[0 * (size_t)B + b], P[1 * (size_t)B + b], x1, x2);
    const double lam = P[8 * (size_t)B + b], beta = P[9 * (size_t)B + b];
    const double ts = tssb_from_l(A.tL_start, lam, beta, 0.0);
    const double te = tssb_from_l(A.tL_end, lam, beta, 0.0);
    if (m == 0) {
      A.t_start[b] = ts;
      A.t_end[b] = te;
      if (fabs(x1) > 1.0) atomicOr(A.flags + 2, 1);
      if (fabs(x2) > 1.0) atomicOr(A.flags + 2, 2);
    }
    double rd22, dm22, rd, dm;
    ringdown_d(fr.m1, fr.m2, fr.chi1, fr.chi2, A.qnm, A.nq, A.dspin, &rd22, &dm22);
    if (A.run_phenomd) {
      rd = rd22;
      dm = dm22;
    } else {
      ringdown_hm(fr.m1, fr.m2, fr.chi1, fr.chi2, ell, mm, &rd, &dm);
    }
    ModeCoeffs c;
    phm_setup_mode(c, fr.m1_SI, fr.m2_SI, fr.chi1, fr.chi2, P[4 * (size_t)B + b], ell, mm, rd, dm,
                   rd22, dm22, A.run_phenomd);
    if (A.coeffs_out != nullptr) {  // heterodyned walker: its record is all that is needed
      A.coeffs_out[r] = c;
      continue;
    }
    RowRec& R = recs[row];
    R.c = c;
    ResponseMode rm;
    response_mode_setup(rm, ell, mm, P[5 * (size_t)B + b], P[7 * (size_t)B + b], lam, beta,
                        P[10 * (size_t)B + b]);
    R.r = rm;
    R.m1 = fr.m1;
    R.m2 = fr.m2;
    R.To = te - ts;
    R.t_ref = P[11 * (size_t)B + b];
  }
}

__global__ void k_clear_build_flags(const BuildMulti* __restrict__ H) {
  if (blockIdx.x < H->ngroups && threadIdx.x < 3) H->g[blockIdx.x].flags[threadIdx.x] = 0;
}

// row = (problem, binary, mode); rows of all problems, CTAs claiming them from a queue.  The
// row's records come from k_row_records.
__global__ void __launch_bounds__(SB_THREADS) k_sparse_build(const BuildMulti* __restrict__ H,
                                                              const RowRec* __restrict__ recs,
                                                              int use_smem,
                                                              unsigned long long* next) {
  extern __shared__ double sb_smem[];
  __shared__ RowRec R;
  __shared__ long long claimed;
  const int tid = threadIdx.x;
  const long long total = H->roff[H->ndirect];
  // rows are claimed from the launch's queue counter (rows of long sparse grids cost several
  // times those of short ones, so a static row stride leaves CTAs idle)
  for (;;) {
    // every thread is done with the previous claim, its records and its work area
    __syncthreads();
    if (tid == 0) claimed = (long long)atomicAdd(next, 1ull);
    __syncthreads();
    const long long row = claimed;
    if (row >= total) break;
    const int g = build_group(H, row);
    const BuildArgs& A = H->g[g];
    const long long r = row - H->roff[g];
    const int B = A.B, L = A.L;
    const int mm = A.run_phenomd ? 2 : A.mms[(int)(r % A.M)];
    double* work = use_smem ? sb_smem : A.scratch + (size_t)blockIdx.x * (4 + 9) * H->max_length;
    {
      const unsigned long long* src = reinterpret_cast<const unsigned long long*>(recs + row);
      unsigned long long* dst = reinterpret_cast<unsigned long long*>(&R);
      for (int i = tid; i < (int)(sizeof(RowRec) / 8); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    // default grid and its t(f) (k_default_freqs, k_phm_tf) in the work area
    double* f0 = work;
    double* tf0 = work + L;
    for (int k = tid; k < L; k += blockDim.x) {
      const double f = default_freq(k, L, A.mf_min, A.mf_max, R.m1, R.m2, mm);
      f0[k] = f;
      tf0[k] = phm_tf_value(R.c, f) + R.t_ref;
    }
    __syncthreads();
    const WindowEdges w = tf_window_edges_block(f0, tf0, L, R.To);  // (k_tf_window)
    if (tid == 0 && w.err) atomicCAS(A.flags, 0, w.err);
    // knots, waveform + response (k_phm_response) and the orbit-coverage check (k_tf_range)
    const long long n = (long long)B * A.M * L;
    const long long ro = r * L;
    bool bad = false;
    for (int k = tid; k < L; k += blockDim.x) {
      const double xk = window_knot(k, L, w.flo, w.fhi);
      A.x[ro + k] = xk;
      phm_response_point(A.y, n, ro + k, xk, R.c, R.r, A.orb, R.t_ref, A.t_init, A.TDItag,
                         A.rescaled, A.tdi2);
      const double tf = A.y[2 * n + ro + k];
      bad = bad || (tf < A.orb_tmin) || (tf > A.orb_tmax);
    }
    if (__syncthreads_or(bad) && tid == 0) atomicOr(A.flags + 1, 1);
    // not-a-knot spline of the nine quantities (k_spline), reading the row just written
    spline_system(A.x + ro, A.y + ro, n, nullptr, A.c1 + ro, A.c2 + ro, A.c3 + ro, L, 9, work);
  }
}

}  // namespace bbhx

using namespace bbhx;

namespace bbhx {
int uneven_like(const bbhx_direct_group* groups, int num_groups, const bbhx_hdyn_group* hgroups,
                int num_het, int precision, int tile_bins, int ctas_per_sm, cudaStream_t s);
}

extern "C" {

int bbhx_uneven_batch(const bbhx_direct_source* direct, int num_direct,
                      const bbhx_hdyn_source* het, int num_het, int precision, int tile_bins,
                      int ctas_per_sm, void* stream) {
  BBHX_REQUIRE(num_direct >= 0 && num_direct <= SB_MAXGROUPS &&
                   (direct != nullptr || num_direct == 0),
               "num_direct must be 0..%d", SB_MAXGROUPS);
  BBHX_REQUIRE(num_het >= 0 && num_het <= SB_MAXGROUPS && (het != nullptr || num_het == 0),
               "num_het must be 0..%d", SB_MAXGROUPS);
  cudaStream_t s = (cudaStream_t)stream;
  BuildMulti H;
  memset(&H, 0, sizeof(H));
  H.ngroups = num_direct;
  long long rows = 0;
  int maxL = 3;
  for (int g = 0; g < num_direct; ++g) {
    const bbhx_direct_source& D = direct[g];
    BBHX_REQUIRE(D.orbits && ((OrbitHandle*)D.orbits)->ready, "direct group %d: orbit information not added", g);
    BBHX_REQUIRE(D.TDItag == 1 || D.TDItag == 2, "direct group %d: TDItag must be 1 or 2", g);
    BBHX_REQUIRE(D.num_modes >= 1 && D.num_modes <= MAX_MODES && (!D.run_phenomd || D.num_modes == 1),
                 "direct group %d: bad mode count %d", g, D.num_modes);
    BBHX_REQUIRE(D.length >= 4 && D.num_bin_all >= 0 && D.qnm_n >= 2 && D.dspin > 0.0,
                 "direct group %d: bad sizes", g);
    BBHX_REQUIRE(D.x && D.y && D.c1 && D.c2 && D.c3 && D.t_start && D.t_end && D.flags && D.params,
                 "direct group %d: missing buffer", g);
    BuildArgs& A = H.g[g];
    A.params = D.params;
    A.ells = D.ells;
    A.mms = D.mms;
    A.qnm = D.qnm_table;
    A.orb = ((OrbitHandle*)D.orbits)->tab;
    A.dspin = D.dspin;
    A.mf_min = D.mf_min;
    A.mf_max = D.mf_max;
    A.t_init = D.t_init;
    A.tL_start = D.t_obs_start_L;
    A.tL_end = D.t_obs_end_L;
    A.orb_tmin = D.orbit_tmin;
    A.orb_tmax = D.orbit_tmax;
    A.x = D.x;
    A.y = D.y;
    A.c1 = D.c1;
    A.c2 = D.c2;
    A.c3 = D.c3;
    A.t_start = D.t_start;
    A.t_end = D.t_end;
    A.flags = D.flags;
    A.nq = D.qnm_n;
    A.TDItag = D.TDItag;
    A.rescaled = D.rescaled;
    A.tdi2 = D.tdi2;
    A.run_phenomd = D.run_phenomd;
    A.M = D.num_modes;
    A.L = D.length;
    A.B = D.num_bin_all;
    H.roff[g] = rows;
    rows += (long long)D.num_bin_all * D.num_modes;
    maxL = std::max(maxL, D.length);
  }
  const long long rows_direct = rows;
  // heterodyned problems: records and observation limits only
  for (int h = 0; h < num_het; ++h) {
    const bbhx_hdyn_source& S = het[h];
    const bbhx_hdyn_group& G = S.group;
    BBHX_REQUIRE(G.num_modes >= 1 && G.num_modes <= MAX_MODES && (!S.run_phenomd || G.num_modes == 1),
                 "heterodyned group %d: bad mode count %d", h, G.num_modes);
    BBHX_REQUIRE(G.num_bin_all >= 0 && S.qnm_n >= 2 && S.dspin > 0.0,
                 "heterodyned group %d: bad sizes", h);
    BBHX_REQUIRE(S.params && G.coeffs && G.t_start && G.t_end && S.flags && G.ells && G.mms,
                 "heterodyned group %d: missing buffer", h);
    BuildArgs& A = H.g[num_direct + h];
    A.params = S.params;
    A.ells = G.ells;
    A.mms = G.mms;
    A.qnm = S.qnm_table;
    A.dspin = S.dspin;
    A.tL_start = S.t_obs_start_L;
    A.tL_end = S.t_obs_end_L;
    A.t_start = const_cast<double*>(G.t_start);
    A.t_end = const_cast<double*>(G.t_end);
    A.coeffs_out = (ModeCoeffs*)const_cast<void*>(G.coeffs);
    A.flags = S.flags;
    A.nq = S.qnm_n;
    A.run_phenomd = S.run_phenomd;
    A.M = G.num_modes;
    A.L = G.length;
    A.B = G.num_bin_all;
    H.roff[num_direct + h] = rows;
    rows += (long long)G.num_bin_all * G.num_modes;
  }
  H.ngroups = num_direct + num_het;
  H.ndirect = num_direct;
  H.roff[H.ngroups] = rows;
  H.max_length = maxL;
  int st = OK;
  std::vector<void*> scratch;
  if (H.ngroups > 0) {
    const size_t smem = sizeof(double) * (size_t)(4 + 9) * maxL;
    const bool use_smem = smem <= kBuildSmemMax;
    const int nsm = sm_count();
    // two CTAs of SB_THREADS per SM (the register limit at 128 registers a thread)
    const unsigned grid = (unsigned)std::max<long long>(
        1, std::min<long long>(rows_direct, (long long)nsm * 2));
    double* work = nullptr;
    BuildMulti* dH = nullptr;
    RowRec* recs = nullptr;
    unsigned long long* next = nullptr;
    if (pool_alloc((void**)&dH, sizeof(BuildMulti), s) != cudaSuccess ||
        pool_alloc((void**)&recs, sizeof(RowRec) * (size_t)std::max(rows_direct, 1ll), s) != cudaSuccess ||
        pool_alloc((void**)&next, sizeof(unsigned long long), s) != cudaSuccess ||
        (!use_smem && pool_alloc((void**)&work, sizeof(double) * grid * (size_t)(4 + 9) * maxL, s) != cudaSuccess)) {
      set_error("device allocation for the sparse build failed");
      st = ERR_CUDA;
    }
    if (dH) scratch.push_back(dH);
    if (recs) scratch.push_back(recs);
    if (next) scratch.push_back(next);
    if (work) scratch.push_back(work);
    if (!st)
      st = cuda_status(cudaMemsetAsync(next, 0, sizeof(unsigned long long), s),
                       "work-queue counter");
    if (!st) {
      for (int g = 0; g < num_direct; ++g) H.g[g].scratch = work;
      st = store_struct(&H, sizeof(H), dH, s);
    }
    if (!st) {
      k_clear_build_flags<<<H.ngroups, 32, 0, s>>>(dH);
      st = launch_status("k_clear_build_flags");
    }
    if (!st && rows > 0) {
      k_row_records<<<grid_for(rows, 64), 64, 0, s>>>(dH, recs);
      st = launch_status("k_row_records");
    }
    if (!st && rows_direct > 0) {
      if (use_smem)
        st = cuda_status(cudaFuncSetAttribute(k_sparse_build,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)smem),
                         "cudaFuncSetAttribute(k_sparse_build)");
      if (!st) {
        k_sparse_build<<<grid, SB_THREADS, use_smem ? smem : 0, s>>>(dH, recs, use_smem ? 1 : 0,
                                                                     next);
        st = launch_status("k_sparse_build");
      }
    }
  }
  if (!st) {
    std::vector<bbhx_direct_group> groups(std::max(num_direct, 1));
    for (int g = 0; g < num_direct; ++g) {
      const bbhx_direct_source& D = direct[g];
      bbhx_direct_group& G = groups[g];
      G.data_freqs = D.data_freqs;
      G.data = D.data;
      G.noise = D.noise;
      G.data_length = D.data_length;
      G.x = D.x;
      G.y = D.y;
      G.c1 = D.c1;
      G.c2 = D.c2;
      G.c3 = D.c3;
      G.t_start = D.t_start;
      G.t_end = D.t_end;
      G.num_modes = D.num_modes;
      G.length = D.length;
      G.num_bin_all = D.num_bin_all;
      G.d_h = D.d_h;
      G.h_h = D.h_h;
      G.data32 = D.data32;
      G.noise32 = D.noise32;
    }
    std::vector<bbhx_hdyn_group> hgroups(std::max(num_het, 1));
    for (int h = 0; h < num_het; ++h) hgroups[h] = het[h].group;
    st = uneven_like(groups.data(), num_direct, hgroups.data(), num_het, precision, tile_bins,
                     ctas_per_sm, s);
  }
  for (void* p : scratch) pool_free(p, s);
  return st;
}

}  // extern "C"
