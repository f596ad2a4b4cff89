// Template construction on the data grid (reference-API forms).
//
// Reference interfaces replaced (src/bbhx/cutils/WaveformBuild.hh:6-10):
//   InterpTDI  (WaveformBuild.cu:67-189): per data bin, evaluate the nine splines of each
//              mode at the bin frequency, combine conj(T A e^{i phi}) behind the t(f) gate,
//              sum the modes; one launch per binary on its own stream in the reference, one
//              launch over all binaries here.
//   direct_sum (WaveformBuild.cu:193-296): the same combination directly on the sparse grid.
// Pointer conventions follow the reference bindings: InterpTDI's template / index pointer
// arrays and its start / length / t_start / t_end arrays are HOST arrays (of device
// addresses where they point at data); direct_sum takes device arrays.
#include <algorithm>
#include <vector>

#include "capi_internal.cuh"
#include "spline_eval.cuh"

namespace bbhx {

struct InterpJob {
  cplx* tmpl;       // [3, len]
  const int* inds;  // [M, len]
  int start, len;
  double t_start, t_end;
};

__global__ void k_interp_tdi(const InterpJob* jobs, const double* __restrict__ data_freqs,
                             const double* __restrict__ x, const double* __restrict__ y,
                             const double* __restrict__ c1, const double* __restrict__ c2,
                             const double* __restrict__ c3, int L, int B, int M) {
  const int b = blockIdx.y;
  const InterpJob J = jobs[b];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < J.len; i += gridDim.x * blockDim.x) {
    double f = data_freqs[J.start + i];
    cplx s1 = mk(0, 0), s2 = mk(0, 0), s3 = mk(0, 0);
    for (int m = 0; m < M; ++m) {
      int k = J.inds[(long long)m * J.len + i];
      if (k <= -1 || k >= L - 1) continue;
      long long row = (long long)b * M + m;
      double u = f - x[row * L + k];
      double v[9];
#pragma unroll
      for (int p = 0; p < 9; ++p) {
        long long o = (((long long)p * B + b) * M + m) * L + k;
        v[p] = y[o] + c1[o] * u + c2[o] * (u * u) + c3[o] * (u * u * u);
      }
      if (!tf_gate(v[2], J.t_start, J.t_end)) continue;
      cplx h1, h2, h3;
      combine_channels(v[0], v[1], mk(v[3], v[4]), mk(v[5], v[6]), mk(v[7], v[8]), h1, h2, h3);
      s1 = s1 + h1;
      s2 = s2 + h2;
      s3 = s3 + h3;
    }
    J.tmpl[i] = s1;
    J.tmpl[(long long)J.len + i] = s2;
    J.tmpl[2LL * J.len + i] = s3;
  }
}

__global__ void k_direct_sum(cplx* out, const double* __restrict__ buf, int B, int L, int M,
                             const double* t_start, const double* t_end) {
  long long n = (long long)B * L;
  long long nb = (long long)B * M * L;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    int b = (int)(t / L), i = (int)(t % L);
    cplx s1 = mk(0, 0), s2 = mk(0, 0), s3 = mk(0, 0);
    double ts = t_start[b], te = t_end[b];
    for (int m = 0; m < M; ++m) {
      long long o = ((long long)b * M + m) * L + i;
      double tf = buf[2 * nb + o];
      if (!tf_gate(tf, ts, te)) continue;
      cplx h1, h2, h3;
      combine_channels(buf[o], buf[nb + o], mk(buf[3 * nb + o], buf[4 * nb + o]),
                       mk(buf[5 * nb + o], buf[6 * nb + o]), mk(buf[7 * nb + o], buf[8 * nb + o]),
                       h1, h2, h3);
      s1 = s1 + h1;
      s2 = s2 + h2;
      s3 = s3 + h3;
    }
    out[((long long)b * 3 + 0) * L + i] = s1;
    out[((long long)b * 3 + 1) * L + i] = s2;
    out[((long long)b * 3 + 2) * L + i] = s3;
  }
}

// Template of each binary placed on the full data grid (waveformbuild.py:663-693, fill=True).
struct FillJob {
  const cplx* tmpl;  // [3, len]
  int start, len;
};

// per binary: out[b, c, start + k] = tmpl[c, k] (out zeroed by the caller)
__global__ void k_fill_each(cplx* __restrict__ out, const FillJob* __restrict__ jobs, int N) {
  const int b = blockIdx.y;
  const FillJob J = jobs[b];
  const long long n = 3LL * J.len;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t / J.len), k = (int)(t - (long long)c * J.len);
    out[((long long)b * 3 + c) * N + J.start + k] = J.tmpl[t];
  }
}

// combined: out[c, i] += tmpl_b[c, i - start_b] for every binary covering bin i, added in
// binary order (the reference's loop of slice additions, so the sums round identically)
__global__ void k_fill_combine(cplx* __restrict__ out, const FillJob* __restrict__ jobs, int B,
                               int N, int i0, int i1) {
  const long long n = 3LL * (i1 - i0);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t / (i1 - i0));
    const int i = i0 + (int)(t - (long long)c * (i1 - i0));
    cplx acc = out[(long long)c * N + i];
    for (int b = 0; b < B; ++b) {
      const FillJob& J = jobs[b];
      const int k = i - J.start;
      if (k >= 0 && k < J.len) acc = acc + J.tmpl[(long long)c * J.len + k];
    }
    out[(long long)c * N + i] = acc;
  }
}

}  // namespace bbhx

using namespace bbhx;

extern "C" {

// WaveformBuild.hh:6
int bbhx_InterpTDI(const int64_t* template_ptrs, const double* data_freqs, const double* freqs,
                   const double* y, const double* c1, const double* c2, const double* c3,
                   const double* t_start, const double* t_end, int length, int data_length,
                   int num_bin_all, int num_modes, const int64_t* inds_ptrs,
                   const int* inds_start, const int* ind_lengths, void* stream) {
  BBHX_REQUIRE(length >= 2 && num_modes >= 1, "bad sizes");
  BBHX_REQUIRE(num_bin_all <= 65535, "InterpTDI handles at most 65535 binaries per call");
  if (num_bin_all == 0) return OK;
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<InterpJob> jobs(num_bin_all);
  int maxlen = 0;
  for (int b = 0; b < num_bin_all; ++b) {
    BBHX_REQUIRE(ind_lengths[b] >= 0 && inds_start[b] >= 0 &&
                     (long long)inds_start[b] + ind_lengths[b] <= data_length,
                 "binary %d: data range [%d, %d) outside the data grid", b, inds_start[b],
                 inds_start[b] + ind_lengths[b]);
    jobs[b].tmpl = (cplx*)template_ptrs[b];
    jobs[b].inds = (const int*)inds_ptrs[b];
    jobs[b].start = inds_start[b];
    jobs[b].len = ind_lengths[b];
    jobs[b].t_start = t_start[b];
    jobs[b].t_end = t_end[b];
    if (ind_lengths[b] > maxlen) maxlen = ind_lengths[b];
  }
  if (maxlen == 0) return OK;
  InterpJob* d_jobs = nullptr;
  BBHX_CHECK_CUDA(pool_alloc((void**)&d_jobs, sizeof(InterpJob) * num_bin_all, s));
  BBHX_CHECK_CUDA(cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(InterpJob) * num_bin_all,
                                  cudaMemcpyHostToDevice, s));
  int threads = 256;
  unsigned gx = (unsigned)((maxlen + threads - 1) / threads);
  if (gx > 1024) gx = 1024;
  k_interp_tdi<<<dim3(gx, num_bin_all), threads, 0, s>>>(d_jobs, data_freqs, freqs, y, c1, c2, c3,
                                                         length, num_bin_all, num_modes);
  int st = launch_status("k_interp_tdi");
  pool_free(d_jobs, s);
  // the host job array must outlive the asynchronous copy
  cudaError_t e = cudaStreamSynchronize(s);
  if (!st && e != cudaSuccess) st = cuda_status(e, "InterpTDI sync");
  return st;
}

// fill=True placement of per-binary templates on the data grid (waveformbuild.py:663-693; the
// reference loops over binaries in Python).  template_ptrs, starts, lengths: HOST arrays (the
// pointers are device addresses of [3, len] complex128 templates, e.g. from InterpTDI).
// combine = 0: out [B, 3, N] with each binary in its own row; 1: out [3, N], the templates
// added in binary order.  out (device complex128) must be zeroed or hold the values to add to.
int bbhx_fill_templates(void* out, const int64_t* template_ptrs, const int* starts,
                        const int* lengths, int num_bin_all, int data_length, int combine,
                        void* stream) {
  BBHX_REQUIRE(num_bin_all >= 0 && num_bin_all <= 65535, "num_bin_all must be 0..65535");
  if (num_bin_all == 0) return OK;
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<FillJob> jobs(num_bin_all);
  int maxlen = 0, lo = data_length, hi = 0;
  for (int b = 0; b < num_bin_all; ++b) {
    BBHX_REQUIRE(lengths[b] >= 0 && starts[b] >= 0 &&
                     (long long)starts[b] + lengths[b] <= data_length,
                 "binary %d: data range [%d, %d) outside the data grid", b, starts[b],
                 starts[b] + lengths[b]);
    jobs[b].tmpl = (const cplx*)template_ptrs[b];
    jobs[b].start = starts[b];
    jobs[b].len = lengths[b];
    if (lengths[b] > 0) {
      maxlen = std::max(maxlen, lengths[b]);
      lo = std::min(lo, starts[b]);
      hi = std::max(hi, starts[b] + lengths[b]);
    }
  }
  if (maxlen == 0) return OK;
  FillJob* d_jobs = nullptr;
  BBHX_CHECK_CUDA(pool_alloc((void**)&d_jobs, sizeof(FillJob) * num_bin_all, s));
  int st = cuda_status(cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(FillJob) * num_bin_all,
                                       cudaMemcpyHostToDevice, s),
                       "fill job upload");
  if (!st) {
    if (combine) {
      k_fill_combine<<<grid_for(3LL * (hi - lo), 256), 256, 0, s>>>((cplx*)out, d_jobs,
                                                                    num_bin_all, data_length, lo, hi);
      st = launch_status("k_fill_combine");
    } else {
      unsigned gx = (unsigned)std::min<long long>((3LL * maxlen + 255) / 256, 1024);
      k_fill_each<<<dim3(gx, num_bin_all), 256, 0, s>>>((cplx*)out, d_jobs, data_length);
      st = launch_status("k_fill_each");
    }
  }
  pool_free(d_jobs, s);
  // the host job array must outlive the asynchronous copy
  cudaError_t e = cudaStreamSynchronize(s);
  if (!st && e != cudaSuccess) st = cuda_status(e, "fill sync");
  return st;
}

// WaveformBuild.hh:8-10: templates [B, 3, L] complex128; buffer [9, B, M, L]
int bbhx_direct_sum(double* templates, const double* buffer, int num_bin_all, int length,
                    int n_channels, int num_modes, const double* t_start, const double* t_end,
                    void* stream) {
  BBHX_REQUIRE(n_channels == 3, "n_channels must be 3");
  if (num_bin_all == 0 || length == 0) return OK;
  long long n = (long long)num_bin_all * length;
  k_direct_sum<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
      (cplx*)templates, buffer, num_bin_all, length, num_modes, t_start, t_end);
  return launch_status("k_direct_sum");
}

}  // extern "C"
