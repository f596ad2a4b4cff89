// Library-wide C-ABI helpers: error strings, version, stream sync, device pointer checks.
#include <cstdint>
#include <cstring>

#include "capi_internal.cuh"

namespace bbhx {

static thread_local char g_err[1024] = {0};

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

const char* get_error() { return g_err; }

static thread_local Arena g_arena;
Arena& thread_arena() { return g_arena; }

int sm_count() {
  static int cached[256] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) {
    cudaGetLastError();
    return 148;
  }
  if (cached[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
      cudaGetLastError();
      return 148;
    }
    cached[dev] = n;
  }
  return cached[dev];
}

int retain_pool_memory() {
  static bool done[256] = {};
  int dev = 0;
  BBHX_CHECK_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256 || done[dev]) return OK;
  cudaMemPool_t pool;
  BBHX_CHECK_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
  unsigned long long thr = ~0ULL;
  BBHX_CHECK_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
  done[dev] = true;
  return OK;
}

}  // namespace bbhx

namespace bbhx {
// out[4 i .. 4 i + 3] = (sin, cos) from the hot-loop sincos_cw and (sin, cos) from CUDA's sincos
__global__ void k_selftest_sincos(const double* x, double* out, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s, c, s2, c2;
    sincos_cw(x[i], &s, &c);
    sincos(x[i], &s2, &c2);
    out[4 * i] = s;
    out[4 * i + 1] = c;
    out[4 * i + 2] = s2;
    out[4 * i + 3] = c2;
  }
}
}  // namespace bbhx

extern "C" {

// Self-test of the hot-loop sine/cosine against CUDA's sincos (used by the kernel tests).
int bbhx_selftest_sincos(const double* x, double* out, int n, void* stream) {
  if (n <= 0) return bbhx::OK;
  bbhx::k_selftest_sincos<<<bbhx::grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(x, out, n);
  return bbhx::launch_status("k_selftest_sincos");
}

const char* bbhx_last_error_string(void) { return bbhx::get_error(); }

// Caller-provided workspace for the calling thread's scratch (see bbhx_b200.h).
int bbhx_workspace_set(void* base, size_t bytes) {
  bbhx::Arena& a = bbhx::thread_arena();
  BBHX_REQUIRE(a.live == 0, "the current workspace is in use by %d scratch buffers", a.live);
  if (base == nullptr) {
    a = bbhx::Arena();
    return bbhx::OK;
  }
  BBHX_REQUIRE(((uintptr_t)base & 255u) == 0, "workspace base must be 256-byte aligned");
  BBHX_REQUIRE(bytes >= 256, "workspace must hold at least 256 bytes");
  a.base = (char*)base;
  a.size = bytes;
  a.top = 0;
  a.peak = 0;
  a.live = 0;
  return bbhx::OK;
}

size_t bbhx_workspace_peak(void) { return bbhx::thread_arena().peak; }

int bbhx_version(void) { return 100; }

// Synchronise the stream, then report (and clear) non-finite likelihood outputs written by
// any call since the previous check on this device: 4 if a <d|h> or <h|h> was NaN / inf.
int bbhx_take_status(void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  unsigned any = 0;
  int st = bbhx::take_nonfinite_likelihood(s, &any);
  if (!st) st = bbhx::take_nonfinite_heterodyne(s, &any);
  if (st) return st;
  if (any) {
    bbhx::set_error("a likelihood output (<d|h> or <h|h>) was not finite");
    return bbhx::ERR_NONFINITE;
  }
  return bbhx::OK;
}

int bbhx_stream_synchronize(void* stream) {
  BBHX_CHECK_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  return bbhx::OK;
}

// 1 if ptr is device (or managed) memory visible to the GPU, 0 if host, <0 on error.
int bbhx_pointer_is_device(const void* ptr) {
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, ptr);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) ? 1 : 0;
}

}  // extern "C"
