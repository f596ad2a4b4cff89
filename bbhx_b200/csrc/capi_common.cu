// Library-wide C-ABI helpers: error strings, version, stream sync, device pointer checks.
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

}  // namespace bbhx

extern "C" {

const char* bbhx_last_error_string(void) { return bbhx::get_error(); }

int bbhx_version(void) { return 100; }

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
