// Host-side helpers shared by the C-ABI translation units: error capture and status codes.
#pragma once

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <initializer_list>
#include <utility>
#include <cuda_runtime.h>

#include "bbhx_common.cuh"
#include "bbhx_b200.h"

namespace bbhx {

// Last error message of the calling host thread (bbhx_last_error_string()).
void set_error(const char* fmt, ...);
const char* get_error();

inline int cuda_status(cudaError_t e, const char* where) {
  if (e == cudaSuccess) return OK;
  set_error("%s: %s", where, cudaGetErrorString(e));
  return ERR_CUDA;
}

#define BBHX_CHECK_CUDA(expr)                                   \
  do {                                                          \
    cudaError_t _e = (expr);                                    \
    if (_e != cudaSuccess) return ::bbhx::cuda_status(_e, #expr); \
  } while (0)

#define BBHX_REQUIRE(cond, ...)          \
  do {                                   \
    if (!(cond)) {                       \
      ::bbhx::set_error(__VA_ARGS__);    \
      return ::bbhx::ERR_BAD_ARG;        \
    }                                    \
  } while (0)

inline int launch_status(const char* kernel) {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return OK;
  set_error("launch of %s failed: %s", kernel, cudaGetErrorString(e));
  return ERR_CUDA;
}

// Keep the stream-ordered pool's memory across synchronisations: the default release
// threshold (0) hands freed pool memory back to the driver at every sync, so the next call's
// cudaMallocAsync would re-map it.  Applied once per device to the device's default pool.
int retain_pool_memory();

// Caller-provided workspace of the calling thread (bbhx_workspace_set): while one is set, the
// entry points' scratch is carved from it, 256-byte aligned, by a bump pointer.  Released
// pieces are reclaimed in stack order (the pieces above the highest live one), and the pointer
// returns to the start when nothing is live (at the end of every entry point).
struct Arena {
  static constexpr int kDepth = 64;  // pieces tracked for stack-order reclamation
  char* base = nullptr;
  size_t size = 0, top = 0, peak = 0;
  int live = 0, depth = 0;
  size_t off[kDepth];
  bool freed[kDepth];
};
Arena& thread_arena();

// Scratch allocation used by the regular entry points: from the caller's workspace when one is
// set, else stream-ordered from the device's default pool.
inline cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t s) {
  Arena& a = thread_arena();
  if (a.base != nullptr) {
    const size_t off = (a.top + 255) & ~(size_t)255;
    a.peak = std::max(a.peak, off + bytes);
    if (off + bytes > a.size) {
      *p = nullptr;
      return cudaErrorMemoryAllocation;
    }
    *p = a.base + off;
    a.top = off + bytes;
    ++a.live;
    if (a.depth < Arena::kDepth) {
      a.off[a.depth] = off;
      a.freed[a.depth] = false;
      ++a.depth;
    }
    return cudaSuccess;
  }
  retain_pool_memory();
  return cudaMallocAsync(p, bytes, s);
}

// Releases scratch from pool_alloc (stream-ordered for pool memory).
inline void pool_free(void* p, cudaStream_t s) {
  if (p == nullptr) return;
  Arena& a = thread_arena();
  if (a.base != nullptr && (char*)p >= a.base && (char*)p < a.base + a.size) {
    const size_t o = (size_t)((char*)p - a.base);
    for (int i = a.depth - 1; i >= 0; --i)
      if (a.off[i] == o && !a.freed[i]) {
        a.freed[i] = true;
        break;
      }
    while (a.depth > 0 && a.freed[a.depth - 1]) a.top = a.off[--a.depth];
    if (--a.live == 0) {
      a.top = 0;
      a.depth = 0;
    }
    return;
  }
  cudaFreeAsync(p, s);
}

// Several stream-ordered allocations, all or none: on a failure the buffers already obtained
// are released (stream-ordered) and every pointer is left null.
inline cudaError_t pool_alloc_all(cudaStream_t s,
                                  std::initializer_list<std::pair<void**, size_t>> req) {
  cudaError_t e = cudaSuccess;
  for (const auto& r : req) *r.first = nullptr;
  for (const auto& r : req) {
    e = pool_alloc(r.first, r.second, s);
    if (e != cudaSuccess) break;
  }
  if (e != cudaSuccess) {
    for (const auto& r : req) {
      pool_free(*r.first, s);
      *r.first = nullptr;
    }
  }
  return e;
}

// Non-finite output detection.  The kernels that write <d|h>, <h|h> set a device word of
// their translation unit when a result is not finite; bbhx_take_status() reads and clears
// the words (one per unit) after synchronising the stream.
int take_nonfinite_likelihood(cudaStream_t s, unsigned* any);
int take_nonfinite_heterodyne(cudaStream_t s, unsigned* any);

// Streaming multiprocessors of the current device (queried once per device and cached);
// grid caps are expressed as multiples of it.
int sm_count();

inline unsigned int grid_for(long long n, int threads, int max_blocks = -1) {
  if (max_blocks < 0) max_blocks = sm_count() * 32;
  long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > max_blocks) b = max_blocks;
  return (unsigned int)b;
}

}  // namespace bbhx
