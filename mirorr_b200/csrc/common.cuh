// common.cuh -- shared definitions of the mirorr_b200 CUDA library.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/mirorr_b200.h"

namespace mb2 {

// Thread-local last-error message (mirorr_last_error).
void set_error(const char *fmt, ...);
void clear_error();

// Kernel launches issued by this library (process-wide counter, also kept per
// context).  Incremented on the host right after every launch.
extern int64_t g_launches;

// Multiprocessor count of the calling thread's current device (queried once
// per device, then cached); grids of the grid-stride kernels are sized in
// multiples of it.
int sm_count();

struct Status {
  mirorr_status code = MIRORR_OK;
  explicit operator bool() const { return code != MIRORR_OK; }
};

#define MB2_CUDA_TRY(expr)                                                           \
  do {                                                                                \
    cudaError_t e_ = (expr);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      ::mb2::set_error("%s failed at %s:%d: %s", #expr, __FILE__, __LINE__,            \
                       cudaGetErrorString(e_));                                       \
      return e_ == cudaErrorMemoryAllocation ? MIRORR_ENOMEM : MIRORR_ECUDA;           \
    }                                                                                 \
  } while (0)

#define MB2_LAUNCH_CHECK()                                                           \
  do {                                                                                \
    ++::mb2::g_launches;                                                              \
    cudaError_t e_ = cudaGetLastError();                                              \
    if (e_ != cudaSuccess) {                                                          \
      ::mb2::set_error("kernel launch failed at %s:%d: %s", __FILE__, __LINE__,       \
                       cudaGetErrorString(e_));                                       \
      return MIRORR_ECUDA;                                                            \
    }                                                                                 \
  } while (0)

#define MB2_TRY(expr)                                                                \
  do {                                                                                \
    mirorr_status s_ = (expr);                                                        \
    if (s_ != MIRORR_OK) return s_;                                                   \
  } while (0)

// Device buffer that grows on demand and is reused across calls.
struct DevBuf {
  void *ptr = nullptr;
  size_t bytes = 0;
  mirorr_status ensure(size_t n) {
    if (n <= bytes) return MIRORR_OK;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    size_t want = n < 256 ? 256 : n;
    cudaError_t e = cudaMalloc(&ptr, want);
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_error("cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
      return MIRORR_ENOMEM;
    }
    bytes = want;
    return MIRORR_OK;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
  }
  template <class T> T *as() const { return static_cast<T *>(ptr); }
};

// Pinned host buffer that grows on demand.
struct HostBuf {
  void *ptr = nullptr;
  size_t bytes = 0;
  mirorr_status ensure(size_t n) {
    if (n <= bytes) return MIRORR_OK;
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
    size_t want = n < 256 ? 256 : n;
    cudaError_t e = cudaMallocHost(&ptr, want);
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_error("cudaMallocHost(%zu) failed: %s", want, cudaGetErrorString(e));
      return MIRORR_ENOMEM;
    }
    bytes = want;
    return MIRORR_OK;
  }
  void release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
  }
  template <class T> T *as() const { return static_cast<T *>(ptr); }
};

inline int64_t vox(const int32_t s[3]) { return (int64_t)s[0] * s[1] * s[2]; }

#ifdef __CUDACC__
// Splits a linear index o of an (n0, n1, ...) grid, x fastest, into i (along
// n0), j (along n1) and k (the rest); 32-bit division when o fits.
__device__ __forceinline__ void split3(long long o, int n0, int n1, int &i, int &j, int &k) {
  if (o < 0x7fffffffLL) {
    const unsigned int u = (unsigned int)o, t = u / (unsigned int)n0;
    i = (int)(u - t * (unsigned int)n0);
    j = (int)(t % (unsigned int)n1);
    k = (int)(t / (unsigned int)n1);
  } else {
    const long long t = o / n0;
    i = (int)(o - t * n0);
    j = (int)(t % n1);
    k = (int)(t / n1);
  }
}
#endif

}  // namespace mb2
