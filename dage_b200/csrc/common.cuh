// common.cuh -- shared helpers of libdagegpu.so: status handling, the
// thread-local error message, small device utilities.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/dage_gpu.h"

namespace dage {

// Records a formatted message as the calling thread's last error and
// returns `code` (so call sites can `return fail(...)`).
int fail(int code, const char *fmt, ...);
void clear_error();

#define DAGE_CUDA_TRY(expr)                                                        \
  do {                                                                             \
    cudaError_t _e = (expr);                                                       \
    if (_e != cudaSuccess) {                                                       \
      return ::dage::fail(_e == cudaErrorMemoryAllocation ? DAGE_E_NOMEM : DAGE_E_CUDA, \
                          "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e),  \
                          __FILE__, __LINE__);                                     \
    }                                                                              \
  } while (0)

#define DAGE_TRY(expr)        \
  do {                        \
    int _rc = (expr);         \
    if (_rc != 0) return _rc; \
  } while (0)

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// Number of SMs of the current device (cached per process).
int sm_count();

// RAII-free device buffer owned by an operator handle.
struct DevBuf {
  void *ptr = nullptr;
  size_t bytes = 0;
  int alloc(size_t n);
  void release();
  template <class T>
  T *as() const {
    return static_cast<T *>(ptr);
  }
};

// A DevBuf released when it leaves scope: the temporaries of setup and
// host-pointer calls.  Not copyable, so no second owner can free it.
struct TmpBuf : DevBuf {
  TmpBuf() = default;
  TmpBuf(const TmpBuf &) = delete;
  TmpBuf &operator=(const TmpBuf &) = delete;
  ~TmpBuf() { release(); }
};

}  // namespace dage
