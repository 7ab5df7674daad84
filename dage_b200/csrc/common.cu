// common.cu -- error state, device info, device buffers.
#include <cstring>
#include <mutex>

#include "common.cuh"

namespace dage {

namespace {
thread_local char g_last_error[1024] = "";
}

int fail(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return code;
}

void clear_error() { g_last_error[0] = '\0'; }

const char *last_error() { return g_last_error; }

int sm_count() {
  static int count = 0;
  static std::once_flag once;
  std::call_once(once, [] {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
    if (count <= 0) count = 148;
  });
  return count;
}

int DevBuf::alloc(size_t n) {
  if (n <= bytes && ptr) return 0;
  release();
  if (n == 0) return 0;
  cudaError_t e = cudaMalloc(&ptr, n);
  if (e != cudaSuccess) {
    ptr = nullptr;
    return fail(DAGE_E_NOMEM, "cudaMalloc(%zu bytes) failed: %s", n, cudaGetErrorString(e));
  }
  bytes = n;
  return 0;
}

void DevBuf::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
}

}  // namespace dage

extern "C" const char *dage_last_error(void) { return dage::last_error(); }
extern "C" int dage_abi_version(void) { return DAGE_ABI_VERSION; }

namespace dage {
// Iteration limit for bounded device-side waits (mbarrier polls).
long long g_wait_limit = 2000000000LL;
}  // namespace dage

extern "C" int dage_set_wait_limit(long long cycles) {
  if (cycles <= 0) return dage::fail(DAGE_E_INVALID, "wait limit must be positive");
  dage::g_wait_limit = cycles;
  return 0;
}
