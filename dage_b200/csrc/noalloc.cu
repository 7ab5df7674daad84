// noalloc.cu -- an FP64 cube-operator apply that allocates no device memory.
//
// Some callers cannot call cudaMalloc/cudaFree around an operator call:
// processes whose free device memory is held by a caching allocator or a
// fixed pool they do not own (a PyTorch process, or Fortran code that
// registers every buffer up front as the reference does), and tight SCF
// loops that must not hit cudaFree, which synchronises the whole device.
// This entry point takes the operator matrices, the input and the output
// from the caller and keeps its two intermediate cubes in one file-scope
// device array of fixed size instead of allocating them.
#include <mutex>

#include "op3d.cuh"

namespace dage {
namespace {

// Room for the two intermediate cubes U (niy*niz*nox) and W (niz*nox*noy):
// 4 Mi doubles = 32 MiB, e.g. two 121^3 cubes.  Every GPU that loads this
// library holds the array until the process exits.
constexpr size_t kScratchDoubles = size_t(4) << 20;
static __device__ __align__(256) double g_scratch[kScratchDoubles];

// Device address of g_scratch, looked up once per device (the name is only
// a host-side stand-in for the device symbol).
constexpr int kMaxDevices = 64;
double *g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mutex;

int scratch_for_current_device(double **ptr) {
  int dev = 0;
  DAGE_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(DAGE_E_UNSUPPORTED, "device index %d", dev);
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess)
      return fail(DAGE_E_CUDA, "cudaGetSymbolAddress(scratch) failed: %s", cudaGetErrorString(e));
    g_scratch_ptr[dev] = static_cast<double *>(p);
  }
  *ptr = g_scratch_ptr[dev];
  return 0;
}

}  // namespace
}  // namespace dage

using namespace dage;

extern "C" int dage_op3d_apply_fp64_noalloc(int nix, int niy, int niz, int nox, int noy, int noz,
                                            int P, const double *Tx, const double *Ty,
                                            const double *Tz, const double *w, const double *rho,
                                            double *V, void *stream) {
  clear_error();
  if (!Tx || !Ty || !Tz || !w || !rho || !V) return fail(DAGE_E_INVALID, "null argument");
  if (nix < 1 || niy < 1 || niz < 1 || nox < 1 || noy < 1 || noz < 1 || P < 1)
    return fail(DAGE_E_INVALID, "shapes and P must be positive");
  const size_t nU = (size_t)niy * niz * nox, nW = (size_t)niz * nox * noy;
  if (nU + nW > kScratchDoubles)
    return fail(DAGE_E_INVALID,
                "intermediates need %zu doubles; this entry point's fixed scratch holds %zu "
                "(use dage_op3d_apply for larger cubes)",
                nU + nW, kScratchDoubles);
  double *scratch = nullptr;
  DAGE_TRY(scratch_for_current_device(&scratch));
  double *U = scratch, *W = scratch + nU;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t sx = (size_t)nox * nix, sy = (size_t)noy * niy, sz = (size_t)noz * niz;
  for (int p = 0; p < P; ++p) {
    DAGE_TRY(launch_stage_fp64(rho, nix, niy * niz, nox, nix, Tx + sx * p, nix, U, 1.0, false, s));
    DAGE_TRY(launch_stage_fp64(U, niy, niz * nox, noy, niy, Ty + sy * p, niy, W, 1.0, false, s));
    DAGE_TRY(launch_stage_fp64(W, niz, nox * noy, noz, niz, Tz + sz * p, niz, V, w[p], p > 0, s));
  }
  return 0;
}
