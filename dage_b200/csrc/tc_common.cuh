// tc_common.cuh -- pieces shared by the tensor-core stage kernels (the cube
// operator's split-precision stages, op3d_mixed.cu, and the GBFMM near-field
// stages, near_mixed.cu): tile geometry, PTX wrappers for mbarriers, TMA,
// TMEM and tcgen05.mma, shared-memory and instruction descriptors, and the
// FP16 two-part split.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

namespace dage {

constexpr int BM = 128;           // tile rows (TMEM lanes)
constexpr int BN = 128;           // tile columns
constexpr int BK = 32;            // K extent of one shared-memory stage (64-byte rows)
constexpr int kGroup = 32;        // K extent of one main-product partial (and of one
                                  // shared quantum in a fixed-point leading part)

// ---------------------------------------------------------------------------
// PTX wrappers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase of parity `parity` to complete.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > limit) return false;
  }
  return true;
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, uint32_t bar,
                                            int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
      : "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// accumulate flag known at compile time after unrolling (no predicate setup)
__device__ __forceinline__ void umma_bf16_c(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                            uint32_t idesc, bool accumulate) {
  if (accumulate)
    asm volatile("tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, 1;\n" ::"r"(d_tmem),
                 "l"(adesc), "l"(bdesc), "r"(idesc)
                 : "memory");
  else
    asm volatile("tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, 0;\n" ::"r"(d_tmem),
                 "l"(adesc), "l"(bdesc), "r"(idesc)
                 : "memory");
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
      : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// 32 lanes x 16 consecutive 32-bit columns; the wait takes the registers as
// operands so no use of them can be scheduled before the load completes.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                 "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                 "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
               :
               : "memory");
}

// Shared-memory matrix descriptor of a K-major tile written by TMA with the
// 64-byte swizzle: rows of 32 bf16 (64 bytes), 8-row swizzle atoms stacked
// at SBO = 512 bytes.  (K blocks of 64 with 128-byte rows halve the TMA boxes
// per byte but make the band blocks coarser; measured, the two are within a
// few percent and 32 is ahead.)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)1 << 16;           // LBO (unused for swizzled K-major)
  d |= (uint64_t)(512 >> 4) << 32;  // SBO
  d |= (uint64_t)1 << 46;           // descriptor version
  d |= (uint64_t)4 << 61;           // SWIZZLE_64B
  return d;
}

// kind::f16 instruction descriptor: BF16 (F16 = false) or FP16 A and B,
// FP32 D, both K-major.
template <bool F16>
__host__ __device__ constexpr uint32_t idesc_f16kind(int M, int N) {
  return (1u << 4) | (F16 ? 0u : (1u << 7) | (1u << 10)) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

// ---------------------------------------------------------------------------
// FP16 two-part split
// ---------------------------------------------------------------------------
// FP16: floating lead fp16(v) and the fp16 rounding of the rest (the value
// is already scaled into FP16 range).
__device__ __forceinline__ void split_f16_f64(double v, __half (&o)[2]) {
  o[0] = __double2half(v);
  o[1] = __double2half(v - (double)__half2float(o[0]));
}

// Two FP16 parts of a scaled FP32 pair (floating lead), as two half2.
__device__ __forceinline__ void split_pair_f16(float2 v, __half2 (&o)[2]) {
  o[0] = __floats2half2_rn(v.x, v.y);
  const float2 l = __half22float2(o[0]);
  o[1] = __floats2half2_rn(v.x - l.x, v.y - l.y);
}

// One ulp toward larger magnitude: the tensor core rounds its FP32 sums
// toward zero, and a main-product partial (two K=16 MMAs) comes out low in
// magnitude by about one ulp on B200 (measured with FP16 parts: relative
// energy bias -2.2e-7 at 121^3 and -2.8e-7 at 481^3 without this step, i.e.
// 0.8 and 1.1 ulp per partial).  Adding 1 to the bit pattern moves the value
// one ulp away from zero (a zero becomes the smallest subnormal).
__device__ __forceinline__ float unbias_rz(float p) {
  return __uint_as_float(__float_as_uint(p) + 1u);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (null when
// the driver does not provide it).
PFN_cuTensorMapEncodeTiled_v12000 encode_fn();

}  // namespace dage
