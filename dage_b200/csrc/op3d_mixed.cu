// op3d_mixed.cu -- split-precision tensor-core path of the cube operator.
//
// Each "contract the fastest index and rotate" stage (see op3d.cu)
//     D(R, n) = sum_K X(K, R) T(n, K)
// runs on the 5th-generation tensor cores (tcgen05.mma kind::f16, BF16 in,
// FP32 accumulate in TMEM).  Every operand is a sum of BF16 parts,
// X = X0 + X1 [+ X2] and T_p(n, :) / s_n = T0 + T1 [+ T2], s_n the power of
// two at or above the row maximum of |T_p(n, :)| (the entries span many
// decades as t grows).  "bf16x3" uses two parts and the products (0,0)
// (0,1) (1,0); "bf16x6" three parts and the six products with part-index
// sum <= 2.
//
// In bf16x6 the leading parts are fixed point: X0 is a multiple of one
// quantum q = 2^(E-7) shared by each run of 32 consecutive K (2^E >= the
// run's largest |X|), and T0 a multiple of 2^-7 along the whole row, so
// |X0 / q|, |T0 * 2^7| <= 128.  The trailing parts are the BF16 roundings
// of what is left.  A K=32 slice of the main product X0 T0 is then an
// integer below 2^19 times q 2^-7: it is exact in FP32, and the tensor
// core, which rounds its FP32 sums toward zero, never has to round it.  The
// kernel gives every such slice a fresh TMEM partial and adds the partials
// in FP32 registers (round to nearest), so the dominant product carries no
// directed rounding at all.  The correction products (~2^-8 of the main
// one and below) accumulate in TMEM over the whole K range, where the
// rounding direction no longer matters at the 1e-7 level.  bf16x3 keeps
// floating leading parts (the BF16 rounding of each value): with a single
// trailing part a fixed-point lead would leave small elements only 8 bits.
// Its main-product partials therefore carry the tensor core's directed
// rounding (~1e-7 relative), far below that mode's 2^-17 representation
// error.
//
// The epilogue rescales by s_n and writes the next stage's input already
// split.  For that it needs the largest |value| of each 32-run of the next
// stage's K index, which is the current row index R modulo d0: the M tiles
// of an intermediate stage are therefore laid out two-dimensionally, 128
// consecutive values of R mod d0 for one R / d0, so that every warp holds
// exactly one 32-run and a warp-wide max reduction gives its quantum.  The
// last stage multiplies by w_p s_n and adds into V (FP64) with L2
// reductions; the sum over t-points is FP64.  K blocks outside the band of
// the matrix tile (entries below 2^-64 of their row's scale) are skipped.
//
// "fp16x3" keeps the bf16x3 structure (two parts, three products, per-run
// main-product partials) with FP16 parts: 11-bit significands give the two
// parts ~22 bits, so the representation error drops from ~2^-18 to ~2^-23
// per element.  FP16's narrow exponent range is handled by power-of-two
// scales: matrix rows as above times 2^14, stage inputs by one scale per
// stage and t-point from an a-priori bound of the stage's values (max |rho|
// times the largest row L1 norm of each earlier stage's matrix), so every
// stored value is below 2^15 and values below 2^-39 of the bound flush.  The
// tensor core's toward-zero rounding of the FP32 partials (~0.5 ulp per
// rounding, all of one sign for positive sums) is then the largest error
// left; the epilogue adds half an ulp to each partial on average (+1 ulp to
// the odd ones) before summing, which removes that bias.
//
// Kernel structure (one persistent CTA per SM, 18 warps):
//   warp 0      TMA producer: X and T tiles -> shared-memory ring (SW64)
//   warp 1      TMEM allocator + single-thread MMA issuer
//   warps 2-17  epilogue, four warps per scheduler (32 columns each):
//               partial sums -> scale -> split -> global stores
// TMEM holds three 128-column partial buffers (the MMAs of the next slices
// overlap the epilogue's reads) and the 128-column correction accumulator.
// Every mbarrier wait is bounded (clock64 budget); on timeout the CTA
// records the failure in a device flag, drains its in-flight copies and
// MMAs, frees TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "op3d.cuh"
#include "tc_common.cuh"
#include "tune.h"

namespace dage {

extern long long g_wait_limit;

namespace {

constexpr int kThreads = 576;     // 18 warps
constexpr int kEpiThreads = 512;  // warps 2-17
constexpr int kMaxGroup = 8;      // t-points summed per pass of the last stage

// ---------------------------------------------------------------------------
// Splitting into BF16 parts
// ---------------------------------------------------------------------------
// v = lead + rest with lead = j 2^(E-7), |j| <= 128 and 2^E >= m >= |v|, the
// smallest such E.  lead is exact in BF16 (8-bit integer times a power of
// two); v - lead is exact in the working precision.  Runs whose largest
// value is below 2^-119 keep everything in the trailing parts.
__device__ __forceinline__ double lead_f64(double v, double m) {
  if (m == 0.0) return 0.0;
  int E = ilogb(m);
  if (ldexp(1.0, E) != m) ++E;
  if (E < -119) return 0.0;
  return ldexp(rint(ldexp(v, 7 - E)), E - 7);
}
// NS == 2 (bf16x3) keeps a floating leading part: with a single trailing
// part, a fixed-point lead would give small elements only 8 bits.
template <int NS>
__device__ __forceinline__ void split_lead_f64(double v, double m, __nv_bfloat16 (&o)[NS]) {
  const double l = NS == 2 ? (double)__bfloat162float(__double2bfloat16(v)) : lead_f64(v, m);
  o[0] = __double2bfloat16(l);
  double r = v - l;
#pragma unroll
  for (int s = 1; s < NS; ++s) {
    o[s] = __double2bfloat16(r);
    r = r - (double)__bfloat162float(o[s]);
  }
}


// BF16 pair <-> FP32 pair by bit moves (integer pipe).  The epilogue keeps
// its FP32 arithmetic packed (FP32x2) and its conversions off the FP32 FMA
// pipe: dense scalar FP32 work on the MMA issuer's scheduler delays the
// issue of tcgen05.mma.
__device__ __forceinline__ float2 bf16x2_to_f32x2(__nv_bfloat162 h) {
  const uint32_t u = *reinterpret_cast<const uint32_t *>(&h);
  return make_float2(__uint_as_float(u << 16), __uint_as_float(u & 0xffff0000u));
}
// exact when both values are representable in BF16 (the low 16 bits are zero)
__device__ __forceinline__ __nv_bfloat162 f32x2_to_bf16x2_exact(float2 v) {
  const uint32_t u = __byte_perm(__float_as_uint(v.x), __float_as_uint(v.y), 0x7632);
  return *reinterpret_cast<const __nv_bfloat162 *>(&u);
}



// The same split for two values sharing one run maximum m, on packed FP32x2
// arithmetic; part s of (v.x, v.y) lands in o[s] as a BF16 pair.
template <int NS>
__device__ __forceinline__ void split_pair_f32(float2 v, float m, __nv_bfloat162 (&o)[NS]) {
  const float2 neg1 = make_float2(-1.0f, -1.0f);
  float2 l;
  if (NS == 2) {
    o[0] = __floats2bfloat162_rn(v.x, v.y);
    l = bf16x2_to_f32x2(o[0]);
  } else {
    const uint32_t mb = __float_as_uint(m);
    const int E = (int)((mb >> 23) & 0xff) - 127 + ((mb & 0x7fffff) != 0);
    if (m == 0.0f || E < -119) {
      l = make_float2(0.0f, 0.0f);
    } else {
      const float up = __uint_as_float((uint32_t)(127 + 7 - E) << 23);    // 2^(7-E)
      const float down = __uint_as_float((uint32_t)(127 - 7 + E) << 23);  // 2^(E-7)
      const float2 t = __fmul2_rn(v, make_float2(up, up));
      l = __fmul2_rn(make_float2(rintf(t.x), rintf(t.y)), make_float2(down, down));
    }
    o[0] = f32x2_to_bf16x2_exact(l);  // an 8-bit integer times a power of two
  }
  float2 r = __ffma2_rn(l, neg1, v);  // v - lead, exact
#pragma unroll
  for (int s = 1; s < NS; ++s) {
    o[s] = __floats2bfloat162_rn(r.x, r.y);
    r = __ffma2_rn(bf16x2_to_f32x2(o[s]), neg1, r);
  }
}

// ---------------------------------------------------------------------------
// Stage kernel
// ---------------------------------------------------------------------------
struct StageArgs {
  int M, N, K;           // D is M x N, contraction length K
  int n_ntiles, ntiles;  // tiles: m-tile major, n-tile minor
  int nkb, last_k16;     // K blocks; MMAs of K=16 in the last block
  int brow0;             // first row of this t-point in the T-part maps
  // M tiling: nrb == 0: tile mt covers rows [128 mt, 128 mt + 128);
  // nrb > 0 (intermediate stages): tile mt covers R = r1 d0 + r0 with
  // r1 = mt / nrb and r0 in [128 (mt % nrb), +128) intersected with [0, d0)
  int nrb;
  // Sub-problems per tile: the last stage sums ng t-points p0 .. p0+ng-1 in
  // one pass over V; sub-problem g reads A rows from g * gM, matrix rows
  // from brow0 + g * N, bands k_range[g * n_ntiles + nt], scales
  // scale[g * N + n] and weight wcoef[g].  Intermediate stages: ng = 1.
  int ng, gM;
  const float *scale;    // s_n, row scales of the t-points
  const float *wcoef;    // w_p of the t-points (device)
  // FP16 intermediate stages: the stage's power-of-two output factor (device
  // scalar, from the bound-based input scales); null for the BF16 modes
  const float *gscale;
  // intermediate output: part s of element (R, n) at
  //   out[s][(R / d0 + d1 * n) * ldn + R % d0]
  __nv_bfloat16 *out0, *out1, *out2;  // FP16 mode: the same bytes as __half
  int d0, d1;
  long long ldn;
  // final output V[R + M * n] (FP64)
  double *V;
  int accumulate;
  // per t-point and n-tile: first and last K index holding a matrix entry
  // above 2^-64 of its row's scale (the matrices are banded for large t; K
  // blocks outside the band add nothing and are skipped)
  const int2 *k_range;
  int *err;
  long long wait_limit;   // normal waits (dage_set_wait_limit)
  long long drain_limit;  // waits for in-flight copies/MMAs after a timeout
};

template <int NSX, int NS, bool F16 = false>
struct StageCfg {
  static constexpr int kRowBytes = BK * 2;
  static constexpr int kABytes = BM * kRowBytes;  // one part of the A tile
  static constexpr int kBBytes = BN * kRowBytes;  // one part of the B tile
  static constexpr int kStageBytes = NSX * kABytes + NSX * kBBytes;
  // fp16x3 folds its correction products into each 32-run's partial (issued
  // before the main product, so their truncations happen at the corrections'
  // scale, 2^-11 below it): four partial buffers, no correction accumulator
  // and no wait for its drain between tiles (4 % faster at 481^3).  The BF16
  // modes keep a correction accumulator: bf16x6's main-product partials are
  // exact, and bf16x3's corrections, only 2^-8 below the main product, add
  // measurable directed rounding when folded (energy error 8.5e-8 -> 1.4e-7).
  static constexpr bool kFold = F16;
  static constexpr int kNP = kFold ? 4 : 3;       // partial buffers
  static constexpr int kTmemCols = 512;           // 4 x 128 columns
  static constexpr int kSmem = NS * kStageBytes + 1024 + 256;
};

// correction products (a-part, b-part): all pairs with 1 <= a + b <= NSX - 1
__device__ __forceinline__ void corr_product(int nsx, int i, int &a, int &b) {
  if (nsx == 2) {
    const int pa[2] = {1, 0}, pb[2] = {0, 1};
    a = pa[i];
    b = pb[i];
  } else {
    const int pa[5] = {2, 1, 0, 1, 0}, pb[5] = {0, 1, 2, 0, 1};
    a = pa[i];
    b = pb[i];
  }
}

// K blocks [first, last] of the band of sub-problem gi, n-tile nt
__device__ __forceinline__ int2 kblocks(const StageArgs &a, int gi, int nt) {
  const int2 r = a.k_range[gi * a.n_ntiles + nt];
  return make_int2(r.x / BK, r.y / BK);
}

__device__ __forceinline__ int tile_row0(const StageArgs &a, int mt) {
  return a.nrb ? (mt / a.nrb) * a.d0 + (mt % a.nrb) * BM : mt * BM;
}

// The MMAs of one 32-run of K (d0: the run's first K column in the stage):
// the main product (part 0 x part 0) into the fresh partial P, committed to
// `pfull` as soon as it is issued, and the correction products into the
// accumulator Cc.  NK K=16 steps; FIRST: the tile's first run (the
// correction accumulator starts).
template <int NSX, int NK, bool FIRST = false>
__device__ __forceinline__ void mma_run(uint32_t P, uint32_t Cc, uint64_t d0, uint32_t idesc,
                                           bool first, uint32_t pfull_bar) {
  constexpr int kABytes = BM * BK * 2, kBBytes = BN * BK * 2;  // one part of a tile
  constexpr int NCORR = NSX == 2 ? 2 : 5;
#pragma unroll
  for (int k = 0; k < NK; ++k) {
    umma_bf16_c(P, d0 + ((k * 32) >> 4), d0 + ((NSX * kABytes + k * 32) >> 4), idesc, k != 0);
    if (k == NK - 1) umma_commit(pfull_bar);
#pragma unroll
    for (int pr = 0; pr < NCORR; ++pr) {
      int ia, ib;
      corr_product(NSX, pr, ia, ib);
      const uint64_t ad = d0 + ((ia * kABytes + k * 32) >> 4);
      const uint64_t bd = d0 + ((NSX * kABytes + ib * kBBytes + k * 32) >> 4);
      if (NK == 1) {
        umma_bf16(Cc, ad, bd, idesc, (!first || pr != 0) ? 1u : 0u);
      } else {
        umma_bf16_c(Cc, ad, bd, idesc, !(FIRST && k == 0 && pr == 0));
      }
    }
  }
}

// fp16x3: the whole product of one 32-run of K into the fresh
// partial P: the corrections (1 x 0) and (0 x 1) first, then the main
// product (0 x 0) on top, committed to `pfull`.  The tensor core truncates
// every accumulation; the corrections' truncations are ~2^-11 of the main
// product's ulp, so the partial carries the same directed rounding as a
// main-product-only partial (two truncations at its own scale).
template <int NK>
__device__ __forceinline__ void fold_run(uint32_t P, uint64_t d0, uint32_t idesc,
                                         uint32_t pfull_bar) {
  constexpr int kABytes = BM * BK * 2, kBBytes = BN * BK * 2;
#pragma unroll
  for (int k = 0; k < NK; ++k) {
    umma_bf16_c(P, d0 + ((kABytes + k * 32) >> 4), d0 + ((2 * kABytes + k * 32) >> 4), idesc,
                k != 0);
    umma_bf16_c(P, d0 + ((k * 32) >> 4), d0 + ((2 * kABytes + kBBytes + k * 32) >> 4), idesc,
                true);
  }
#pragma unroll
  for (int k = 0; k < NK; ++k)
    umma_bf16_c(P, d0 + ((k * 32) >> 4), d0 + ((2 * kABytes + k * 32) >> 4), idesc, true);
  umma_commit(pfull_bar);
}

// NSX parts per operand; NS shared-memory stages; the main product starts a
// fresh partial every kGroup / 16 MMAs (one 32-run of K).
// 576 threads x 96 registers (55296 of the SM's 65536): one CTA per SM.
template <int NSX, int NS, bool FINAL, bool F16 = false>
__global__ void __maxnreg__(96)
    stage_bf16_kernel(const __grid_constant__ CUtensorMap mapA0,
                      const __grid_constant__ CUtensorMap mapA1,
                      const __grid_constant__ CUtensorMap mapA2,
                      const __grid_constant__ CUtensorMap mapB0,
                      const __grid_constant__ CUtensorMap mapB1,
                      const __grid_constant__ CUtensorMap mapB2, const StageArgs a) {
  using C = StageCfg<NSX, NS, F16>;
  constexpr int GRAN = kGroup / 16;
  // an earlier launch of this apply timed out: do nothing
  if (*reinterpret_cast<volatile int *>(a.err)) return;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t *tiles = smem;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + NS * C::kStageBytes);
  // bars: full[NS], empty[NS], pfull[kNP], pempty[kNP], cfull, cempty, drain
  constexpr int NP = C::kNP;
  constexpr bool FOLD = C::kFold;
  uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(bars + 2 * NS + 2 * NP + 3);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_holder + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto full = [&](int i) { return smem_u32(bars + i); };
  auto empty = [&](int i) { return smem_u32(bars + NS + i); };
  auto pfull = [&](int i) { return smem_u32(bars + 2 * NS + i); };
  auto pempty = [&](int i) { return smem_u32(bars + 2 * NS + NP + i); };
  const uint32_t cfull = smem_u32(bars + 2 * NS + 2 * NP),
                 cempty = smem_u32(bars + 2 * NS + 2 * NP + 1);
  const uint32_t drain = smem_u32(bars + 2 * NS + 2 * NP + 2);

  if (threadIdx.x == 0) {
    for (int i = 0; i < NS; ++i) {
      mbar_init(full(i), 1);
      mbar_init(empty(i), 1);
    }
    for (int i = 0; i < C::kNP; ++i) {
      mbar_init(pfull(i), 1);
      mbar_init(pempty(i), kEpiThreads / 32);  // one arrival per epilogue warp
    }
    mbar_init(cfull, 1);
    mbar_init(cempty, kEpiThreads / 32);
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(smem_u32(tmem_holder), C::kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_holder;
  const uint32_t tmem_corr = tmem_base + C::kNP * BN;
  auto on_timeout = [&]() {
    *abort_flag = 1;
    atomicCAS(a.err, 0, 1);
  };
  // K=16 steps of a tile with K blocks [lo, hi]
  auto tile_steps = [&](int2 r) {
    return (r.y - r.x) * (BK / 16) + (r.y == a.nkb - 1 ? a.last_k16 : BK / 16);
  };

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      const CUtensorMap *mA[3] = {&mapA0, &mapA1, &mapA2};
      const CUtensorMap *mB[3] = {&mapB0, &mapB1, &mapB2};
      int s = 0;
      uint32_t ph = 0;
      int issued[NS];
      uint32_t issued_ph[NS];
      for (int i = 0; i < NS; ++i) issued[i] = 0, issued_ph[i] = 0;
      for (int u = blockIdx.x * a.ng; u < a.ntiles * a.ng && !*abort_flag;
           u += (u % a.ng == a.ng - 1) ? (gridDim.x - 1) * a.ng + 1 : 1) {
        const int tile = u / a.ng, gi = u % a.ng;
        const int row0 = tile_row0(a, tile / a.n_ntiles) + gi * a.gM;
        const int n0 = (tile % a.n_ntiles) * BN + gi * a.N;
        const int2 r = kblocks(a, gi, tile % a.n_ntiles);
        for (int kb = r.x; kb <= r.y; ++kb) {
          if (!mbar_wait(empty(s), ph ^ 1, a.wait_limit)) {
            on_timeout();
            break;
          }
          uint8_t *st = tiles + s * C::kStageBytes;
          mbar_expect_tx(full(s), C::kStageBytes);
#pragma unroll
          for (int i = 0; i < NSX; ++i)
            tma_load_2d(smem_u32(st + i * C::kABytes), mA[i], full(s), kb * BK, row0);
#pragma unroll
          for (int j = 0; j < NSX; ++j)
            tma_load_2d(smem_u32(st + NSX * C::kABytes + j * C::kBBytes), mB[j], full(s),
                        kb * BK, a.brow0 + n0);
          issued[s] = 1;
          issued_ph[s] = ph;
          if (++s == NS) s = 0, ph ^= 1;
        }
      }
      if (*abort_flag)  // let every copy that was issued land first
        for (int i = 0; i < NS; ++i)
          if (issued[i]) mbar_wait(full(i), issued_ph[i], a.drain_limit);
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer
    // The tensor core runs these MMAs back to back only if the issuing
    // thread spends almost nothing between them (a 128x128x16 MMA is 64
    // cycles): every K block is straight-line code with compile-time
    // operand offsets and accumulate flags.
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      int b = 0;            // partial buffer of the current K block (one 32-run)
      uint32_t pph = 0;     // phase of the partial buffers' current round
      int t = 0;
      bool ok = true;
      const uint64_t dbase = sdesc(smem_u32(tiles));
      int u = blockIdx.x * a.ng;
      int2 r = u < a.ntiles * a.ng ? kblocks(a, u % a.ng, (u / a.ng) % a.n_ntiles) : make_int2(0, -1);
      for (; u < a.ntiles * a.ng && ok && !*abort_flag; ++t) {
        const int tile = u / a.ng;
        const int n0 = (tile % a.n_ntiles) * BN;
        int nt = a.N - n0;
        if (nt > BN) nt = BN;
        nt = (nt + 15) & ~15;
        const uint32_t idesc = idesc_f16kind<F16>(BM, nt);
        const int2 rc = r;
        // next tile's band, loaded while this tile's MMAs run
        u += (u % a.ng == a.ng - 1) ? (gridDim.x - 1) * a.ng + 1 : 1;
        if (u < a.ntiles * a.ng) r = kblocks(a, u % a.ng, (u / a.ng) % a.n_ntiles);
        for (int kb = rc.x; kb <= rc.y; ++kb) {
          const bool first = kb == rc.x;
          if (!mbar_wait(full(s), ph, a.wait_limit) ||
              (!FOLD && first && !mbar_wait(cempty, (t & 1) ^ 1, a.wait_limit))) {
            on_timeout();
            ok = false;
            break;
          }
          tc_fence_after();
          const uint64_t d0 = dbase + (uint64_t)((s * C::kStageBytes) >> 4);
          const int nk16 = (kb == a.nkb - 1) ? a.last_k16 : BK / 16;
#pragma unroll
          for (int rr = 0; rr < BK / kGroup; ++rr) {
            const int nk = min(nk16 - rr * GRAN, GRAN);  // K=16 steps of this run
            if (nk <= 0) break;
            if (!mbar_wait(pempty(b), pph ^ 1, a.wait_limit)) {
              on_timeout();
              ok = false;
              break;
            }
            tc_fence_after();
            const uint64_t dr = d0 + (uint64_t)((rr * kGroup * 2) >> 4);
            const uint32_t P = tmem_base + b * BN;
            if (FOLD) {
              if (nk == 1)
                fold_run<1>(P, dr, idesc, pfull(b));
              else
                fold_run<2>(P, dr, idesc, pfull(b));
            } else if (nk == 1) {
              mma_run<NSX, 1>(P, tmem_corr, dr, idesc, first && rr == 0, pfull(b));
            } else if (first && rr == 0) {
              mma_run<NSX, 2, true>(P, tmem_corr, dr, idesc, true, pfull(b));
            } else {
              mma_run<NSX, 2, false>(P, tmem_corr, dr, idesc, false, pfull(b));
            }
            if (++b == C::kNP) b = 0, pph ^= 1;
          }
          if (!ok) break;
          umma_commit(empty(s));
          if (++s == NS) s = 0, ph ^= 1;
        }
        if (ok && !FOLD) umma_commit(cfull);
      }
      // every MMA this thread issued has completed once `drain` fires
      umma_commit(drain);
      mbar_wait(drain, 0, a.drain_limit);
    }
  } else {
    // ------------------------------------------------------------ epilogue
    // 16 warps, four per scheduler: warp w reads TMEM lanes 32 (w % 4) ..
    // +31 (the hardware's lane quarter) and the 32 columns (w - 2) / 4.
    constexpr int CW = BN / 4;
    // Per-column matrix scales matter only for bf16x6 (fixed-point matrix
    // leads on a per-row quantum); bf16x3 splits the unscaled matrix and
    // fp16x3 scales each t-point's matrix by one power of two, folded into
    // the stage factor gfac.
    constexpr bool kColScale = NSX > 2;
    const float gfac = (F16 && !FINAL) ? *a.gscale : 1.0f;
    const int q = warp & 3;
    const uint32_t lane_off = (uint32_t)(32 * q) << 16;
    const uint32_t col0 = ((warp - 2) >> 2) * CW;
    int g = 0, t = 0;
    for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
      float2 acc[CW / 2];   // one t-point, columns (2j, 2j + 1)
      float2 accg[CW / 2];  // last stage: sum over the group of w_p s_n D_p
#pragma unroll
      for (int j = 0; j < CW / 2; ++j) accg[j] = make_float2(0.0f, 0.0f);
      bool ok = true;
      const int ncol = (tile % a.n_ntiles) * BN + col0 + lane;  // this lane's column
      // intermediate stages: the scale of column ncol, loaded before the
      // partial drains so its latency overlaps them
      const float scl = (!FINAL && kColScale && ncol < a.N) ? a.scale[ncol] : 0.0f;
      for (int gi = 0; gi < a.ng && ok; ++gi, ++t) {
        // last stage: w_p s_n of column ncol for sub-problem gi
        const float fcol = (FINAL && ncol < a.N) ? a.wcoef[gi] * a.scale[(size_t)gi * a.N + ncol] : 0.0f;
#pragma unroll
        for (int j = 0; j < CW / 2; ++j) acc[j] = make_float2(0.0f, 0.0f);
        const int nparts =
            (tile_steps(kblocks(a, gi, tile % a.n_ntiles)) + GRAN - 1) / GRAN;
        for (int pi = 0; pi < nparts; ++pi, ++g) {
          const int b = g % C::kNP;
          // warp-uniform outcome: the TMEM loads below are warp-collective
          const bool got = __all_sync(0xffffffffu, mbar_wait(pfull(b), (g / C::kNP) & 1, a.wait_limit));
          if (!got) {
            on_timeout();
            ok = false;
            break;
          }
          tc_fence_after();
#pragma unroll
          for (int hh = 0; hh < 2; ++hh) {  // 16 columns at a time: fewer live registers
            uint32_t r[16];
            tmem_ld16(tmem_base + lane_off + b * BN + col0 + hh * 16, r);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              float2 pv = make_float2(__uint_as_float(r[2 * j]), __uint_as_float(r[2 * j + 1]));
              if (F16) pv = make_float2(unbias_rz(pv.x), unbias_rz(pv.y));
              acc[hh * 8 + j] = __fadd2_rn(acc[hh * 8 + j], pv);
            }
          }
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(pempty(b));
        }
        if (!ok) break;
        if (!FOLD) {
          const bool got = __all_sync(0xffffffffu, mbar_wait(cfull, t & 1, a.wait_limit));
          if (!got) {
            on_timeout();
            ok = false;
            break;
          }
          tc_fence_after();
#pragma unroll
          for (int hh = 0; hh < 2; ++hh) {
            uint32_t r[16];
            tmem_ld16(tmem_corr + lane_off + col0 + hh * 16, r);
#pragma unroll
            for (int j = 0; j < 8; ++j)
              acc[hh * 8 + j] = __fadd2_rn(acc[hh * 8 + j],
                                           make_float2(__uint_as_float(r[2 * j]),
                                                       __uint_as_float(r[2 * j + 1])));
          }
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(cempty);
        }
        if (FINAL) {
#pragma unroll
          for (int j = 0; j < CW / 2; ++j) {
            const float2 f = make_float2(__shfl_sync(0xffffffffu, fcol, 2 * j),
                                         __shfl_sync(0xffffffffu, fcol, 2 * j + 1));
            accg[j] = __ffma2_rn(f, acc[j], accg[j]);
          }
        }
      }
      if (!ok) break;
      const int mt = tile / a.n_ntiles, n0 = (tile % a.n_ntiles) * BN + col0;
      if (FINAL) {
        // V[R + M n] (+)= sum over the group of w_p s_n D_p (FP32 sum of the
        // group's terms, round to nearest).  Additions are L2 reductions:
        // each element gets exactly one correctly rounded FP64 add per group,
        // and the warp does not wait for the old values.
        const int R = mt * BM + 32 * q + lane;
        if (R < a.M) {
          double *col = a.V + (size_t)R;
#pragma unroll
          for (int j = 0; j < CW; ++j) {
            const int n = n0 + j;
            if (n < a.N) {
              const double add = (double)((j & 1) ? accg[j >> 1].y : accg[j >> 1].x);
              double *dst = col + (size_t)a.M * n;
              if (a.accumulate)
                atomicAdd(dst, add);
              else
                __stcs(dst, add);
            }
          }
        }
      } else {
        // next stage: row R / d0 + d1 n, K index R mod d0; this warp holds
        // one aligned 32-run of that K index.  Columns go in pairs: the two
        // lanes of a pair swap one value so that the even lane holds K
        // indices (r0, r0 + 1) of column j and the odd lane those of column
        // j + 1; each stores its two elements as one packed BF16 pair per
        // part.  (ld is even; index d0 < ld is padding and receives zeros.)
        const int r1 = mt / a.nrb;
        const int r0 = (mt % a.nrb) * BM + 32 * q + lane;
        const bool valid = r0 < a.d0;
        const bool odd = lane & 1;
        const int rpair = r0 & ~1;
        // The warp's 32 column scales are one per lane (scl, loaded at the
        // tile's start): loads placed between the loop's global stores could
        // not be moved ahead of them (the compiler cannot rule out aliasing),
        // and each would expose its full latency.
#pragma unroll
        for (int j = 0; j < CW; j += 2) {
          const int n = n0 + j;
          if (n < a.N) {  // uniform across the warp
            const bool has1 = n + 1 < a.N;
            const float2 sc = kColScale ? make_float2(__shfl_sync(0xffffffffu, scl, j),
                                                      __shfl_sync(0xffffffffu, scl, j + 1))
                                        : make_float2(gfac, gfac);
            const float2 v = !valid ? make_float2(0.0f, 0.0f)
                             : (kColScale || F16) ? __fmul2_rn(acc[j >> 1], sc) : acc[j >> 1];
            float m = 0.0f;
            if (NSX > 2) {
              const float m0 =
                  __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(v.x) & 0x7fffffffu));
              const float m1 =
                  __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(v.y) & 0x7fffffffu));
              m = odd ? m1 : m0;
            }
            const float recv = __shfl_xor_sync(0xffffffffu, odd ? v.x : v.y, 1);
            const float mine = odd ? v.y : v.x;
            const float2 vv = odd ? make_float2(recv, mine) : make_float2(mine, recv);
            const size_t off =
                (size_t)(r1 + (long long)a.d1 * (n + (odd ? 1 : 0))) * a.ldn + rpair;
            const bool store = rpair < a.d0 && (!odd || has1);
            if (F16) {
              __half2 hh2[2];
              split_pair_f16(vv, hh2);
              if (store) {
                *reinterpret_cast<__half2 *>(a.out0 + off) = hh2[0];
                *reinterpret_cast<__half2 *>(a.out1 + off) = hh2[1];
              }
            } else {
              __nv_bfloat162 pp[NSX];
              split_pair_f32<NSX>(vv, m, pp);
              if (store) {
                *reinterpret_cast<__nv_bfloat162 *>(a.out0 + off) = pp[0];
                *reinterpret_cast<__nv_bfloat162 *>(a.out1 + off) = pp[1];
                if (NSX > 2) *reinterpret_cast<__nv_bfloat162 *>(a.out2 + off) = pp[NSX > 2 ? 2 : 0];
              }
            }
          }
        }
      }
    }
  }

  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem_base, C::kTmemCols);
  }
}

// ---------------------------------------------------------------------------
// Input and matrix preparation
// ---------------------------------------------------------------------------
// rho (FP64, x fastest, rows of K) -> NSX BF16 parts, rows of ld elements.
// One warp per 32-run of a row; the run's largest |rho| sets the quantum of
// the leading part.  Elements K..ld-1 are written as zeros.
template <int NSX>
__global__ void split_input_kernel(const double *__restrict__ rho, int K, long long rows,
                                   long long ld, __nv_bfloat16 *o0, __nv_bfloat16 *o1,
                                   __nv_bfloat16 *o2) {
  const int runs = (int)((ld + kGroup - 1) / kGroup);
  const long long nwork = rows * runs;
  const int lane = threadIdx.x & 31;
  const long long wstride = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; w < nwork;
       w += wstride) {
    const long long r = w / runs;
    const int k = (int)(w % runs) * kGroup + lane;
    const double v = k < K ? rho[r * K + k] : 0.0;
    double m = fabs(v);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    __nv_bfloat16 p[NSX];
    split_lead_f64<NSX>(v, m, p);
    if (k < ld) {
      const size_t off = (size_t)r * ld + k;
      o0[off] = p[0];
      o1[off] = p[1];
      if (NSX > 2) o2[off] = p[NSX > 2 ? 2 : 0];
    }
  }
}

// FP16 mode: rho * 2^-e0 (device scalar *gin, from max |rho|) -> two FP16
// parts, rows of ld elements, zeros from K to ld.
__global__ void split_input_f16_kernel(const double *__restrict__ rho, int K, long long rows,
                                       long long ld, const float *__restrict__ gin, __half *o0,
                                       __half *o1) {
  const double g = (double)*gin;
  // one warp per row, lanes over k (no per-element index division)
  const int lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows;
       r += nwarps) {
    for (int k = lane; k < ld; k += 32) {
      __half p[2];
      split_f16_f64(k < K ? rho[r * K + k] * g : 0.0, p);
      o0[r * ld + k] = p[0];
      o1[r * ld + k] = p[1];
    }
  }
}

// max |rho| as the bits of a non-negative float (ordered like the values);
// *out must start at 0.
__global__ void absmax_kernel(const double *__restrict__ x, long long n, unsigned *out) {
  float m = 0.0f;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x)
    m = fmaxf(m, (float)fabs(x[e]));
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

// Power-of-two scales of the FP16 mode for one apply.  With M = max |rho|
// (rounded up to a float) and L_a(p) the largest row L1 norm of axis a's
// matrix at t-point p, stage s of t-point p stores its input times 2^-e_s(p),
//   e_0 = floor(log2 M) - 14,  e_1(p) = floor(log2(M L_x)) - 14,
//   e_2(p) = floor(log2(M L_x L_y)) - 14,
// so every stored value is below 2^15.  Axis a's matrix parts at t-point p
// carry 2^14 / S_a(p), S_a(p) the power of two at or above the matrix's
// largest |entry|; the stage epilogues multiply by g_s(p) = S(p) 2^(e_s - 14 -
// e_(s+1)) and the last stage by w_p S_z(p) 2^(e_2 - 14).  gin = 2^-e_0.
__global__ void f16_scales_kernel(const unsigned *maxbits, const double *l1x, const double *l1y,
                                  const double *sx, const double *sy, const double *sz,
                                  const double *w, int P, float *gin, float *g01, float *wcoef) {
  const double M = (double)__uint_as_float(*maxbits);
  auto ex = [](double b) { return b > 0.0 ? (int)floor(log2(b)) - 14 : 0; };
  const int e0 = ex(M);
  if (blockIdx.x == 0 && threadIdx.x == 0) *gin = (float)ldexp(1.0, -e0);
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
    const int e1 = ex(M * l1x[p]), e2 = ex(M * l1x[p] * l1y[p]);
    g01[p] = (float)(sx[p] * ldexp(1.0, e0 - 14 - e1));
    g01[P + p] = (float)(sy[p] * ldexp(1.0, e1 - 14 - e2));
    wcoef[p] = (float)(w[p] * sz[p] * ldexp(1.0, e2 - 14));
  }
}

// Per t-point: the largest row L1 norm of the matrix (out) and the power of
// two at or above its largest |entry| (pscale); one block per t-point over
// its n rows of K values.
__global__ void row_l1max_kernel(const double *__restrict__ T, int N, int K, double *out,
                                 double *pscale) {
  const double *Tp = T + (size_t)blockIdx.x * N * K;
  double m = 0.0, mx = 0.0;
  for (int n = threadIdx.x >> 5; n < N; n += blockDim.x >> 5) {
    double sum = 0.0;
    for (int k = threadIdx.x & 31; k < K; k += 32) {
      const double v = fabs(Tp[(size_t)n * K + k]);
      sum += v;
      mx = fmax(mx, v);
    }
    for (int o = 16; o > 0; o >>= 1) {
      sum += __shfl_xor_sync(0xffffffffu, sum, o);
      mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    m = fmax(m, sum);
  }
  __shared__ double red[32], redx[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m, redx[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0, rx = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r = fmax(r, red[i]), rx = fmax(rx, redx[i]);
    out[blockIdx.x] = r;
    pscale[blockIdx.x] = rx > 0.0 ? exp2(ceil(log2(rx))) : 1.0;
  }
}

// One block per matrix row (p, n).  bf16x6: s = 2^ceil(log2 max_K |T|),
// parts of T / s with the leading part on the quantum 2^-7.  bf16x3: the
// floating BF16 parts of T itself (s = 1).  fp16x3: floating FP16 parts of
// 2^14 T / S(p), S(p) the t-point's power-of-two scale (pscale, rows of N),
// and s = 1 (S(p) goes into the stage factors).
template <int NSX, bool F16 = false>
__global__ void split_matrix_kernel(const double *__restrict__ T, int K, long long ld,
                                    float *scale, double *scale64, __nv_bfloat16 *o0,
                                    __nv_bfloat16 *o1, __nv_bfloat16 *o2,
                                    const double *__restrict__ pscale = nullptr, int N = 1) {
  const long long row = blockIdx.x;
  const double *src = T + row * K;
  __shared__ double red[32];
  double m = 0.0;
  for (int k = threadIdx.x; k < K; k += blockDim.x) m = fmax(m, fabs(src[k]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) red[0] = m;
  }
  __syncthreads();
  // power-of-two scale: the division is exact
  const double s = (NSX == 2 || F16) ? 1.0 : red[0] > 0.0 ? exp2(ceil(log2(red[0]))) : 1.0;
  const double tsc = F16 ? ldexp(1.0, 14) / pscale[row / N] : 1.0;
  if (threadIdx.x == 0) {
    scale[row] = (float)s;
    scale64[row] = s;
  }
  for (int k = threadIdx.x; k < (int)ld; k += blockDim.x) {
    const size_t off = (size_t)row * ld + k;
    if (F16) {
      __half h[2];
      split_f16_f64(k < K ? src[k] * tsc : 0.0, h);
      reinterpret_cast<__half *>(o0)[off] = h[0];
      reinterpret_cast<__half *>(o1)[off] = h[1];
      continue;
    }
    __nv_bfloat16 p[NSX];
    split_lead_f64<NSX>(k < K ? src[k] / s : 0.0, 1.0, p);
    o0[off] = p[0];
    o1[off] = p[1];
    if (NSX > 2) o2[off] = p[NSX > 2 ? 2 : 0];
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

// 2-D BF16 map: inner extent `inner` (contiguous), `rows` rows of `ld`
// elements; box = box_inner x box_rows with the swizzle matching BK.
int make_map(CUtensorMap *m, const void *base, long long inner, long long rows, long long ld,
             int box_inner, int box_rows) {
  auto fn = encode_fn();
  if (!fn) return fail(DAGE_E_CUDA, "cuTensorMapEncodeTiled unavailable");
  if (reinterpret_cast<uintptr_t>(base) % 16 || (ld * 2) % 16)
    return fail(DAGE_E_INVALID, "tensor map base/stride not 16-byte aligned");
  cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(ld * 2)};
  cuuint32_t box[2] = {(cuuint32_t)box_inner, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  const CUtensorMapSwizzle sw =
      box_inner == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B;
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims,
                  strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(DAGE_E_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return 0;
}

struct MixedState {
  bool f16 = false; // FP16 parts (fp16x3) instead of BF16
  int nparts = 2;   // BF16 parts per operand
  int G = 1;        // t-points per pass of the last stage (used slots of X[2])
  int Gmax = 1;     // allocated slots of X[2]
  int ns = 6;       // TMA/MMA ring stages of the stage kernel (autotuned)
  DevBuf wdev;      // w_p as FP32 on the device
  long long ld[3];  // padded K extent of each stage's input rows
  long long rows[3];
  DevBuf X[3];      // stage inputs: nparts planes of rows x ld BF16
  DevBuf Tp[3];     // per-axis matrix parts: nparts planes of P*n_out x ld
  DevBuf sc[3], sc64[3];
  int towner[3];
  CUtensorMap mapA[3][3], mapB[3][3];
  DevBuf err;
  // FP16 mode: per-t-point largest row L1 norm of each owner axis's matrix,
  // the weights in FP64, and the per-apply scales (f16_scales_kernel)
  DevBuf l1[3], psc[3], w64, maxbits, gin, g01, wcoef;
};

long long round_up(long long v, long long m) { return (v + m - 1) / m * m; }

__nv_bfloat16 *plane(DevBuf &b, int part, long long plane_elems) {
  return b.as<__nv_bfloat16>() + (size_t)part * plane_elems;
}

// One stage launch.  nrb > 0 selects the two-dimensional M tiling of the
// intermediate stages (see StageArgs).
template <int NSX, int NS, bool FINAL, bool F16>
int launch_stage(MixedState &st, int stage, int M, int N, int K, int p, int nrb, int ng,
                 const StageArgs &base, cudaStream_t s) {
  using C = StageCfg<NSX, NS, F16>;
  auto kern = stage_bf16_kernel<NSX, NS, FINAL, F16>;
  static bool attr_set = false;
  if (!attr_set) {
    DAGE_CUDA_TRY(
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, C::kSmem));
    attr_set = true;
  }
  StageArgs a = base;
  a.M = M;
  a.N = N;
  a.K = K;
  a.nrb = nrb;
  a.ng = ng;
  a.gM = M;
  a.n_ntiles = ceil_div(N, BN);
  const long long nmt = nrb ? (long long)(M / a.d0) * nrb : ceil_div(M, BM);
  a.ntiles = (int)(nmt * a.n_ntiles);
  a.nkb = ceil_div(K, BK);
  a.last_k16 = ceil_div(K - (a.nkb - 1) * BK, 16);
  a.brow0 = p * N;
  const int grid = std::min(a.ntiles, sm_count());
  const CUtensorMap *mA = st.mapA[stage];
  const CUtensorMap *mB = st.mapB[st.towner[stage]];
  kern<<<grid, kThreads, C::kSmem, s>>>(mA[0], mA[1], mA[NSX > 2 ? 2 : 1], mB[0], mB[1],
                                        mB[NSX > 2 ? 2 : 1], a);
  DAGE_CUDA_TRY(cudaGetLastError());
  return 0;
}

template <int NSX, int NS, bool F16>
int run_stages(dage_op3d *op, MixedState &st, const double *d_rho, double *d_V, cudaStream_t s) {
  const int nix = op->nin[0], niy = op->nin[1], niz = op->nin[2];
  const int nox = op->nout[0], noy = op->nout[1], noz = op->nout[2];
  const long long pe[3] = {st.rows[0] * st.ld[0], st.rows[1] * st.ld[1], st.rows[2] * st.ld[2]};
  // input split (FP16: after the bound-based scales of this input)
  {
    const int t = op->tmark_begin(1);
    if (F16) {
      const long long n = (long long)nix * st.rows[0];
      const int blocks = (int)std::min<long long>((n + 255) / 256, sm_count() * 8LL);
      DAGE_CUDA_TRY(cudaMemsetAsync(st.maxbits.ptr, 0, sizeof(unsigned), s));
      absmax_kernel<<<blocks, 256, 0, s>>>(d_rho, n, st.maxbits.as<unsigned>());
      f16_scales_kernel<<<1, 128, 0, s>>>(
          st.maxbits.as<unsigned>(), st.l1[st.towner[0]].as<double>(),
          st.l1[st.towner[1]].as<double>(), st.psc[st.towner[0]].as<double>(),
          st.psc[st.towner[1]].as<double>(), st.psc[st.towner[2]].as<double>(),
          st.w64.as<double>(), op->P, st.gin.as<float>(), st.g01.as<float>(),
          st.wcoef.as<float>());
      const long long ne = st.rows[0] * st.ld[0];
      split_input_f16_kernel<<<(int)std::min<long long>((ne + 255) / 256, sm_count() * 16LL), 256, 0,
                               s>>>(d_rho, nix, st.rows[0], st.ld[0], st.gin.as<float>(),
                                    reinterpret_cast<__half *>(plane(st.X[0], 0, pe[0])),
                                    reinterpret_cast<__half *>(plane(st.X[0], 1, pe[0])));
    } else {
      const long long nwarps = st.rows[0] * ((st.ld[0] + kGroup - 1) / kGroup);
      const int blocks = (int)std::min<long long>((nwarps + 7) / 8, sm_count() * 16LL);
      split_input_kernel<NSX><<<blocks, 256, 0, s>>>(
          d_rho, nix, st.rows[0], st.ld[0], plane(st.X[0], 0, pe[0]), plane(st.X[0], 1, pe[0]),
          plane(st.X[0], NSX > 2 ? 2 : 1, pe[0]));
    }
    DAGE_CUDA_TRY(cudaGetLastError());
    op->tmark_end(t);
  }
  StageArgs base{};
  base.err = st.err.as<int>();
  base.wait_limit = g_wait_limit;
  base.drain_limit = 4000000000LL;  // ~2 s: copies and MMAs in flight always finish
  const int ni[3] = {nix, niy, niz}, no[3] = {nox, noy, noz};
  const long long M[3] = {(long long)niy * niz, (long long)niz * nox, (long long)nox * noy};
  const int d0[3] = {niy, niz, 0}, d1[3] = {niz, nox, 0};
  auto common = [&](StageArgs &a, int stage, int p) {
    const int ow = st.towner[stage];
    a.scale = st.sc[ow].as<float>() + (size_t)p * no[stage];
    a.k_range = op->band[ow].as<int2>() + (size_t)p * ceil_div(no[stage], BN);
  };
  // last-stage input: slot p % G of X[2], parts stored [part][slot][rows][ld]
  auto slot_plane = [&](int part, int slot) {
    return plane(st.X[2], part, pe[2] * st.Gmax) + (size_t)slot * pe[2];
  };
  int p0 = 0;  // first t-point of the open group
  for (int p = 0; p < op->P; ++p) {
    for (int stage = 0; stage < 2; ++stage) {
      StageArgs a = base;
      common(a, stage, p);
      const int slot = p % st.G;
      a.out0 = stage == 0 ? plane(st.X[1], 0, pe[1]) : slot_plane(0, slot);
      a.out1 = stage == 0 ? plane(st.X[1], 1, pe[1]) : slot_plane(1, slot);
      a.out2 = stage == 0 ? plane(st.X[1], NSX > 2 ? 2 : 1, pe[1]) : slot_plane(NSX > 2 ? 2 : 1, slot);
      a.d0 = d0[stage];
      a.d1 = d1[stage];
      a.ldn = st.ld[stage + 1];
      if (F16) a.gscale = st.g01.as<float>() + (size_t)stage * op->P + p;
      const int t = op->tmark_begin(0);
      DAGE_TRY((launch_stage<NSX, NS, false, F16>(st, stage, (int)M[stage], no[stage], ni[stage], p,
                                                  ceil_div(d0[stage], BM), 1, a, s)));
      op->tmark_end(t);
    }
    if (p - p0 + 1 == st.G || p == op->P - 1) {
      StageArgs a = base;
      common(a, 2, p0);
      const int ng = p - p0 + 1;
      a.wcoef = (F16 ? st.wcoef.as<float>() : st.wdev.as<float>()) + p0;
      a.V = d_V;
      a.accumulate = p0 > 0;
      const int t = op->tmark_begin(0);
      DAGE_TRY((launch_stage<NSX, NS, true, F16>(st, 2, (int)M[2], no[2], ni[2], p0, 0, ng, a, s)));
      op->tmark_end(t);
      p0 = p + 1;
    }
  }
  return 0;
}

}  // namespace

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

int mixed_setup(dage_op3d *op) {
  auto *st = new MixedState();
  op->mixed = st;
  st->f16 = op->precision == DAGE_MIXED_FP16X3;
  st->nparts = op->precision == DAGE_MIXED_BF16X6 ? 3 : 2;
  const int nix = op->nin[0], niy = op->nin[1], niz = op->nin[2];
  const int nox = op->nout[0], noy = op->nout[1];
  const int ni[3] = {nix, niy, niz};
  st->rows[0] = (long long)niy * niz;
  st->rows[1] = (long long)niz * nox;
  st->rows[2] = (long long)nox * noy;
  st->G = st->Gmax = std::min(op->P, kMaxGroup);
  st->ns = st->nparts == 3 ? 4 : 6;
  for (int s = 0; s < 3; ++s) {
    st->ld[s] = round_up(ni[s], 8);
    const int slots = s == 2 ? st->Gmax : 1;
    const long long pe = st->rows[s] * st->ld[s] * slots;
    DAGE_TRY(st->X[s].alloc(sizeof(__nv_bfloat16) * pe * st->nparts));
    DAGE_CUDA_TRY(cudaMemsetAsync(st->X[s].ptr, 0, st->X[s].bytes, op->stream));
    for (int i = 0; i < st->nparts; ++i)
      DAGE_TRY(make_map(&st->mapA[s][i], plane(st->X[s], i, pe), ni[s], st->rows[s] * slots,
                        st->ld[s], BK, BM));
  }
  DAGE_TRY(st->err.alloc(sizeof(int)));
  DAGE_CUDA_TRY(cudaMemsetAsync(st->err.ptr, 0, sizeof(int), op->stream));
  for (int ax = 0; ax < 3; ++ax) {
    st->towner[ax] = op->Towner[ax];
    if (op->Towner[ax] != ax) continue;
    const int K = op->nin[ax], N = op->nout[ax];
    const long long ld = round_up(K, 8);
    const long long nrows = (long long)op->P * N;
    const long long pe = nrows * ld;
    DAGE_TRY(st->Tp[ax].alloc(sizeof(__nv_bfloat16) * pe * st->nparts));
    DAGE_TRY(st->sc[ax].alloc(sizeof(float) * nrows));
    DAGE_TRY(st->sc64[ax].alloc(sizeof(double) * nrows));
    __nv_bfloat16 *o0 = plane(st->Tp[ax], 0, pe), *o1 = plane(st->Tp[ax], 1, pe),
                  *o2 = plane(st->Tp[ax], st->nparts > 2 ? 2 : 1, pe);
    if (st->f16) {
      DAGE_TRY(st->l1[ax].alloc(sizeof(double) * op->P));
      DAGE_TRY(st->psc[ax].alloc(sizeof(double) * op->P));
      row_l1max_kernel<<<op->P, 256, 0, op->stream>>>(op->T(ax), N, K, st->l1[ax].as<double>(),
                                                      st->psc[ax].as<double>());
      split_matrix_kernel<2, true><<<(unsigned)nrows, 256, 0, op->stream>>>(
          op->T(ax), K, ld, st->sc[ax].as<float>(), st->sc64[ax].as<double>(), o0, o1, o2,
          st->psc[ax].as<double>(), N);
    } else if (st->nparts == 2)
      split_matrix_kernel<2><<<(unsigned)nrows, 256, 0, op->stream>>>(
          op->T(ax), K, ld, st->sc[ax].as<float>(), st->sc64[ax].as<double>(), o0, o1, o2);
    else
      split_matrix_kernel<3><<<(unsigned)nrows, 256, 0, op->stream>>>(
          op->T(ax), K, ld, st->sc[ax].as<float>(), st->sc64[ax].as<double>(), o0, o1, o2);
    DAGE_CUDA_TRY(cudaGetLastError());
    for (int i = 0; i < st->nparts; ++i)
      DAGE_TRY(make_map(&st->mapB[ax][i], plane(st->Tp[ax], i, pe), K, nrows, ld, BK, BN));
  }
  if (st->f16) {
    DAGE_TRY(st->maxbits.alloc(sizeof(unsigned)));
    DAGE_TRY(st->gin.alloc(sizeof(float)));
    DAGE_TRY(st->g01.alloc(sizeof(float) * 2 * op->P));
    DAGE_TRY(st->wcoef.alloc(sizeof(float) * op->P));
  }
  return mixed_set_weights(op);
}

int mixed_set_weights(dage_op3d *op) {
  auto *st = static_cast<MixedState *>(op->mixed);
  if (!st) return 0;
  std::vector<float> w(op->w.begin(), op->w.end());
  DAGE_TRY(st->wdev.alloc(sizeof(float) * w.size()));
  DAGE_CUDA_TRY(cudaMemcpyAsync(st->wdev.ptr, w.data(), sizeof(float) * w.size(),
                                cudaMemcpyHostToDevice, op->stream));
  if (st->f16) {
    DAGE_TRY(st->w64.alloc(sizeof(double) * op->w.size()));
    DAGE_CUDA_TRY(cudaMemcpyAsync(st->w64.ptr, op->w.data(), sizeof(double) * op->w.size(),
                                  cudaMemcpyHostToDevice, op->stream));
  }
  return cudaStreamSynchronize(op->stream) == cudaSuccess ? 0 : fail(DAGE_E_CUDA, "weights upload");
}

int mixed_apply(dage_op3d *op, const double *d_rho, double *d_V, cudaStream_t s) {
  DAGE_TRY(mixed_enqueue(op, d_rho, d_V, s));
  return mixed_check(op, s);
}

int mixed_enqueue(dage_op3d *op, const double *d_rho, double *d_V, cudaStream_t s) {
  auto *st = static_cast<MixedState *>(op->mixed);
  if (!st) return fail(DAGE_E_INVALID, "mixed state missing");
  int rc;
  if (st->f16)
    rc = st->ns == 4 ? run_stages<2, 4, true>(op, *st, d_rho, d_V, s)
                     : run_stages<2, 6, true>(op, *st, d_rho, d_V, s);
  else if (st->nparts == 2)
    rc = st->ns == 4 ? run_stages<2, 4, false>(op, *st, d_rho, d_V, s)
                     : run_stages<2, 6, false>(op, *st, d_rho, d_V, s);
  else
    rc = run_stages<3, 4, false>(op, *st, d_rho, d_V, s);
  return rc;
}

int mixed_check(dage_op3d *op, cudaStream_t s) {
  auto *st = static_cast<MixedState *>(op->mixed);
  if (!st) return fail(DAGE_E_INVALID, "mixed state missing");
  int herr = 0;
  DAGE_CUDA_TRY(cudaMemcpyAsync(&herr, st->err.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
  DAGE_CUDA_TRY(cudaStreamSynchronize(s));
  if (herr) {
    cudaMemsetAsync(st->err.ptr, 0, sizeof(int), s);
    return fail(DAGE_E_TIMEOUT, "tensor-core stage kernel timed out waiting on an mbarrier");
  }
  return 0;
}

namespace {
__global__ void fill_kernel(double *x, size_t n, double v) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    x[i] = v;
}
}  // namespace

// Autotuner of the tensor-core path: ring depth of the stage kernel (4 or 6
// TMA/MMA stages; bf16x6's three-part stages fit 4 only), each candidate
// timed over one apply of a scratch cube after one untimed apply; keyed on
// (device, precision, points per axis, t-points) in the tune cache.  The
// ring depth changes no arithmetic.  The t-points summed per pass of the
// last stage stay at min(P, 8) unless a cache entry names another group:
// the group sets the order of the last stage's FP32 sums, and a choice by
// timing could differ from process to process.
int mixed_tune(dage_op3d *op) {
  auto *st = static_cast<MixedState *>(op->mixed);
  if (!st) return fail(DAGE_E_INVALID, "mixed state missing");
  std::string key = tune_device_key() + "/op3d_mixed" + std::to_string(op->precision) + "/";
  for (int d = 0; d < 3; ++d) key += std::to_string(op->nin[d]) + "x" + std::to_string(op->nout[d]) + ",";
  key += "P" + std::to_string(op->P);
  std::vector<int> v;
  if (tune_lookup(key, v) && v.size() == 2 && (v[0] == 4 || v[0] == 6) && v[1] >= 1 &&
      v[1] <= st->Gmax && (st->nparts == 2 || v[0] == 4)) {
    st->ns = v[0];
    st->G = v[1];
    return 0;
  }
  const size_t nin = (size_t)op->nin[0] * op->nin[1] * op->nin[2];
  const size_t nout = (size_t)op->nout[0] * op->nout[1] * op->nout[2];
  TmpBuf rho, V;
  DAGE_TRY(rho.alloc(sizeof(double) * nin));
  DAGE_TRY(V.alloc(sizeof(double) * nout));
  cudaStream_t s = op->stream;
  fill_kernel<<<(int)std::min<size_t>((nin + 255) / 256, (size_t)sm_count() * 16), 256, 0, s>>>(
      rho.as<double>(), nin, 1.0);
  DAGE_CUDA_TRY(cudaGetLastError());
  std::vector<int> nss = st->nparts == 2 ? std::vector<int>{6, 4} : std::vector<int>{4};
  const std::vector<int> gs = {st->Gmax};
  int best_ns = st->ns, best_g = st->G;
  float best = 0.0f;
  for (int ns : nss)
    for (int g : gs) {
      st->ns = ns;
      st->G = g;
      DAGE_TRY(mixed_apply(op, rho.as<double>(), V.as<double>(), s));
      DAGE_CUDA_TRY(cudaEventRecord(op->ev0, s));
      DAGE_TRY(mixed_apply(op, rho.as<double>(), V.as<double>(), s));
      DAGE_CUDA_TRY(cudaEventRecord(op->ev1, s));
      DAGE_CUDA_TRY(cudaEventSynchronize(op->ev1));
      float ms = 0.0f;
      DAGE_CUDA_TRY(cudaEventElapsedTime(&ms, op->ev0, op->ev1));
      if (best == 0.0f || ms < best) {
        best = ms;
        best_ns = ns;
        best_g = g;
      }
    }
  st->ns = best_ns;
  st->G = best_g;
  tune_store(key, {best_ns, best_g});
  return 0;
}

int mixed_schedule(const dage_op3d *op, int *ring_stages, int *group) {
  const auto *st = static_cast<const MixedState *>(op->mixed);
  if (!st) return fail(DAGE_E_INVALID, "not a split-precision operator");
  *ring_stages = st->ns;
  *group = st->G;
  return 0;
}

void mixed_destroy(dage_op3d *op) {
  auto *st = static_cast<MixedState *>(op->mixed);
  if (!st) return;
  for (int i = 0; i < 3; ++i) {
    st->X[i].release();
    st->Tp[i].release();
    st->sc[i].release();
    st->sc64[i].release();
    st->l1[i].release();
    st->psc[i].release();
  }
  st->w64.release();
  st->maxbits.release();
  st->gin.release();
  st->g01.release();
  st->wcoef.release();
  st->err.release();
  st->wdev.release();
  delete st;
  op->mixed = nullptr;
}

}  // namespace dage
