// near_mixed.cu -- GBFMM near field in the fp16x3 split precision on the
// 5th-generation tensor cores (tcgen05.mma kind::f16, FP16 parts, FP32
// accumulation in TMEM).
//
// Per t-point the near field of every box is three stages (the FP64 form is
// `near_descs` in gbfmm.cu):
//   stage x: rho(x, y, z) on the near region -> U(y, z; x own)   K = x near
//   stage y: U                                -> W(z, x; y own)   K = y near
//   stage z: W                                -> V(x, y; z own)   K = z near
// Each stage is ONE grouped launch over all boxes of all densities of a set
// ("jobs").  A job's output rows are two-dimensional, (a, b) with a the
// next stage's contraction index, and a tile is 32 values of a times 4 of b
// (128 rows, the TMEM lanes), so every stage's A operand is a 3-D TMA box
// {64 K, 32 a, 4 b} of a 3-D tensor:
//   stage x: the FP16 split of the whole density, (x, y, z) -- the box's
//            near region is a window of it, so the input is split once per
//            apply and, at 241^3, stays in L2 (56 MB) for all 64 boxes;
//   stage y: U as [x slice][z (padded to 32)][y (padded to 8)];
//   stage z: W as [slot][y slice][x (padded to 32)][z (padded to 8)].
// The x window of a box starts at a point index that need not be a multiple
// of 8 (TMA wants 16-byte aligned inner coordinates): the box's x matrices
// are stored with koff = q0 mod 8 leading zero columns and the window starts
// at q0 - koff.  Rows and columns outside a job (tile edges) read zeros or
// finite neighbouring data that meets zero matrix columns, and their
// results are not stored.  K blocks are 64 wide (128-byte rows, SWIZZLE_128B:
// half the TMA rows of 64-byte rows per byte moved); the main product still
// starts a fresh TMEM partial every 32 K and the partials are added in FP32
// registers after the +1 ulp toward-zero bias correction, as in the cube
// operator's fp16x3 stages (op3d_mixed.cu).  Scales: the cube operator's
// bound-based powers of two, with L1 norms and entry maxima taken over all
// box positions of the axis, and one max |rho| per density.
//
// Kernel structure (one persistent CTA per SM, 18 warps): warp 0 TMA
// producer, warp 1 TMEM allocator + single-thread MMA issuer, warps 2-17
// epilogue (four per TMEM lane quarter, TNW / 4 columns each).  Every
// mbarrier wait is bounded; on timeout the CTA sets the error word, drains
// its copies and MMAs in flight, frees TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "near_mixed.cuh"
#include "tc_common.cuh"

namespace dage {

extern long long g_wait_limit;

namespace {

constexpr int BKN = 64;            // K extent of one shared-memory stage (128-byte rows)
constexpr int kNThreads = 576;     // 18 warps
constexpr int kNEpiThreads = 512;  // warps 2-17
constexpr int kNMaxGroup = 4;      // t-points summed per pass of the last stage (W slots)
constexpr int kRowsA = 32, kRowsB = 4;  // tile rows: 32 along a x 4 along b
static_assert(kRowsA * kRowsB == BM, "tile rows");

struct NearJob {
  int ax, ay, az;      // A tensor coordinates of the job's row (0, 0) and K column 0
  int na, nb, N;       // valid rows along a and b; output columns
  int brow;            // B (matrix) row of t-point 0, column 0
  int koff;            // the job's K columns start at koff in its matrix rows
  int kr_ps;           // K bands per t-point (128-column tiles)
  int inst;            // density of the set (scales)
  int ta;              // 32-row blocks along a
  int pad_;
  long long ooff;      // intermediate stages: first output slice
  const int2 *band;    // K band [first, last] per (t-point, 128-column tile)
  double *V;           // last stage: V at the box's first owned point
  long long vs_b, vs_n;
};

struct NearArgs {
  const NearJob *jobs;
  const int4 *tiles;   // per tile: job, n-tile, a-block, b-block
  int ntiles;
  int p;               // t-point (the group's first in the last stage)
  int ng;              // last stage: t-points of the group (member gi reads slot gi)
  int slot_rows;       // last stage: A outer rows per slot
  const float *gscale; // intermediate: output factor of (inst, p) at gscale[inst * gstride + p]
  int gstride;
  const float *wcoef;  // last stage: w_p times the scales, at wcoef[inst * wstride + p]
  int wstride;
  __half *out0, *out1; // intermediate output planes
  long long oslice0;   // first output slice of this launch (the W slot)
  int opad;            // rows per output slice
  long long ldn;       // output row length
  int accumulate;
  int *err;
  long long wait_limit, drain_limit;
};

template <int TNW, int NS>
struct NearCfg {
  static constexpr int kABytes = BM * BKN * 2;   // one FP16 part of the A tile
  static constexpr int kBBytes = TNW * BKN * 2;  // one FP16 part of the B tile
  static constexpr int kStageBytes = 2 * kABytes + 2 * kBBytes;
  static constexpr int kNP = 3;                  // partial buffers
  static constexpr int kTmemCols = 4 * TNW;      // 3 partials + correction
  static constexpr int kSmem = NS * kStageBytes + 1024 + 256;
  static_assert(kSmem <= 227 * 1024, "shared memory");
};

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, uint32_t bar,
                                            int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y), "r"(z)
      : "memory");
}

// K-major tile written by TMA with the 128-byte swizzle: rows of 64 FP16,
// 8-row atoms at SBO = 1024 bytes.
__device__ __forceinline__ uint64_t sdesc128(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)1 << 16;            // LBO (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;  // SBO
  d |= (uint64_t)1 << 46;            // descriptor version
  d |= (uint64_t)2 << 61;            // SWIZZLE_128B
  return d;
}

// The MMAs of one 32-run of K: main product (part 0 x part 0) into the fresh
// partial P (committed to pfull), corrections (1 x 0) and (0 x 1) into Cc.
template <int TNW, bool FIRST>
__device__ __forceinline__ void near_mma_run(uint32_t P, uint32_t Cc, uint64_t d0, uint32_t idesc,
                                             uint32_t pfull_bar) {
  constexpr int kA = BM * BKN * 2, kB = TNW * BKN * 2;
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const uint64_t a0 = d0 + ((k * 32) >> 4), a1 = d0 + ((kA + k * 32) >> 4);
    const uint64_t b0 = d0 + ((2 * kA + k * 32) >> 4), b1 = d0 + ((2 * kA + kB + k * 32) >> 4);
    umma_bf16_c(P, a0, b0, idesc, k != 0);
    if (k == 1) umma_commit(pfull_bar);
    umma_bf16_c(Cc, a1, b0, idesc, !(FIRST && k == 0));
    umma_bf16_c(Cc, a0, b1, idesc, true);
  }
}

// K blocks [first, last] of job j, n-tile nt, t-point p + gi
template <int TNW>
__device__ __forceinline__ int2 near_kblocks(const NearArgs &a, const NearJob &j, int nt, int gi) {
  const int2 r = j.band[(size_t)(a.p + gi) * j.kr_ps + (nt * TNW) / 128];
  return make_int2((r.x + j.koff) / BKN, (r.y + j.koff) / BKN);
}

template <bool FINAL, int TNW, int NS>
__global__ void __maxnreg__(96)
    near_f16_kernel(const __grid_constant__ CUtensorMap mapA0,
                    const __grid_constant__ CUtensorMap mapA1,
                    const __grid_constant__ CUtensorMap mapB0,
                    const __grid_constant__ CUtensorMap mapB1, const NearArgs a) {
  using C = NearCfg<TNW, NS>;
  if (*reinterpret_cast<volatile int *>(a.err)) return;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t *tiles = smem;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + NS * C::kStageBytes);
  // bars: full[NS], empty[NS], pfull[3], pempty[3], cfull, cempty, drain
  uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(bars + 2 * NS + 9);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_holder + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto full = [&](int i) { return smem_u32(bars + i); };
  auto empty = [&](int i) { return smem_u32(bars + NS + i); };
  auto pfull = [&](int i) { return smem_u32(bars + 2 * NS + i); };
  auto pempty = [&](int i) { return smem_u32(bars + 2 * NS + 3 + i); };
  const uint32_t cfull = smem_u32(bars + 2 * NS + 6), cempty = smem_u32(bars + 2 * NS + 7);
  const uint32_t drain = smem_u32(bars + 2 * NS + 8);

  if (threadIdx.x == 0) {
    for (int i = 0; i < NS; ++i) {
      mbar_init(full(i), 1);
      mbar_init(empty(i), 1);
    }
    for (int i = 0; i < C::kNP; ++i) {
      mbar_init(pfull(i), 1);
      mbar_init(pempty(i), kNEpiThreads / 32);
    }
    mbar_init(cfull, 1);
    mbar_init(cempty, kNEpiThreads / 32);
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(smem_u32(tmem_holder), C::kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_holder;
  const uint32_t tmem_corr = tmem_base + C::kNP * TNW;
  auto on_timeout = [&]() {
    *abort_flag = 1;
    atomicCAS(a.err, 0, 1);
  };
  const int nunits = a.ntiles * a.ng;
  auto next_unit = [&](int u) { return u + ((u % a.ng == a.ng - 1) ? (gridDim.x - 1) * a.ng + 1 : 1); };

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      int issued[NS];
      uint32_t issued_ph[NS];
      for (int i = 0; i < NS; ++i) issued[i] = 0, issued_ph[i] = 0;
      for (int u = blockIdx.x * a.ng; u < nunits && !*abort_flag; u = next_unit(u)) {
        const int gi = u % a.ng;
        const int4 t = a.tiles[u / a.ng];
        const NearJob &j = a.jobs[t.x];
        const int2 r = near_kblocks<TNW>(a, j, t.y, gi);
        const int ay = j.ay + kRowsA * t.z, az = j.az + kRowsB * t.w + gi * a.slot_rows;
        const int brow = j.brow + (a.p + gi) * j.N + t.y * TNW;
        for (int kb = r.x; kb <= r.y; ++kb) {
          if (!mbar_wait(empty(s), ph ^ 1, a.wait_limit)) {
            on_timeout();
            break;
          }
          uint8_t *st = tiles + s * C::kStageBytes;
          mbar_expect_tx(full(s), C::kStageBytes);
          tma_load_3d(smem_u32(st), &mapA0, full(s), j.ax + kb * BKN, ay, az);
          tma_load_3d(smem_u32(st + C::kABytes), &mapA1, full(s), j.ax + kb * BKN, ay, az);
          tma_load_2d(smem_u32(st + 2 * C::kABytes), &mapB0, full(s), kb * BKN, brow);
          tma_load_2d(smem_u32(st + 2 * C::kABytes + C::kBBytes), &mapB1, full(s), kb * BKN, brow);
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
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      int b = 0;         // partial buffer of the current 32-run
      uint32_t pph = 0;  // phase of the partial buffers' current round
      int t = 0;
      bool ok = true;
      const uint64_t dbase = sdesc128(smem_u32(tiles));
      for (int u = blockIdx.x * a.ng; u < nunits && ok && !*abort_flag; u = next_unit(u), ++t) {
        const int gi = u % a.ng;
        const int4 tl = a.tiles[u / a.ng];
        const NearJob &j = a.jobs[tl.x];
        const int2 rc = near_kblocks<TNW>(a, j, tl.y, gi);
        int nt = j.N - tl.y * TNW;
        if (nt > TNW) nt = TNW;
        nt = (nt + 15) & ~15;
        const uint32_t idesc = idesc_f16kind<true>(BM, nt);
        for (int kb = rc.x; kb <= rc.y; ++kb) {
          const bool first = kb == rc.x;
          if (!mbar_wait(full(s), ph, a.wait_limit) ||
              (first && !mbar_wait(cempty, (t & 1) ^ 1, a.wait_limit))) {
            on_timeout();
            ok = false;
            break;
          }
          tc_fence_after();
          const uint64_t d0 = dbase + (uint64_t)((s * C::kStageBytes) >> 4);
#pragma unroll
          for (int rr = 0; rr < BKN / kGroup; ++rr) {
            if (!mbar_wait(pempty(b), pph ^ 1, a.wait_limit)) {
              on_timeout();
              ok = false;
              break;
            }
            tc_fence_after();
            const uint64_t dr = d0 + (uint64_t)((rr * kGroup * 2) >> 4);
            const uint32_t P = tmem_base + b * TNW;
            if (first && rr == 0)
              near_mma_run<TNW, true>(P, tmem_corr, dr, idesc, pfull(b));
            else
              near_mma_run<TNW, false>(P, tmem_corr, dr, idesc, pfull(b));
            if (++b == C::kNP) b = 0, pph ^= 1;
          }
          if (!ok) break;
          umma_commit(empty(s));
          if (++s == NS) s = 0, ph ^= 1;
        }
        if (ok) umma_commit(cfull);
      }
      umma_commit(drain);
      mbar_wait(drain, 0, a.drain_limit);
    }
  } else {
    // ------------------------------------------------------------ epilogue
    // warp w reads TMEM lanes 32 (w % 4) .. +31 (its lane quarter = the
    // tile's b row w % 4, a = lane) and the CW columns (w - 2) / 4.
    constexpr int CW = TNW / 4;
    const int q = warp & 3;
    const uint32_t lane_off = (uint32_t)(32 * q) << 16;
    const uint32_t col0 = ((warp - 2) >> 2) * CW;
    int g = 0, t = 0;
    for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
      const int4 tl = a.tiles[tile];
      const NearJob &j = a.jobs[tl.x];
      float2 acc[CW / 2];
      float2 accg[CW / 2];
#pragma unroll
      for (int k = 0; k < CW / 2; ++k) accg[k] = make_float2(0.0f, 0.0f);
      bool ok = true;
      for (int gi = 0; gi < a.ng && ok; ++gi, ++t) {
        const float fw = FINAL ? a.wcoef[(size_t)j.inst * a.wstride + a.p + gi] : 0.0f;
#pragma unroll
        for (int k = 0; k < CW / 2; ++k) acc[k] = make_float2(0.0f, 0.0f);
        const int2 rc = near_kblocks<TNW>(a, j, tl.y, gi);
        const int nparts = (rc.y - rc.x + 1) * (BKN / kGroup);
        for (int pi = 0; pi < nparts; ++pi, ++g) {
          const int b = g % C::kNP;
          const bool got =
              __all_sync(0xffffffffu, mbar_wait(pfull(b), (g / C::kNP) & 1, a.wait_limit));
          if (!got) {
            on_timeout();
            ok = false;
            break;
          }
          tc_fence_after();
#pragma unroll
          for (int hh = 0; hh < CW / 16; ++hh) {
            uint32_t r[16];
            tmem_ld16(tmem_base + lane_off + b * TNW + col0 + hh * 16, r);
#pragma unroll
            for (int k = 0; k < 8; ++k) {
              const float2 pv = make_float2(unbias_rz(__uint_as_float(r[2 * k])),
                                            unbias_rz(__uint_as_float(r[2 * k + 1])));
              acc[hh * 8 + k] = __fadd2_rn(acc[hh * 8 + k], pv);
            }
          }
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(pempty(b));
        }
        if (!ok) break;
        const bool got = __all_sync(0xffffffffu, mbar_wait(cfull, t & 1, a.wait_limit));
        if (!got) {
          on_timeout();
          ok = false;
          break;
        }
        tc_fence_after();
#pragma unroll
        for (int hh = 0; hh < CW / 16; ++hh) {
          uint32_t r[16];
          tmem_ld16(tmem_corr + lane_off + col0 + hh * 16, r);
#pragma unroll
          for (int k = 0; k < 8; ++k)
            acc[hh * 8 + k] = __fadd2_rn(acc[hh * 8 + k], make_float2(__uint_as_float(r[2 * k]),
                                                                      __uint_as_float(r[2 * k + 1])));
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(cempty);
        if (FINAL) {
          const float2 f = make_float2(fw, fw);
#pragma unroll
          for (int k = 0; k < CW / 2; ++k) accg[k] = __ffma2_rn(f, acc[k], accg[k]);
        }
      }
      if (!ok) break;
      const int n0 = tl.y * TNW + col0;
      const int av = kRowsA * tl.z + lane, bv = kRowsB * tl.w + q;
      if (bv >= j.nb) continue;  // warp-uniform: this warp's b row lies outside the job
      if (FINAL) {
        // V(a, b, n) (+)= the group's sum; one FP64 add per element per group
        if (av < j.na) {
          double *dst = j.V + av + j.vs_b * bv;
#pragma unroll
          for (int k = 0; k < CW; ++k) {
            const int n = n0 + k;
            if (n < j.N) {
              const double add = (double)((k & 1) ? accg[k >> 1].y : accg[k >> 1].x);
              if (a.accumulate)
                atomicAdd(dst + j.vs_n * n, add);
              else
                __stcs(dst + j.vs_n * n, add);
            }
          }
        }
      } else {
        // next stage: element (a, b, n) at out[((oslice0 + ooff + n) opad + b) ldn + a];
        // lane pairs swap one value so each lane stores two consecutive a of
        // one column as one packed FP16 pair per part (the a = na slot of an
        // odd na is the zero padding of the next stage's rows).
        const float gs = a.gscale[(size_t)j.inst * a.gstride + a.p];
        const bool valid = av < j.na;
        const bool odd = lane & 1;
        const int apair = av & ~1;
        const long long rowbase = (long long)bv * a.ldn + apair;
#pragma unroll
        for (int k = 0; k < CW; k += 2) {
          const int n = n0 + k;
          if (n < j.N) {  // uniform across the warp
            const bool has1 = n + 1 < j.N;
            const float2 v = valid ? __fmul2_rn(acc[k >> 1], make_float2(gs, gs))
                                   : make_float2(0.0f, 0.0f);
            const float recv = __shfl_xor_sync(0xffffffffu, odd ? v.x : v.y, 1);
            const float mine = odd ? v.y : v.x;
            const float2 vv = odd ? make_float2(recv, mine) : make_float2(mine, recv);
            const size_t off =
                (size_t)(a.oslice0 + j.ooff + n + (odd ? 1 : 0)) * a.opad * a.ldn + rowbase;
            if (apair < j.na && (!odd || has1)) {
              __half2 hh2[2];
              split_pair_f16(vv, hh2);
              *reinterpret_cast<__half2 *>(a.out0 + off) = hh2[0];
              *reinterpret_cast<__half2 *>(a.out1 + off) = hh2[1];
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
// Preparation kernels
// ---------------------------------------------------------------------------
// Per (t-point p, position v): largest |entry| and largest row L1 norm of
// T_v[p] (own_v rows of nq_v).
__global__ void near_mstats_kernel(const double *const *T, const int *own, const int *nq, int P,
                                   double *stats) {
  const int p = blockIdx.x, v = blockIdx.y;
  const int N = own[v], K = nq[v];
  const double *Tp = T[v] + (size_t)p * N * K;
  double m = 0.0, mx = 0.0;
  for (int n = threadIdx.x >> 5; n < N; n += blockDim.x >> 5) {
    double sum = 0.0;
    for (int k = threadIdx.x & 31; k < K; k += 32) {
      const double x = fabs(Tp[(size_t)n * K + k]);
      sum += x;
      mx = fmax(mx, x);
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
    stats[2 * ((size_t)v * P + p)] = r;
    stats[2 * ((size_t)v * P + p) + 1] = rx;
  }
}

// Per t-point over the positions: l1[p] = largest row L1 norm, psc[p] = the
// power of two at or above the largest |entry| (1 when all are zero).
__global__ void near_mreduce_kernel(const double *stats, int P, int npos, double *l1,
                                    double *psc) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
    double r = 0.0, rx = 0.0;
    for (int v = 0; v < npos; ++v) {
      r = fmax(r, stats[2 * ((size_t)v * P + p)]);
      rx = fmax(rx, stats[2 * ((size_t)v * P + p) + 1]);
    }
    l1[p] = r;
    psc[p] = rx > 0.0 ? exp2(ceil(log2(rx))) : 1.0;
  }
}

// One block per matrix row (v, p, n): FP16 parts of 2^14 T / psc[p] at
// B[brow_v + p own_v + n][koff_v + k] (the rest of the row stays zero).
__global__ void near_split_matrix_kernel(const double *const *T, const int *own, const int *nq,
                                         const int *brow, const int *koff, int npos, int P,
                                         const double *psc, long long ldb, __half *o0,
                                         __half *o1) {
  const int row = blockIdx.x;
  int v = 0;
  while (v + 1 < npos && row >= brow[v + 1]) ++v;
  const int local = row - brow[v];
  const int N = own[v], K = nq[v];
  const int p = local / N, n = local % N;
  const double *src = T[v] + ((size_t)p * N + n) * K;
  const double tsc = ldexp(1.0, 14) / psc[p];
  for (int k = threadIdx.x; k < K; k += blockDim.x) {
    __half h[2];
    split_f16_f64(src[k] * tsc, h);
    const size_t off = (size_t)row * ldb + koff[v] + k;
    o0[off] = h[0];
    o1[off] = h[1];
  }
}

// max |rho_i| as float bits (ordered like the values); maxbits must start at 0
__global__ void near_absmax_kernel(const double *const *rho, long long n, unsigned *maxbits) {
  const double *x = rho[blockIdx.y];
  float m = 0.0f;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x)
    m = fmaxf(m, (float)fabs(x[e]));
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(maxbits + blockIdx.y, __float_as_uint(m));
}

// Power-of-two scales per density i (the cube operator's fp16x3 rule with
// the positions' norms): e_0 = floor(log2 M_i) - 14, e_1(p) = floor(log2(M_i
// L_x(p))) - 14, e_2(p) = floor(log2(M_i L_x L_y)) - 14; the x/y epilogues
// multiply by S(p) 2^(e_s - 14 - e_(s+1)) and the last one by w_p S_z(p)
// 2^(e_2 - 14).
__global__ void near_scales_kernel(const unsigned *maxbits, const double *l1x, const double *l1y,
                                   const double *sx, const double *sy, const double *sz,
                                   const double *const *w, int P, float *gin, float *g01,
                                   float *wcoef) {
  const int i = blockIdx.x;
  const double M = (double)__uint_as_float(maxbits[i]);
  auto ex = [](double b) { return b > 0.0 ? (int)floor(log2(b)) - 14 : 0; };
  const int e0 = ex(M);
  if (threadIdx.x == 0) gin[i] = (float)ldexp(1.0, -e0);
  for (int p = threadIdx.x; p < P; p += blockDim.x) {
    const int e1 = ex(M * l1x[p]), e2 = ex(M * l1x[p] * l1y[p]);
    g01[(size_t)i * 2 * P + p] = (float)(sx[p] * ldexp(1.0, e0 - 14 - e1));
    g01[(size_t)i * 2 * P + P + p] = (float)(sy[p] * ldexp(1.0, e1 - 14 - e2));
    wcoef[(size_t)i * P + p] = (float)(w[i][p] * sz[p] * ldexp(1.0, e2 - 14));
  }
}

// rho_i * gin_i -> two FP16 planes of rows of ld (x fastest, zeros from Nx)
__global__ void near_split_input_kernel(const double *const *rho, int Nx, long long rows,
                                        long long ld, const float *gin, __half *o0, __half *o1) {
  const int i = blockIdx.y;
  const double *x = rho[i];
  const double g = (double)gin[i];
  const size_t base = (size_t)i * rows * ld;
  // one warp per row, lanes over x (no per-element index division)
  const int lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows;
       r += nwarps) {
    for (int k = lane; k < ld; k += 32) {
      __half p[2];
      split_f16_f64(k < Nx ? x[r * Nx + k] * g : 0.0, p);
      o0[base + r * ld + k] = p[0];
      o1[base + r * ld + k] = p[1];
    }
  }
}

long long round_up(long long v, long long m) { return (v + m - 1) / m * m; }

// 2-D FP16 map: rows of ld elements, inner extent `inner`, box {64, box_rows}
int make_map_2d(CUtensorMap *m, const void *base, long long inner, long long rows, long long ld,
                int box_rows) {
  auto fn = encode_fn();
  if (!fn) return fail(DAGE_E_CUDA, "cuTensorMapEncodeTiled unavailable");
  if (reinterpret_cast<uintptr_t>(base) % 16 || (ld * 2) % 16)
    return fail(DAGE_E_INVALID, "tensor map base/stride not 16-byte aligned");
  cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(ld * 2)};
  cuuint32_t box[2] = {(cuuint32_t)BKN, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, const_cast<void *>(base), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(DAGE_E_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return 0;
}

// 3-D FP16 map: [d2][d1][inner] with row length ld and d1 rows per plane,
// box {64, 32, 4}
int make_map_3d(CUtensorMap *m, const void *base, long long inner, long long d1, long long d2,
                long long ld, long long plane_rows) {
  auto fn = encode_fn();
  if (!fn) return fail(DAGE_E_CUDA, "cuTensorMapEncodeTiled unavailable");
  if (reinterpret_cast<uintptr_t>(base) % 16 || (ld * 2) % 16)
    return fail(DAGE_E_INVALID, "tensor map base/stride not 16-byte aligned");
  cuuint64_t dims[3] = {(cuuint64_t)inner, (cuuint64_t)d1, (cuuint64_t)d2};
  cuuint64_t strides[2] = {(cuuint64_t)(ld * 2), (cuuint64_t)(ld * plane_rows * 2)};
  cuuint32_t box[3] = {(cuuint32_t)BKN, (cuuint32_t)kRowsA, (cuuint32_t)kRowsB};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3, const_cast<void *>(base), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(DAGE_E_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return 0;
}

template <bool FINAL, int TNW, int NS>
int set_smem_attr() {
  using C = NearCfg<TNW, NS>;
  DAGE_CUDA_TRY(cudaFuncSetAttribute(near_f16_kernel<FINAL, TNW, NS>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, C::kSmem));
  return 0;
}

template <bool FINAL, int TNW, int NS>
int launch_near(const CUtensorMap *mA, const CUtensorMap *mB, const NearArgs &a, cudaStream_t s) {
  using C = NearCfg<TNW, NS>;
  const int grid = std::min(a.ntiles, sm_count());
  near_f16_kernel<FINAL, TNW, NS><<<grid, kNThreads, C::kSmem, s>>>(mA[0], mA[1], mB[0], mB[1], a);
  DAGE_CUDA_TRY(cudaGetLastError());
  return 0;
}

}  // namespace

// ---------------------------------------------------------------------------
// Host objects
// ---------------------------------------------------------------------------
struct NearF16Plan {
  NearGeom g;
  long long ldb[3] = {0, 0, 0}, rows[3] = {0, 0, 0};
  std::vector<int> brow[3], koff[3];
  DevBuf Bp[3];          // two FP16 planes of rows x ldb
  DevBuf l1[3], psc[3];  // per t-point: largest row L1 norm, power-of-two entry scale
  int maxnq[3] = {0, 0, 0}, maxown[3] = {0, 0, 0};
};

struct NearF16Set {
  const NearF16Plan *plan = nullptr;
  int n = 0, tile_n = 64, G = 1, P = 0;
  std::vector<NearBox> boxes;
  long long ld[3] = {0, 0, 0};  // stage input row lengths (x: density rows; y: U; z: W)
  int zpad = 0, xpad = 0;
  long long xsl = 0, ysl = 0;   // x slices of U, y slices of W per slot
  long long xs_rows = 0;        // rows (y, z) of one density's split input
  DevBuf X, U, W;               // two FP16 planes each (when the set owns them)
  __half *xp = nullptr, *up = nullptr, *wp = nullptr;  // the planes in use
  DevBuf jobs[3], tiles[3];
  int ntiles[3] = {0, 0, 0};
  std::vector<int4> htiles[3];
  DevBuf maxbits, gin, g01, wcoef, rhoptr, wptr;
  CUtensorMap mapA[3][2], mapB[3][2];
  DevBuf err;
};

int near_f16_prepare() {
  DAGE_TRY((set_smem_attr<false, 64, 4>()));
  DAGE_TRY((set_smem_attr<true, 64, 4>()));
  DAGE_TRY((set_smem_attr<false, 128, 3>()));
  DAGE_TRY((set_smem_attr<true, 128, 3>()));
  return 0;
}

int near_f16_plan_create(NearF16Plan **out, const NearGeom &geom, cudaStream_t s) {
  auto *pl = new NearF16Plan();
  *out = pl;
  pl->g = geom;
  const int P = geom.P;
  for (int d = 0; d < 3; ++d) {
    const int npos = (int)geom.own[d].size();
    long long rows = 0, kmax = 0;
    for (int v = 0; v < npos; ++v) {
      pl->brow[d].push_back((int)rows);
      pl->koff[d].push_back(d == 0 ? geom.q0[d][v] % 8 : 0);
      rows += (long long)P * geom.own[d][v];
      kmax = std::max<long long>(kmax, pl->koff[d][v] + geom.nq[d][v]);
      pl->maxnq[d] = std::max(pl->maxnq[d], geom.nq[d][v]);
      pl->maxown[d] = std::max(pl->maxown[d], geom.own[d][v]);
    }
    if (rows >= (1LL << 31)) return fail(DAGE_E_INVALID, "near-field matrices too large");
    pl->rows[d] = rows;
    pl->ldb[d] = round_up(kmax, 8);
    const size_t pe = (size_t)rows * pl->ldb[d];
    DAGE_TRY(pl->Bp[d].alloc(sizeof(__half) * pe * 2));
    DAGE_CUDA_TRY(cudaMemsetAsync(pl->Bp[d].ptr, 0, pl->Bp[d].bytes, s));
    DAGE_TRY(pl->l1[d].alloc(sizeof(double) * P));
    DAGE_TRY(pl->psc[d].alloc(sizeof(double) * P));
    // per-position tables on the device
    std::vector<long long> tab;  // T pointers, then own, nq, brow, koff as int
    TmpBuf dT, dI, stats;
    DAGE_TRY(dT.alloc(sizeof(double *) * npos));
    DAGE_TRY(dI.alloc(sizeof(int) * 4 * npos));
    DAGE_TRY(stats.alloc(sizeof(double) * 2 * npos * P));
    std::vector<int> ints;
    for (int v = 0; v < npos; ++v) ints.push_back(geom.own[d][v]);
    for (int v = 0; v < npos; ++v) ints.push_back(geom.nq[d][v]);
    for (int v = 0; v < npos; ++v) ints.push_back(pl->brow[d][v]);
    for (int v = 0; v < npos; ++v) ints.push_back(pl->koff[d][v]);
    DAGE_CUDA_TRY(cudaMemcpyAsync(dT.ptr, geom.T[d].data(), sizeof(double *) * npos,
                                  cudaMemcpyHostToDevice, s));
    DAGE_CUDA_TRY(cudaMemcpyAsync(dI.ptr, ints.data(), sizeof(int) * 4 * npos,
                                  cudaMemcpyHostToDevice, s));
    const int *own = dI.as<int>(), *nq = own + npos, *brow = nq + npos, *koff = brow + npos;
    near_mstats_kernel<<<dim3(P, npos), 256, 0, s>>>(dT.as<const double *>(), own, nq, P,
                                                     stats.as<double>());
    DAGE_CUDA_TRY(cudaGetLastError());
    near_mreduce_kernel<<<1, 128, 0, s>>>(stats.as<double>(), P, npos, pl->l1[d].as<double>(),
                                          pl->psc[d].as<double>());
    DAGE_CUDA_TRY(cudaGetLastError());
    __half *o0 = pl->Bp[d].as<__half>(), *o1 = o0 + pe;
    near_split_matrix_kernel<<<(unsigned)rows, 128, 0, s>>>(dT.as<const double *>(), own, nq,
                                                           brow, koff, npos, P,
                                                           pl->psc[d].as<double>(), pl->ldb[d],
                                                           o0, o1);
    DAGE_CUDA_TRY(cudaGetLastError());
    // the tables are freed on return: finish the kernels that read them
    DAGE_CUDA_TRY(cudaStreamSynchronize(s));
  }
  return 0;
}

void near_f16_plan_destroy(NearF16Plan *pl) {
  if (!pl) return;
  for (int d = 0; d < 3; ++d) {
    pl->Bp[d].release();
    pl->l1[d].release();
    pl->psc[d].release();
  }
  delete pl;
}

namespace {

struct SetDims {
  long long ld[3], xs_rows, xsl, ysl;
  int zpad, xpad, G;
};

SetDims set_dims(const NearF16Plan *pl, const std::vector<NearBox> &boxes, int n) {
  SetDims d{};
  const NearGeom &g = pl->g;
  d.ld[0] = round_up(g.npts[0], 8);
  d.ld[1] = round_up(pl->maxnq[1], 8);
  d.ld[2] = round_up(pl->maxnq[2], 8);
  d.zpad = (int)round_up(pl->maxnq[2], kRowsA);
  d.xpad = (int)round_up(pl->maxown[0], kRowsA);
  d.xs_rows = (long long)g.npts[1] * g.npts[2];
  d.xsl = d.ysl = 0;
  for (const auto &b : boxes) {
    d.xsl += g.own[0][b.pos[0]];
    d.ysl += g.own[1][b.pos[1]];
  }
  d.xsl *= n;
  d.ysl *= n;
  d.G = std::min(g.P, kNMaxGroup);
  return d;
}

}  // namespace

void near_f16_set_sizes(const NearF16Plan *pl, const std::vector<NearBox> &boxes, int n,
                        size_t bytes[3]) {
  const SetDims d = set_dims(pl, boxes, n);
  bytes[0] = sizeof(__half) * 2 * ((size_t)n * d.xs_rows * d.ld[0]);
  bytes[1] = sizeof(__half) * 2 * ((size_t)d.xsl * d.zpad * d.ld[1]);
  bytes[2] = sizeof(__half) * 2 * ((size_t)d.G * d.ysl * d.xpad * d.ld[2]);
}

size_t near_f16_set_bytes(const NearF16Plan *pl, const std::vector<NearBox> &boxes, int n) {
  size_t b[3];
  near_f16_set_sizes(pl, boxes, n, b);
  return b[0] + b[1] + b[2];
}

int near_f16_set_create(NearF16Set **out, const NearF16Plan *pl, const std::vector<NearBox> &boxes,
                        int n, int tile_n, cudaStream_t s0, void *const ws[3]) {
  if (tile_n != 64 && tile_n != 128) return fail(DAGE_E_INVALID, "near-field tile width %d", tile_n);
  auto *st = new NearF16Set();
  *out = st;
  st->plan = pl;
  st->n = n;
  st->tile_n = tile_n;
  st->boxes = boxes;
  const NearGeom &g = pl->g;
  st->P = g.P;
  const SetDims d = set_dims(pl, boxes, n);
  for (int s = 0; s < 3; ++s) st->ld[s] = d.ld[s];
  st->zpad = d.zpad;
  st->xpad = d.xpad;
  st->xsl = d.xsl;
  st->ysl = d.ysl;
  st->xs_rows = d.xs_rows;
  st->G = d.G;
  if (d.xsl >= (1LL << 31) / d.zpad || (long long)d.G * d.ysl >= (1LL << 31) / d.xpad ||
      (long long)n * g.npts[2] >= (1LL << 31))
    return fail(DAGE_E_INVALID, "near-field set too large for 32-bit tensor coordinates");
  const size_t xe = (size_t)n * d.xs_rows * d.ld[0];
  const size_t ue = (size_t)d.xsl * d.zpad * d.ld[1];
  const size_t we = (size_t)d.G * d.ysl * d.xpad * d.ld[2];
  if (ws) {  // shared workspace (sets that run one after another)
    st->xp = static_cast<__half *>(ws[0]);
    st->up = static_cast<__half *>(ws[1]);
    st->wp = static_cast<__half *>(ws[2]);
  } else {
    DAGE_TRY(st->X.alloc(sizeof(__half) * 2 * xe));
    DAGE_TRY(st->U.alloc(sizeof(__half) * 2 * ue));
    DAGE_TRY(st->W.alloc(sizeof(__half) * 2 * we));
    // Elements the stages never write (tile edges, padding) are read only
    // against zero matrix columns or into rows that are not stored: they
    // must be finite, so the buffers start as zeros (every later write is
    // a finite FP16 value).
    DAGE_CUDA_TRY(cudaMemsetAsync(st->U.ptr, 0, st->U.bytes, s0));
    DAGE_CUDA_TRY(cudaMemsetAsync(st->W.ptr, 0, st->W.bytes, s0));
    st->xp = st->X.as<__half>();
    st->up = st->U.as<__half>();
    st->wp = st->W.as<__half>();
  }
  DAGE_TRY(st->maxbits.alloc(sizeof(unsigned) * n));
  DAGE_TRY(st->gin.alloc(sizeof(float) * n));
  DAGE_TRY(st->g01.alloc(sizeof(float) * 2 * g.P * n));
  DAGE_TRY(st->wcoef.alloc(sizeof(float) * g.P * n));
  DAGE_TRY(st->rhoptr.alloc(sizeof(double *) * n));
  DAGE_TRY(st->wptr.alloc(sizeof(double *) * n));
  DAGE_TRY(st->err.alloc(sizeof(int)));
  DAGE_CUDA_TRY(cudaMemsetAsync(st->err.ptr, 0, sizeof(int), s0));
  // A maps: x stage over the densities stacked along z; U; W with its slots
  __half *x0 = st->xp, *u0 = st->up, *w0 = st->wp;
  for (int part = 0; part < 2; ++part) {
    DAGE_TRY(make_map_3d(&st->mapA[0][part], x0 + part * xe, g.npts[0], g.npts[1],
                         (long long)n * g.npts[2], d.ld[0], g.npts[1]));
    DAGE_TRY(make_map_3d(&st->mapA[1][part], u0 + part * ue, d.ld[1], d.zpad, d.xsl, d.ld[1],
                         d.zpad));
    DAGE_TRY(make_map_3d(&st->mapA[2][part], w0 + part * we, d.ld[2], d.xpad,
                         (long long)d.G * d.ysl, d.ld[2], d.xpad));
    for (int s = 0; s < 3; ++s) {
      const size_t pe = (size_t)pl->rows[s] * pl->ldb[s];
      DAGE_TRY(make_map_2d(&st->mapB[s][part], pl->Bp[s].as<__half>() + part * pe, pl->ldb[s],
                           pl->rows[s], pl->ldb[s], tile_n));
    }
  }
  // tiles: per job (density-major, then box), n-tile fastest, then a, then b
  const int ntn = tile_n;
  for (int s = 0; s < 3; ++s) {
    int job = 0;
    for (int i = 0; i < n; ++i)
      for (const auto &b : boxes) {
        int na, nb, N;
        if (s == 0) {
          na = g.nq[1][b.pos[1]], nb = g.nq[2][b.pos[2]], N = g.own[0][b.pos[0]];
        } else if (s == 1) {
          na = g.nq[2][b.pos[2]], nb = g.own[0][b.pos[0]], N = g.own[1][b.pos[1]];
        } else {
          na = g.own[0][b.pos[0]], nb = g.own[1][b.pos[1]], N = g.own[2][b.pos[2]];
        }
        const int ta = ceil_div(na, kRowsA), tb = ceil_div(nb, kRowsB), tn = ceil_div(N, ntn);
        for (int y = 0; y < tb; ++y)
          for (int x = 0; x < ta; ++x)
            for (int c = 0; c < tn; ++c) st->htiles[s].push_back(make_int4(job, c, x, y));
        ++job;
      }
    st->ntiles[s] = (int)st->htiles[s].size();
    DAGE_TRY(st->tiles[s].alloc(sizeof(int4) * st->htiles[s].size()));
    DAGE_CUDA_TRY(cudaMemcpyAsync(st->tiles[s].ptr, st->htiles[s].data(),
                                  sizeof(int4) * st->htiles[s].size(), cudaMemcpyHostToDevice, s0));
    DAGE_TRY(st->jobs[s].alloc(sizeof(NearJob) * job));
  }
  DAGE_CUDA_TRY(cudaStreamSynchronize(s0));
  return 0;
}

void near_f16_set_destroy(NearF16Set *st) {
  if (!st) return;
  for (DevBuf *b : {&st->X, &st->U, &st->W, &st->maxbits, &st->gin, &st->g01, &st->wcoef,
                    &st->rhoptr, &st->wptr, &st->err})
    b->release();
  for (int s = 0; s < 3; ++s) {
    st->jobs[s].release();
    st->tiles[s].release();
  }
  delete st;
}

int near_f16_set_bind(NearF16Set *st, const double *const *rho, double *const *V,
                      const double *const *w, cudaStream_t s) {
  const NearF16Plan *pl = st->plan;
  const NearGeom &g = pl->g;
  const int n = st->n;
  std::vector<NearJob> js[3];
  long long xoff = 0, yoff = 0;
  for (int i = 0; i < n; ++i)
    for (const auto &b : st->boxes) {
      const int vx = b.pos[0], vy = b.pos[1], vz = b.pos[2];
      NearJob x{}, y{}, z{};
      // stage x: rows (a = y, b = z) of the near region of density i, K = x
      x.koff = pl->koff[0][vx];
      x.ax = g.q0[0][vx] - x.koff;
      x.ay = g.q0[1][vy];
      x.az = g.q0[2][vz] + i * g.npts[2];
      x.na = g.nq[1][vy];
      x.nb = g.nq[2][vz];
      x.N = g.own[0][vx];
      x.brow = pl->brow[0][vx];
      x.kr_ps = ceil_div(x.N, 128);
      x.band = g.band[0][vx];
      x.ooff = xoff;  // U slices of this job: x own
      x.ta = ceil_div(x.na, kRowsA);
      x.inst = i;
      // stage y: U rows (a = z near, b = x own), K = y near
      y.ax = 0;
      y.ay = 0;
      y.az = (int)xoff;
      y.na = g.nq[2][vz];
      y.nb = g.own[0][vx];
      y.N = g.own[1][vy];
      y.brow = pl->brow[1][vy];
      y.kr_ps = ceil_div(y.N, 128);
      y.band = g.band[1][vy];
      y.ooff = yoff;  // W slices: y own
      y.ta = ceil_div(y.na, kRowsA);
      y.inst = i;
      // stage z: W rows (a = x own, b = y own), K = z near -> V
      z.ax = 0;
      z.ay = 0;
      z.az = (int)yoff;
      z.na = g.own[0][vx];
      z.nb = g.own[1][vy];
      z.N = g.own[2][vz];
      z.brow = pl->brow[2][vz];
      z.kr_ps = ceil_div(z.N, 128);
      z.band = g.band[2][vz];
      z.ta = ceil_div(z.na, kRowsA);
      z.inst = i;
      z.V = V[i] + g.p0[0][vx] + (size_t)g.npts[0] * g.p0[1][vy] +
            (size_t)g.npts[0] * g.npts[1] * g.p0[2][vz];
      z.vs_b = g.npts[0];
      z.vs_n = (long long)g.npts[0] * g.npts[1];
      js[0].push_back(x);
      js[1].push_back(y);
      js[2].push_back(z);
      xoff += x.N;
      yoff += y.N;
    }
  for (int d = 0; d < 3; ++d)
    DAGE_CUDA_TRY(cudaMemcpyAsync(st->jobs[d].ptr, js[d].data(), sizeof(NearJob) * js[d].size(),
                                  cudaMemcpyHostToDevice, s));
  DAGE_CUDA_TRY(cudaMemcpyAsync(st->rhoptr.ptr, rho, sizeof(double *) * n, cudaMemcpyHostToDevice, s));
  DAGE_CUDA_TRY(cudaMemcpyAsync(st->wptr.ptr, w, sizeof(double *) * n, cudaMemcpyHostToDevice, s));
  // the host tables are pageable and go out of scope
  DAGE_CUDA_TRY(cudaStreamSynchronize(s));
  return 0;
}

int near_f16_set_run(NearF16Set *st, cudaStream_t s) {
  const NearF16Plan *pl = st->plan;
  const NearGeom &g = pl->g;
  const int n = st->n, P = st->P;
  const long long cube = (long long)g.npts[0] * g.npts[1] * g.npts[2];
  DAGE_CUDA_TRY(cudaMemsetAsync(st->maxbits.ptr, 0, sizeof(unsigned) * n, s));
  const int bx = (int)std::min<long long>((cube + 255) / 256, sm_count() * 4LL);
  near_absmax_kernel<<<dim3(bx, n), 256, 0, s>>>(st->rhoptr.as<const double *>(), cube,
                                                 st->maxbits.as<unsigned>());
  DAGE_CUDA_TRY(cudaGetLastError());
  near_scales_kernel<<<n, 128, 0, s>>>(st->maxbits.as<unsigned>(), pl->l1[0].as<double>(),
                                       pl->l1[1].as<double>(), pl->psc[0].as<double>(),
                                       pl->psc[1].as<double>(), pl->psc[2].as<double>(),
                                       st->wptr.as<const double *>(), P, st->gin.as<float>(),
                                       st->g01.as<float>(), st->wcoef.as<float>());
  DAGE_CUDA_TRY(cudaGetLastError());
  const long long xe = (long long)n * st->xs_rows * st->ld[0];
  const long long per = st->xs_rows * st->ld[0];
  const int sx = (int)std::min<long long>((per + 255) / 256, sm_count() * 8LL);
  near_split_input_kernel<<<dim3(sx, n), 256, 0, s>>>(
      st->rhoptr.as<const double *>(), g.npts[0], st->xs_rows, st->ld[0], st->gin.as<float>(),
      st->xp, st->xp + xe);
  DAGE_CUDA_TRY(cudaGetLastError());

  const long long ue = st->xsl * st->zpad * st->ld[1];
  const long long we = (long long)st->G * st->ysl * st->xpad * st->ld[2];
  NearArgs base{};
  base.err = st->err.as<int>();
  base.wait_limit = g_wait_limit;
  base.drain_limit = 4000000000LL;
  base.ng = 1;
  base.gstride = 2 * P;
  base.wstride = P;
  auto launch = [&](int stage, bool fin, const NearArgs &a) -> int {
    const CUtensorMap *mA = st->mapA[stage], *mB = st->mapB[stage];
    if (st->tile_n == 64)
      return fin ? launch_near<true, 64, 4>(mA, mB, a, s) : launch_near<false, 64, 4>(mA, mB, a, s);
    return fin ? launch_near<true, 128, 3>(mA, mB, a, s) : launch_near<false, 128, 3>(mA, mB, a, s);
  };
  for (int p = 0; p < P; ++p) {
    const int slot = p % st->G;
    {  // stage x -> U
      NearArgs a = base;
      a.jobs = st->jobs[0].as<NearJob>();
      a.tiles = st->tiles[0].as<int4>();
      a.ntiles = st->ntiles[0];
      a.p = p;
      a.gscale = st->g01.as<float>();
      a.out0 = st->up;
      a.out1 = st->up + ue;
      a.oslice0 = 0;
      a.opad = st->zpad;
      a.ldn = st->ld[1];
      DAGE_TRY(launch(0, false, a));
    }
    {  // stage y -> W slot
      NearArgs a = base;
      a.jobs = st->jobs[1].as<NearJob>();
      a.tiles = st->tiles[1].as<int4>();
      a.ntiles = st->ntiles[1];
      a.p = p;
      a.gscale = st->g01.as<float>() + P;
      a.out0 = st->wp;
      a.out1 = st->wp + we;
      a.oslice0 = (long long)slot * st->ysl;
      a.opad = st->xpad;
      a.ldn = st->ld[2];
      DAGE_TRY(launch(1, false, a));
    }
    if (slot == st->G - 1 || p == P - 1) {  // stage z over the group -> V
      NearArgs a = base;
      const int p0 = p - slot;
      a.jobs = st->jobs[2].as<NearJob>();
      a.tiles = st->tiles[2].as<int4>();
      a.ntiles = st->ntiles[2];
      a.p = p0;
      a.ng = slot + 1;
      a.slot_rows = (int)st->ysl;
      a.wcoef = st->wcoef.as<float>();
      a.accumulate = p0 > 0;
      DAGE_TRY(launch(2, true, a));
    }
  }
  return 0;
}

int near_f16_set_check(NearF16Set *st, cudaStream_t s) {
  int herr = 0;
  DAGE_CUDA_TRY(cudaMemcpyAsync(&herr, st->err.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
  DAGE_CUDA_TRY(cudaStreamSynchronize(s));
  if (herr) {
    cudaMemsetAsync(st->err.ptr, 0, sizeof(int), s);
    return fail(DAGE_E_TIMEOUT, "near-field tensor-core kernel timed out waiting on an mbarrier");
  }
  return 0;
}

}  // namespace dage
