// op3d.cu -- the tensor-product cube operator (Coulomb3D / Helmholtz3D cube
// part) on one B200: quadrature and operator matrices built on the GPU in
// FP64, the FP64 contraction, the coda term and the fused LIP-weighted
// energy, and the C ABI around them.
//
// Contraction layout.  V = sum_p w_p (T^x_p (x) T^y_p (x) T^z_p) rho is
// computed as three "contract the fastest index and rotate" stages per
// t-point:
//     U(b,c,i) = sum_a rho(a,b,c) Tx(i,a)     rho: a fastest -> U: b fastest
//     W(c,i,j) = sum_b U(b,c,i)  Ty(j,b)      -> W: c fastest
//     V(i,j,k) = sum_c W(c,i,j)  Tz(k,c)      -> V: i fastest (input layout)
// Every stage is the same GEMM D(R, n) = sum_K X(K, R) T(n, K) with both
// operands contiguous in K and the result written R-fastest, so one kernel
// (and one tensor-core kernel in op3d_mixed.cu) serves all three.  This is
// the same arithmetic as the reference's per-slice DGEMMs
// (src/bubbles/function3d.F90:4296-4332), reordered for coalescing.
#include <cmath>
#include <cstdio>
#include <string>
#include <mutex>
#include <cstring>

#include "expo.cuh"
#include "fp64_stage.cuh"
#include "op3d.cuh"
#include "tune.h"

namespace dage {

namespace {

// ---------------------------------------------------------------------------
// Gauss-Legendre t-points and weights (src/bubbles/gauss.F90:307-383):
// Newton iteration on P_n from z = cos(pi (i - 1/4) / (n + 1/2)), then the
// linear map to [tstart, tlin] and the logarithmic map to [tlin, tlog].
// ---------------------------------------------------------------------------
__global__ void quad_kernel(int nlin, int nlog, double tstart, double tlin, double tlog,
                            double *tp, double *tw) {
  const int seg = blockIdx.x;  // 0: linear part, 1: logarithmic tail
  const int n = seg == 0 ? nlin : nlog;
  const int i = threadIdx.x + 1;
  const int m = (n + 1) / 2;
  if (n <= 0 || i > m) return;
  double *x = tp + (seg == 0 ? 0 : nlin);
  double *w = tw + (seg == 0 ? 0 : nlin);
  const double pi = acos(-1.0);
  double z = cos(pi * (i - 0.25) / (n + 0.5));
  double p1, p2, p3, pp, z1;
  for (int it = 0; it < 100; ++it) {  // converges in a handful of steps
    p1 = 1.0;
    p2 = 0.0;
    for (int j = 1; j <= n; ++j) {
      p3 = p2;
      p2 = p1;
      p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
    }
    pp = n * (z * p1 - p2) / (z * z - 1.0);
    z1 = z;
    z = z1 - p1 / pp;
    if (!(fabs(z - z1) > 3.0e-15)) break;
  }
  const double wt = 2.0 / ((1.0 - z * z) * pp * pp);
  const int idx[2] = {i - 1, n - i};
  const double xs[2] = {-z, z};
  for (int s = 0; s < 2; ++s) {
    double t = xs[s], ww = wt;
    if (seg == 0) {
      t = 0.5 * ((tlin + tstart) + (tlin - tstart) * t);
      ww = 0.5 * (tlin - tstart) * ww;
    } else {
      t = tlin * pow(tlog / tlin, 0.5 * (t + 1.0));
      ww = 0.5 * log(tlog / tlin) * ww * t;
    }
    x[idx[s]] = t;
    w[idx[s]] = ww;
  }
}

// ---------------------------------------------------------------------------
// Operator matrices (src/bubbles/exponentials.F90:178-346, no PBC images):
//   T_p(i, j) = sum over the input cells c that contain point j of
//     h_c * sum_k coeff[k][j - j0(c)] * I_{nlip-1-k}(first, last, t_p h_c, q_i)
// with q_i = (x_i - celld_c)/h_c + first the output point in the cell's
// coordinates.  One thread per (t-point, cell, output point); cells of one
// parity per launch, so the two cells sharing a boundary point never write
// it concurrently (the shared point receives c's term, then c+1's term).
// ---------------------------------------------------------------------------
struct TmatArgs {
  const double *tp;
  const double *celld;
  const double *h;
  const double *xout;
  const double *coeff;  // nlip*nlip, coeff[k*nlip + j]
  double first, last;
  int P, ncell, n_in, n_out;
  double *T;  // T[p][i_out][j_in]
};

template <int NLIP>
__global__ void tmatrix_kernel(TmatArgs a, int parity) {
  const int ncells_par = (a.ncell - parity + 1) / 2;
  const long long total = (long long)a.P * ncells_par * a.n_out;
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
       id += (long long)gridDim.x * blockDim.x) {
    const int io = (int)(id % a.n_out);
    const long long rest = id / a.n_out;
    const int c = parity + 2 * (int)(rest % ncells_par);
    const int ip = (int)(rest / ncells_par);
    const double h = a.h[c];
    const double pst0 = (a.xout[io] - a.celld[c]) / h + a.first;
    double vals[NLIP];
    expo::integrals(a.first, a.last, a.tp[ip] * h, pst0, NLIP, vals);
    double *row = a.T + ((size_t)ip * a.n_out + io) * a.n_in + (size_t)c * (NLIP - 1);
#pragma unroll
    for (int j = 0; j < NLIP; ++j) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < NLIP; ++k) s += a.coeff[k * NLIP + j] * vals[k];
      row[j] += s * h;
    }
  }
}

int launch_tmatrix(const TmatArgs &a, int nlip, cudaStream_t s) {
  for (int parity = 0; parity < 2; ++parity) {
    const long long total = (long long)a.P * ((a.ncell - parity + 1) / 2) * a.n_out;
    if (total == 0) continue;
    const int threads = 128;
    const int blocks = (int)std::min<long long>((total + threads - 1) / threads, 148LL * 64);
    switch (nlip) {
      case 2: tmatrix_kernel<2><<<blocks, threads, 0, s>>>(a, parity); break;
      case 3: tmatrix_kernel<3><<<blocks, threads, 0, s>>>(a, parity); break;
      case 4: tmatrix_kernel<4><<<blocks, threads, 0, s>>>(a, parity); break;
      case 5: tmatrix_kernel<5><<<blocks, threads, 0, s>>>(a, parity); break;
      case 6: tmatrix_kernel<6><<<blocks, threads, 0, s>>>(a, parity); break;
      case 7: tmatrix_kernel<7><<<blocks, threads, 0, s>>>(a, parity); break;
      default: return fail(DAGE_E_UNSUPPORTED, "nlip=%d", nlip);
    }
    DAGE_CUDA_TRY(cudaGetLastError());
  }
  return 0;
}

// ---------------------------------------------------------------------------
// FP64 contraction stage (fp64_stage.cuh) on DMMA
// ---------------------------------------------------------------------------
constexpr int BM = kFp64TileM, BN = kFp64TileN, BK = 16, SROW = BK + 4, NST = 3;

__device__ __forceinline__ void cp_async8(double *smem, const double *gmem, bool pred) {
  const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(sa), "l"(gmem),
               "r"(pred ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
// D(8x8) += A(8x4, row) B(4x8, col); lane l holds A[l/4][l%4], B[l%4][l/4]
// and D[l/4][2(l%4) + {0,1}]
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// TN: tile width in n (32, 64 or 128); warps 2 (M) x 4 (N), each 64 x TN/4.
template <int TN>
constexpr int stage_smem() {
  return NST * (BM + TN) * SROW * (int)sizeof(double);
}

template <bool ACCUM, int TN>
__device__ __forceinline__ void stage_tile(const StageDesc &d, double alpha, int m0, int n0) {
  constexpr int NB = TN / 32;   // 8-column MMA tiles per warp
  constexpr int BR = TN / 16;   // B rows copied per thread per K step
  extern __shared__ double fsm[];
  double *As = fsm;                    // [NST][BM][SROW]
  double *Bs = fsm + NST * BM * SROW;  // [NST][TN][SROW]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp & 1) * 64, wn = (warp >> 1) * (TN / 4);
  int kt0 = 0, kt1 = (d.K + BK - 1) / BK - 1;
  if (d.krange) {  // bands are kept per 128 columns
    const int2 r = d.krange[n0 / kFp64TileN];
    kt0 = r.x / BK;
    kt1 = r.y / BK;
  }
  const int nk = kt1 - kt0 + 1;

  // this thread copies rows (tid >> 4) + 16 i at K offset tid & 15
  const int kk = tid & 15;
  const double *arow[8];
  const double *brow[BR];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const long long m = m0 + (tid >> 4) + 16 * i;
    arow[i] = m < d.M ? d.X + (m % d.a_d0) * d.a_s1 + (m / d.a_d0) * d.a_s2 : nullptr;
  }
#pragma unroll
  for (int i = 0; i < BR; ++i) {
    const int n = n0 + (tid >> 4) + 16 * i;
    brow[i] = n < d.N ? d.T + (size_t)n * d.ldt : nullptr;
  }
  auto load = [&](int slot, int kt) {
    const int k = kt * BK + kk;
    double *as = As + slot * BM * SROW + (tid >> 4) * SROW + kk;
    double *bs = Bs + slot * TN * SROW + (tid >> 4) * SROW + kk;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const bool pa = arow[i] && k < d.K;
      cp_async8(as + 16 * i * SROW, pa ? arow[i] + k : d.X, pa);
    }
#pragma unroll
    for (int i = 0; i < BR; ++i) {
      const bool pb = brow[i] && k < d.K;
      cp_async8(bs + 16 * i * SROW, pb ? brow[i] + k : d.T, pb);
    }
  };

  double acc[8][NB][2];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < NB; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
  for (int st = 0; st < NST - 1; ++st) {
    if (st < nk) load(st, kt0 + st);
    cp_async_commit();
  }
  for (int i = 0; i < nk; ++i) {
    cp_async_wait<NST - 2>();
    __syncthreads();  // slot i landed for all threads; slot i-1 is free
    if (i + NST - 1 < nk) load((i + NST - 1) % NST, kt0 + i + NST - 1);
    cp_async_commit();
    const double *as = As + (i % NST) * BM * SROW + (wm + (lane >> 2)) * SROW + (lane & 3);
    const double *bs = Bs + (i % NST) * TN * SROW + (wn + (lane >> 2)) * SROW + (lane & 3);
#pragma unroll
    for (int ks = 0; ks < BK / 4; ++ks) {
      double fa[8], fb[NB];
#pragma unroll
      for (int mb = 0; mb < 8; ++mb) fa[mb] = as[mb * 8 * SROW + ks * 4];
#pragma unroll
      for (int nb = 0; nb < NB; ++nb) fb[nb] = bs[nb * 8 * SROW + ks * 4];
#pragma unroll
      for (int mb = 0; mb < 8; ++mb)
#pragma unroll
        for (int nb = 0; nb < NB; ++nb) dmma(acc[mb][nb], fa[mb], fb[nb]);
    }
  }
  cp_async_wait<0>();

#pragma unroll
  for (int mb = 0; mb < 8; ++mb) {
    const long long m = m0 + wm + mb * 8 + (lane >> 2);
    if (m >= d.M) continue;
    double *orow = d.out + (m % d.o_d0) * d.o_s1 + (m / d.o_d0) * d.o_s2;
#pragma unroll
    for (int nb = 0; nb < NB; ++nb)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int n = n0 + wn + nb * 8 + 2 * (lane & 3) + h;
        if (n >= d.N) continue;
        double *dst = orow + (long long)n * d.o_sn;
        if (ACCUM)
          atomicAdd(dst, alpha * acc[mb][nb][h]);
        else
          *dst = alpha * acc[mb][nb][h];
      }
  }
}

template <bool ACCUM, int TN>
__global__ void __launch_bounds__(256, 1)
    stage_fp64_kernel(const __grid_constant__ StageDesc d, double alpha) {
  stage_tile<ACCUM, TN>(d, alpha, blockIdx.x * BM, blockIdx.y * TN);
}

template <bool ACCUM, int TN>
__global__ void __launch_bounds__(256, 1)
    stage_fp64_batched_kernel(const StageDesc *__restrict__ descs, int p, double alpha) {
  StageDesc d = descs[blockIdx.z];
  d.T += p * d.t_ps;
  if (d.krange) d.krange += p * d.kr_ps;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * TN;
  if (m0 >= d.M || n0 >= d.N) return;  // uniform across the block
  stage_tile<ACCUM, TN>(d, d.wp ? d.wp[p] : alpha, m0, n0);
}

// Band of each (t-point, 128-row tile) of an axis matrix T[p][n][K]: the
// first and last K index holding an entry above 2^-64 of its row's scale
// 2^ceil(log2 max_K |T(n, :)|).  One block per (p, tile), one warp per row.
// Tiles of all-zero rows get [0, 0].
__global__ void band_kernel(const double *__restrict__ T, int K, int N, int ntiles,
                            int2 *range) {
  const int p = blockIdx.x / ntiles, tile = blockIdx.x % ntiles;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __shared__ int lo, hi;
  if (threadIdx.x == 0) {
    lo = K;
    hi = -1;
  }
  __syncthreads();
  for (int rr = warp; rr < BN; rr += blockDim.x >> 5) {
    const int n = tile * BN + rr;
    if (n >= N) break;
    const double *row = T + ((size_t)p * N + n) * K;
    double m = 0.0;
    for (int k = lane; k < K; k += 32) m = fmax(m, fabs(row[k]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (m == 0.0) continue;
    const double thr = ldexp(exp2(ceil(log2(m))), -64);
    int mylo = K, myhi = -1;
    for (int k = lane; k < K; k += 32)
      if (fabs(row[k]) > thr) {
        mylo = min(mylo, k);
        myhi = max(myhi, k);
      }
    atomicMin(&lo, mylo);
    atomicMax(&hi, myhi);
  }
  __syncthreads();
  if (threadIdx.x == 0) range[blockIdx.x] = hi < 0 ? make_int2(0, 0) : make_int2(lo, hi);
}

// ---------------------------------------------------------------------------
// Coda + LIP-weighted integral, deterministic two-pass FP64 reduction.
// ---------------------------------------------------------------------------
constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 148 * 4;

__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  v = 0.0;
  if (wid == 0) {
    v = lane < (blockDim.x >> 5) ? sh[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

__global__ void __launch_bounds__(kRedThreads)
    finalize_kernel(const double *__restrict__ f1, double *__restrict__ f2,
                    const double *__restrict__ rho,
                    double coda, const double *__restrict__ wx, const double *__restrict__ wy,
                    const double *__restrict__ wz, int nx, int ny, int nz, double *partials,
                    int want_integral) {
  __shared__ double sh[32];
  // one warp per x row (y, z): the row's weight wy wz once, lanes over x
  // (coalesced, no per-element index division)
  const int lane = threadIdx.x & 31;
  const long long rows = (long long)ny * nz;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  double s = 0.0;
  for (long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows;
       r += nwarps) {
    const size_t base = (size_t)r * nx;
    double srow = 0.0;
    for (int x = lane; x < nx; x += 32) {
      const size_t i = base + x;
      double v2 = 1.0;
      if (f2) {
        v2 = f2[i];
        if (rho) {
          v2 = v2 + coda * rho[i];
          f2[i] = v2;
        }
      }
      if (want_integral) srow += f1[i] * v2 * wx[x];
    }
    if (want_integral) s += srow * (wy[r % ny] * wz[r / ny]);
  }
  if (!want_integral) return;
  s = block_sum(s, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void sum_partials_kernel(const double *partials, int n, double *result) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += partials[i];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) *result = s;
}

}  // namespace

template <bool ACCUM, int TN>
int attr_variants() {
  DAGE_CUDA_TRY(cudaFuncSetAttribute(stage_fp64_kernel<ACCUM, TN>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, stage_smem<TN>()));
  DAGE_CUDA_TRY(cudaFuncSetAttribute(stage_fp64_batched_kernel<ACCUM, TN>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, stage_smem<TN>()));
  return 0;
}

int prepare_fp64_stages() {
  // once per process
  static std::mutex mu;
  static bool done = false;
  std::lock_guard<std::mutex> lock(mu);
  if (done) return 0;
  DAGE_TRY((attr_variants<false, 32>()));
  DAGE_TRY((attr_variants<true, 32>()));
  DAGE_TRY((attr_variants<false, 64>()));
  DAGE_TRY((attr_variants<true, 64>()));
  DAGE_TRY((attr_variants<false, 128>()));
  DAGE_TRY((attr_variants<true, 128>()));
  done = true;
  return 0;
}

template <bool ACCUM, int TN>
int launch_single(const StageDesc &d, double alpha, cudaStream_t s) {
  auto kern = stage_fp64_kernel<ACCUM, TN>;
  DAGE_TRY(prepare_fp64_stages());
  dim3 grid(ceil_div(d.M, BM), ceil_div(d.N, TN));
  if (grid.y > 65535) return fail(DAGE_E_UNSUPPORTED, "N=%d too large", d.N);
  kern<<<grid, 256, stage_smem<TN>(), s>>>(d, alpha);
  DAGE_CUDA_TRY(cudaGetLastError());
  return 0;
}

template <bool ACCUM, int TN>
int launch_batched(const StageDesc *d_descs, int ndesc, int mtiles, int ncols, int p,
                   double alpha, cudaStream_t s) {
  auto kern = stage_fp64_batched_kernel<ACCUM, TN>;
  DAGE_TRY(prepare_fp64_stages());
  dim3 grid(mtiles, ceil_div(ncols, TN), ndesc);
  if (grid.y > 65535 || ndesc > 65535) return fail(DAGE_E_UNSUPPORTED, "batch too large");
  kern<<<grid, 256, stage_smem<TN>(), s>>>(d_descs, p, alpha);
  DAGE_CUDA_TRY(cudaGetLastError());
  return 0;
}

int launch_fp64_stage(const StageDesc &d, double alpha, bool accumulate, cudaStream_t s, int tn) {
  switch (tn) {
    case 32: return accumulate ? launch_single<true, 32>(d, alpha, s) : launch_single<false, 32>(d, alpha, s);
    case 64: return accumulate ? launch_single<true, 64>(d, alpha, s) : launch_single<false, 64>(d, alpha, s);
    case 128: return accumulate ? launch_single<true, 128>(d, alpha, s) : launch_single<false, 128>(d, alpha, s);
  }
  return fail(DAGE_E_INVALID, "tile width %d", tn);
}

int launch_fp64_stages(const StageDesc *d_descs, int ndesc, int mtiles, int ncols, int p,
                       double alpha, bool accumulate, cudaStream_t s, int tn) {
  if (ndesc <= 0) return 0;
#define DAGE_BATCHED(TNV)                                                                  \
  return accumulate ? launch_batched<true, TNV>(d_descs, ndesc, mtiles, ncols, p, alpha, s) \
                    : launch_batched<false, TNV>(d_descs, ndesc, mtiles, ncols, p, alpha, s)
  switch (tn) {
    case 32: DAGE_BATCHED(32);
    case 64: DAGE_BATCHED(64);
    case 128: DAGE_BATCHED(128);
  }
#undef DAGE_BATCHED
  return fail(DAGE_E_INVALID, "tile width %d", tn);
}

int launch_stage_fp64(const double *X, long long ldx, int M, int N, int K, const double *T,
                      long long ldt, double *out, double alpha, bool accumulate,
                      cudaStream_t s, const int2 *krange, int tn) {
  return launch_fp64_stage(cube_stage(X, ldx, M, N, K, T, ldt, out, krange), alpha, accumulate, s,
                           tn);
}

int launch_band(const double *T, int K, int N, int P, int2 *range, cudaStream_t s) {
  const int ntiles = ceil_div(N, BN);
  band_kernel<<<P * ntiles, 256, 0, s>>>(T, K, N, ntiles, range);
  DAGE_CUDA_TRY(cudaGetLastError());
  return 0;
}

int finalize_partials_count() { return kRedBlocks + 1; }

int launch_finalize(const double *f1, double *f2_or_V, const double *rho_for_coda, double coda,
                    const double *wx, const double *wy, const double *wz, int nx, int ny,
                    int nz, double *partials, int npartials, double *d_result,
                    cudaStream_t s) {
  const int want = d_result != nullptr;
  if (!want && !rho_for_coda) return 0;
  const int blocks = std::min(kRedBlocks, npartials - 1);
  finalize_kernel<<<blocks, kRedThreads, 0, s>>>(f1, f2_or_V, rho_for_coda, coda, wx, wy, wz,
                                                  nx, ny, nz, partials, want);
  DAGE_CUDA_TRY(cudaGetLastError());
  if (want) {
    sum_partials_kernel<<<1, 1024, 0, s>>>(partials, blocks, d_result);
    DAGE_CUDA_TRY(cudaGetLastError());
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Operator construction
// ---------------------------------------------------------------------------
int build_quadrature(const dage_quad &q, std::vector<double> &tp, std::vector<double> &tw,
                     DevBuf &d_tp, cudaStream_t s) {
  const int P = q.nlin + q.nlog;
  TmpBuf d_tw;
  DAGE_TRY(d_tp.alloc(sizeof(double) * P));
  DAGE_TRY(d_tw.alloc(sizeof(double) * P));
  quad_kernel<<<2, 128, 0, s>>>(q.nlin, q.nlog, q.tstart, q.tlin, q.tlog, d_tp.as<double>(),
                                d_tw.as<double>());
  DAGE_CUDA_TRY(cudaGetLastError());
  tp.resize(P);
  tw.resize(P);
  DAGE_CUDA_TRY(cudaMemcpyAsync(tp.data(), d_tp.ptr, sizeof(double) * P, cudaMemcpyDeviceToHost, s));
  DAGE_CUDA_TRY(cudaMemcpyAsync(tw.data(), d_tw.ptr, sizeof(double) * P, cudaMemcpyDeviceToHost, s));
  DAGE_CUDA_TRY(cudaStreamSynchronize(s));
  return 0;
}

int build_axis_matrix(const Axis &ai, const double *out_points, int n_out, const double *d_tp,
                      int P, double *d_T, cudaStream_t s) {
  LipBasis L;
  DAGE_TRY(make_lip_basis(ai.nlip, ai.grid_type, L));
  const size_t nT = (size_t)P * n_out * ai.n();
  DAGE_CUDA_TRY(cudaMemsetAsync(d_T, 0, sizeof(double) * nT, s));
  TmpBuf d_celld, d_h, d_x, d_c;
  DAGE_TRY(d_celld.alloc(sizeof(double) * ai.ncell));
  DAGE_TRY(d_h.alloc(sizeof(double) * ai.ncell));
  DAGE_TRY(d_x.alloc(sizeof(double) * n_out));
  DAGE_TRY(d_c.alloc(sizeof(double) * L.coeff.size()));
  DAGE_CUDA_TRY(cudaMemcpyAsync(d_celld.ptr, ai.celld.data(), sizeof(double) * ai.ncell,
                                cudaMemcpyHostToDevice, s));
  DAGE_CUDA_TRY(cudaMemcpyAsync(d_h.ptr, ai.h.data(), sizeof(double) * ai.ncell,
                                cudaMemcpyHostToDevice, s));
  DAGE_CUDA_TRY(cudaMemcpyAsync(d_x.ptr, out_points, sizeof(double) * n_out,
                                cudaMemcpyHostToDevice, s));
  DAGE_CUDA_TRY(cudaMemcpyAsync(d_c.ptr, L.coeff.data(), sizeof(double) * L.coeff.size(),
                                cudaMemcpyHostToDevice, s));
  TmatArgs a;
  a.tp = d_tp;
  a.celld = d_celld.as<double>();
  a.h = d_h.as<double>();
  a.xout = d_x.as<double>();
  a.coeff = d_c.as<double>();
  a.first = L.first;
  a.last = L.last;
  a.P = P;
  a.ncell = ai.ncell;
  a.n_in = ai.n();
  a.n_out = n_out;
  a.T = d_T;
  DAGE_TRY(launch_tmatrix(a, ai.nlip, s));
  DAGE_CUDA_TRY(cudaStreamSynchronize(s));  // before the small buffers go
  return 0;
}

// ---------------------------------------------------------------------------
// On-disk operator cache (dage_op3d_create_cached).  A file holds the key
// and the FP64 matrices, in the stream-access layout of the reference's
// store_Grid1Ds / resume_Grid1Ds (src/bubbles/grid.F90:2024-2068): per grid
// ncell, nlip, cell_scales, grid_type (int32 / float64), here preceded by a
// magic and version and followed by qmin (the reference resumes grids at
// qmin = 0; the operator's matrices depend on it), for the 3 input and the 3
// output axes; then the quadrature (nlin, nlog, tstart, tlin, tlog), P, and
// per axis its owner index and, for owner axes, the P x n_out x n_in matrix.
// ---------------------------------------------------------------------------
namespace {
constexpr char kCacheMagic[8] = {'D', 'A', 'G', 'E', 'O', 'P', '3', 'D'};
constexpr int kCacheVersion = 1;

void put_axis(std::string &b, const Axis &a) {
  auto put = [&](const void *p, size_t n) { b.append(static_cast<const char *>(p), n); };
  const int32_t nc = a.ncell, nl = a.nlip, gt = a.grid_type;
  put(&nc, 4);
  put(&nl, 4);
  put(a.h.data(), sizeof(double) * a.h.size());
  put(&gt, 4);
  put(&a.qmin, 8);
}

// the key bytes: magic, version, the six axes and the quadrature
std::string cache_key(const dage_op3d *op) {
  std::string b(kCacheMagic, 8);
  const int32_t v = kCacheVersion, three = 3;
  b.append(reinterpret_cast<const char *>(&v), 4);
  for (const Axis *ax : {op->in, op->out}) {
    b.append(reinterpret_cast<const char *>(&three), 4);
    for (int d = 0; d < 3; ++d) put_axis(b, ax[d]);
  }
  const int32_t q[2] = {op->quad.nlin, op->quad.nlog};
  const double t[3] = {op->quad.tstart, op->quad.tlin, op->quad.tlog};
  b.append(reinterpret_cast<const char *>(q), 8);
  b.append(reinterpret_cast<const char *>(t), 24);
  return b;
}

std::string cache_file(const std::string &dir, const std::string &key) {
  uint64_t h = 1469598103934665603ull;  // FNV-1a 64
  for (unsigned char c : key) h = (h ^ c) * 1099511628211ull;
  char name[40];
  std::snprintf(name, sizeof(name), "/op3d_%016llx.bin", (unsigned long long)h);
  return dir + name;
}
}  // namespace

// Reads the matrices of op from a cache file whose key matches; returns 1 if
// they were loaded, 0 if there is no matching file.
static int cache_load(dage_op3d *op, const std::string &path) {
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) return 0;
  const std::string key = cache_key(op);
  std::string got(key.size(), '\0');
  bool ok = std::fread(&got[0], 1, key.size(), f) == key.size() && got == key;
  int32_t P = 0, owner[3] = {0, 1, 2};
  ok = ok && std::fread(&P, 4, 1, f) == 1 && P == op->P;
  std::vector<double> host;
  for (int d = 0; d < 3 && ok; ++d) {
    ok = std::fread(&owner[d], 4, 1, f) == 1 && owner[d] == op->Towner[d];
    if (!ok || owner[d] != d) continue;
    const size_t nT = (size_t)op->P * op->nout[d] * op->nin[d];
    host.resize(nT);
    ok = std::fread(host.data(), sizeof(double), nT, f) == nT;
    if (ok) {
      if (op->Tbuf[d].alloc(sizeof(double) * nT) ||
          cudaMemcpy(op->Tbuf[d].ptr, host.data(), sizeof(double) * nT, cudaMemcpyHostToDevice) !=
              cudaSuccess) {
        std::fclose(f);
        return fail(DAGE_E_CUDA, "cache upload failed");
      }
    }
  }
  std::fclose(f);
  return ok ? 1 : 0;
}

static int cache_store(const dage_op3d *op, const std::string &path) {
  const std::string tmp = path + ".tmp";
  FILE *f = std::fopen(tmp.c_str(), "wb");
  if (!f) return fail(DAGE_E_INVALID, "cannot write operator cache %s", tmp.c_str());
  const std::string key = cache_key(op);
  bool ok = std::fwrite(key.data(), 1, key.size(), f) == key.size();
  const int32_t P = op->P;
  ok = ok && std::fwrite(&P, 4, 1, f) == 1;
  std::vector<double> host;
  for (int d = 0; d < 3 && ok; ++d) {
    const int32_t owner = op->Towner[d];
    ok = std::fwrite(&owner, 4, 1, f) == 1;
    if (!ok || owner != d) continue;
    const size_t nT = (size_t)op->P * op->nout[d] * op->nin[d];
    host.resize(nT);
    if (cudaMemcpy(host.data(), op->Tbuf[d].ptr, sizeof(double) * nT, cudaMemcpyDeviceToHost) !=
        cudaSuccess) {
      std::fclose(f);
      return fail(DAGE_E_CUDA, "cache download failed");
    }
    ok = std::fwrite(host.data(), sizeof(double), nT, f) == nT;
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok || std::rename(tmp.c_str(), path.c_str()) != 0) {
    std::remove(tmp.c_str());
    return fail(DAGE_E_INVALID, "cannot write operator cache %s", path.c_str());
  }
  return 0;
}

// Matrices from the cache directory when a file with this operator's key is
// there (cache_dir non-null), else built on the GPU (and stored there).
static int build_matrices(dage_op3d *op, const char *cache_dir = nullptr) {
  cudaStream_t s = op->stream;
  TmpBuf d_tp;
  DAGE_TRY(build_quadrature(op->quad, op->tp, op->tw, d_tp, s));
  const double two_over_sqrtpi = 2.0 / std::sqrt(std::acos(-1.0));
  op->w.resize(op->P);
  for (int p = 0; p < op->P; ++p) op->w[p] = two_over_sqrtpi * op->tw[p];
  op->coda = std::acos(-1.0) / (op->quad.tlog * op->quad.tlog);

  for (int d = 0; d < 3; ++d) {
    op->Towner[d] = d;
    for (int e = 0; e < d; ++e)
      if (same_axis(op->in[d], op->in[e]) && same_axis(op->out[d], op->out[e])) {
        op->Towner[d] = op->Towner[e];
        break;
      }
  }
  std::string path;
  int loaded = 0;
  if (cache_dir) {
    DAGE_CUDA_TRY(cudaStreamSynchronize(s));
    path = cache_file(cache_dir, cache_key(op));
    loaded = cache_load(op, path);
    if (loaded < 0 || loaded > 1) return loaded;  // an error code
  }
  op->from_cache = loaded == 1;
  for (int d = 0; d < 3; ++d) {
    if (op->Towner[d] != d) continue;
    const Axis &ai = op->in[d];
    const Axis &ao = op->out[d];
    const size_t nT = (size_t)op->P * ao.n() * ai.n();
    if (!loaded) {
      DAGE_TRY(op->Tbuf[d].alloc(sizeof(double) * nT));
      DAGE_TRY(build_axis_matrix(ai, ao.points.data(), ao.n(), d_tp.as<double>(), op->P,
                                 op->Tbuf[d].as<double>(), s));
    }
    DAGE_TRY(op->band[d].alloc(sizeof(int2) * (size_t)op->P * ceil_div(ao.n(), BN)));
    DAGE_TRY(launch_band(op->Tbuf[d].as<double>(), ai.n(), ao.n(), op->P,
                         op->band[d].as<int2>(), s));
  }
  d_tp.release();
  if (cache_dir && !loaded) {
    DAGE_CUDA_TRY(cudaStreamSynchronize(s));
    DAGE_TRY(cache_store(op, path));
  }
  return 0;
}

static int upload_weights(dage_op3d *op) {
  DAGE_TRY(op->d_w.alloc(sizeof(double) * op->P));
  DAGE_CUDA_TRY(cudaMemcpyAsync(op->d_w.ptr, op->w.data(), sizeof(double) * op->P,
                                cudaMemcpyHostToDevice, op->stream));
  if (op->precision != DAGE_FP64) DAGE_TRY(mixed_set_weights(op));
  return 0;
}

static int tune_fp64(dage_op3d *op);

static int create_impl(const dage_grid1d grid_in[3], const dage_grid1d grid_out[3],
                       const dage_quad *quad, int precision, dage_op3d *op,
                       const char *cache_dir = nullptr) {
  if (!grid_in || !grid_out || !quad) return fail(DAGE_E_INVALID, "null argument");
  if (quad->nlin < 0 || quad->nlog < 0 || quad->nlin + quad->nlog < 1 ||
      quad->nlin > 256 || quad->nlog > 256)
    return fail(DAGE_E_INVALID, "quadrature needs 1..512 t-points");
  if (quad->nlog > 0 && !(quad->tlog > quad->tlin && quad->tlin > 0.0))
    return fail(DAGE_E_INVALID, "logarithmic tail needs 0 < tlin < tlog");
  if (precision != DAGE_FP64 && precision != DAGE_MIXED_BF16X3 &&
      precision != DAGE_MIXED_BF16X6 && precision != DAGE_MIXED_FP16X3)
    return fail(DAGE_E_INVALID, "unknown precision %d", precision);
  op->precision = precision;
  op->quad = *quad;
  op->P = quad->nlin + quad->nlog;
  DAGE_CUDA_TRY(cudaGetDevice(&op->device));
  for (int d = 0; d < 3; ++d) {
    DAGE_TRY(make_axis(grid_in[d], op->in[d]));
    DAGE_TRY(make_axis(grid_out[d], op->out[d]));
    op->nin[d] = op->in[d].n();
    op->nout[d] = op->out[d].n();
    if (op->in[d].nlip != op->in[0].nlip || op->in[d].grid_type != op->in[0].grid_type)
      return fail(DAGE_E_UNSUPPORTED, "all axes must share nlip and grid_type");
  }
  op->same_grid = same_axis(op->in[0], op->out[0]) && same_axis(op->in[1], op->out[1]) &&
                  same_axis(op->in[2], op->out[2]);
  // the compute stream and the host-pointer pipeline's copy-in and copy-out
  // streams
  DAGE_CUDA_TRY(cudaStreamCreateWithFlags(&op->own_stream, cudaStreamNonBlocking));
  DAGE_CUDA_TRY(cudaStreamCreateWithFlags(&op->pipe_in, cudaStreamNonBlocking));
  DAGE_CUDA_TRY(cudaStreamCreateWithFlags(&op->pipe_out, cudaStreamNonBlocking));
  op->stream = op->own_stream;
  DAGE_CUDA_TRY(cudaEventCreate(&op->ev0));
  DAGE_CUDA_TRY(cudaEventCreate(&op->ev1));
  DAGE_TRY(build_matrices(op, cache_dir));
  for (int d = 0; d < 3; ++d) {
    DAGE_TRY(op->wts[d].alloc(sizeof(double) * op->nout[d]));
    DAGE_CUDA_TRY(cudaMemcpyAsync(op->wts[d].ptr, op->out[d].weights.data(),
                                  sizeof(double) * op->nout[d], cudaMemcpyHostToDevice,
                                  op->stream));
  }
  DAGE_TRY(op->partials.alloc(sizeof(double) * (finalize_partials_count() + 1)));
  if (precision != DAGE_FP64) DAGE_TRY(mixed_setup(op));
  DAGE_TRY(upload_weights(op));
  DAGE_CUDA_TRY(cudaStreamSynchronize(op->stream));
  if (precision == DAGE_FP64) DAGE_TRY(tune_fp64(op));
  else DAGE_TRY(mixed_tune(op));
  return 0;
}

static void destroy_impl(dage_op3d *op) {
  if (!op) return;
  if (op->stream) cudaStreamSynchronize(op->stream);
  mixed_destroy(op);
  for (int d = 0; d < 3; ++d) {
    op->Tbuf[d].release();
    op->band[d].release();
    op->wts[d].release();
  }
  op->d_w.release();
  op->d_rho.release();
  op->d_V.release();
  op->tmp1.release();
  op->tmp2.release();
  op->partials.release();
  if (op->pipe_in) cudaStreamSynchronize(op->pipe_in);
  if (op->pipe_out) cudaStreamSynchronize(op->pipe_out);
  for (int k = 0; k < 2; ++k) {
    op->pipe_rho[k].release();
    op->pipe_V[k].release();
    for (cudaEvent_t e : {op->pipe_h2d[k], op->pipe_comp[k], op->pipe_d2h[k]})
      if (e) cudaEventDestroy(e);
  }
  if (op->pipe_in) cudaStreamDestroy(op->pipe_in);
  if (op->pipe_out) cudaStreamDestroy(op->pipe_out);
  for (cudaEvent_t e : op->tev) cudaEventDestroy(e);
  if (op->ev0) cudaEventDestroy(op->ev0);
  if (op->ev1) cudaEventDestroy(op->ev1);
  if (op->own_stream) cudaStreamDestroy(op->own_stream);
  delete op;
}

// Autotuner of the FP64 path: the tile width (32, 64 or 128 output columns)
// of each stage, timed on the operator's own matrices at three t-points
// (first, middle, last: the widest and narrowest bands) over scratch cubes;
// keyed on (device, input and output points per axis, t-points) in the tune
// cache.  Small cubes fill the GPU only with narrow tiles (121^3: 115 row
// tiles of 128 for 148 SMs).
static int tune_fp64(dage_op3d *op) {
  std::string key = tune_device_key() + "/op3d_fp64/";
  for (int d = 0; d < 3; ++d) key += std::to_string(op->nin[d]) + "x" + std::to_string(op->nout[d]) + ",";
  key += "P" + std::to_string(op->P);
  std::vector<int> v;
  if (tune_lookup(key, v) && v.size() == 3) {
    for (int d = 0; d < 3; ++d) op->tile_n[d] = v[d];
    return 0;
  }
  cudaStream_t s = op->stream;
  const int nix = op->nin[0], niy = op->nin[1], niz = op->nin[2];
  const int nox = op->nout[0], noy = op->nout[1], noz = op->nout[2];
  TmpBuf X, U, W, V;
  DAGE_TRY(X.alloc(sizeof(double) * (size_t)nix * niy * niz));
  DAGE_TRY(U.alloc(sizeof(double) * (size_t)niy * niz * nox));
  DAGE_TRY(W.alloc(sizeof(double) * (size_t)niz * nox * noy));
  DAGE_TRY(V.alloc(sizeof(double) * (size_t)nox * noy * noz));
  DAGE_CUDA_TRY(cudaMemsetAsync(X.ptr, 0, X.bytes, s));
  DAGE_CUDA_TRY(cudaMemsetAsync(U.ptr, 0, U.bytes, s));
  DAGE_CUDA_TRY(cudaMemsetAsync(W.ptr, 0, W.bytes, s));
  cudaEvent_t e0, e1;
  DAGE_CUDA_TRY(cudaEventCreate(&e0));
  DAGE_CUDA_TRY(cudaEventCreate(&e1));
  const size_t sT[3] = {(size_t)nox * nix, (size_t)noy * niy, (size_t)noz * niz};
  const double *in[3] = {X.as<double>(), U.as<double>(), W.as<double>()};
  double *outp[3] = {U.as<double>(), W.as<double>(), V.as<double>()};
  const int M[3] = {niy * niz, niz * nox, nox * noy}, N[3] = {nox, noy, noz}, K[3] = {nix, niy, niz};
  const int ps[3] = {0, op->P / 2, op->P - 1};
  int rc = 0;
  for (int d = 0; d < 3 && !rc; ++d) {
    float best = 1e30f;
    for (int tn : {32, 64, 128}) {
      auto run = [&](int p) {
        const int2 *band = op->band[op->Towner[d]].as<int2>() + (size_t)p * ceil_div(N[d], BN);
        return launch_stage_fp64(in[d], K[d], M[d], N[d], K[d], op->T(d) + sT[d] * p, K[d], outp[d],
                                 1.0, false, s, band, tn);
      };
      rc = run(ps[0]);  // warm-up
      if (!rc) rc = cudaEventRecord(e0, s) == cudaSuccess ? 0 : fail(DAGE_E_CUDA, "event");
      for (int i = 0; i < 3 && !rc; ++i) rc = run(ps[i]);
      if (rc) break;
      cudaEventRecord(e1, s);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best) {
        best = ms;
        op->tile_n[d] = tn;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  tune_store(key, {op->tile_n[0], op->tile_n[1], op->tile_n[2]});
  return 0;
}

static int apply_fp64(dage_op3d *op, const double *rho, double *V, bool accumulate) {
  cudaStream_t s = op->stream;
  const int nix = op->nin[0], niy = op->nin[1], niz = op->nin[2];
  const int nox = op->nout[0], noy = op->nout[1], noz = op->nout[2];
  DAGE_TRY(op->tmp1.alloc(sizeof(double) * (size_t)niy * niz * nox));
  DAGE_TRY(op->tmp2.alloc(sizeof(double) * (size_t)niz * nox * noy));
  double *U = op->tmp1.as<double>(), *W = op->tmp2.as<double>();
  const size_t sx = (size_t)nox * nix, sy = (size_t)noy * niy, sz = (size_t)noz * niz;
  auto band = [&](int d, int p) {
    return op->band[op->Towner[d]].as<int2>() + (size_t)p * ceil_div(op->nout[d], BN);
  };
  for (int p = 0; p < op->P; ++p) {
    int t = op->tmark_begin(0);
    DAGE_TRY(launch_stage_fp64(rho, nix, niy * niz, nox, nix, op->T(0) + sx * p, nix, U, 1.0,
                               false, s, band(0, p), op->tile_n[0]));
    op->tmark_end(t);
    t = op->tmark_begin(0);
    DAGE_TRY(launch_stage_fp64(U, niy, niz * nox, noy, niy, op->T(1) + sy * p, niy, W, 1.0,
                               false, s, band(1, p), op->tile_n[1]));
    op->tmark_end(t);
    t = op->tmark_begin(0);
    DAGE_TRY(launch_stage_fp64(W, niz, nox * noy, noz, niz, op->T(2) + sz * p, niz, V,
                               op->w[p], accumulate || p > 0, s, band(2, p), op->tile_n[2]));
    op->tmark_end(t);
  }
  return 0;
}

}  // namespace dage

using namespace dage;

int dage_op3d::tmark_begin(int kind) {
  if (!timing) return -1;
  const size_t slot = tq.size();
  while (tev.size() < 2 * (slot + 1)) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return -1;
    tev.push_back(e);
  }
  cudaEventRecord(tev[2 * slot], stream);
  tq.push_back({kind, (int)(2 * slot)});
  return (int)slot;
}

void dage_op3d::tmark_end(int slot) {
  if (slot < 0) return;
  cudaEventRecord(tev[tq[slot].second + 1], stream);
}

int dage_op3d::tcollect() {
  for (auto &q : tq) {
    float ms = 0.0f;
    DAGE_CUDA_TRY(cudaEventElapsedTime(&ms, tev[q.second], tev[q.second + 1]));
    t_ms[q.first] += ms;
    t_launches[q.first] += 1;
  }
  tq.clear();
  return 0;
}

extern "C" {

int dage_op3d_create(const dage_grid1d grid_in[3], const dage_grid1d grid_out[3],
                     const dage_quad *quad, int precision, dage_op3d **out) {
  clear_error();
  if (!out) return fail(DAGE_E_INVALID, "null output handle pointer");
  *out = nullptr;
  dage_op3d *op = new dage_op3d();
  int rc = create_impl(grid_in, grid_out, quad, precision, op);
  if (rc) {
    destroy_impl(op);
    return rc;
  }
  *out = op;
  return 0;
}

int dage_op3d_create_cached(const dage_grid1d grid_in[3], const dage_grid1d grid_out[3],
                            const dage_quad *quad, int precision, const char *cache_dir,
                            int *from_cache, dage_op3d **out) {
  clear_error();
  if (!out || !cache_dir || !*cache_dir) return fail(DAGE_E_INVALID, "null argument");
  *out = nullptr;
  dage_op3d *op = new dage_op3d();
  int rc = create_impl(grid_in, grid_out, quad, precision, op, cache_dir);
  if (rc) {
    destroy_impl(op);
    return rc;
  }
  if (from_cache) *from_cache = op->from_cache ? 1 : 0;
  *out = op;
  return 0;
}

int dage_op3d_tiles(const dage_op3d *op, int tile_n[3]) {
  if (!op || !tile_n) return fail(DAGE_E_INVALID, "null argument");
  for (int d = 0; d < 3; ++d) tile_n[d] = op->precision == DAGE_FP64 ? op->tile_n[d] : 128;
  return 0;
}

int dage_op3d_mixed_schedule(const dage_op3d *op, int *ring_stages, int *tpoint_group) {
  clear_error();
  if (!op || !ring_stages || !tpoint_group) return fail(DAGE_E_INVALID, "null argument");
  return mixed_schedule(op, ring_stages, tpoint_group);
}

int dage_op3d_destroy(dage_op3d *op) {
  clear_error();
  destroy_impl(op);
  return 0;
}

int dage_op3d_set_stream(dage_op3d *op, void *stream) {
  if (!op) return fail(DAGE_E_INVALID, "null handle");
  op->stream = stream ? (cudaStream_t)stream : op->own_stream;
  return 0;
}

int dage_op3d_set_weights(dage_op3d *op, int P, const double *w) {
  clear_error();
  if (!op || !w) return fail(DAGE_E_INVALID, "null argument");
  if (P != op->P) return fail(DAGE_E_INVALID, "expected %d weights, got %d", op->P, P);
  op->w.assign(w, w + P);
  DAGE_TRY(upload_weights(op));
  DAGE_CUDA_TRY(cudaStreamSynchronize(op->stream));
  return 0;
}

int dage_op3d_set_energy(dage_op3d *op, double energy) {
  if (!op) return fail(DAGE_E_INVALID, "null handle");
  const double two_over_sqrtpi = 2.0 / std::sqrt(std::acos(-1.0));
  std::vector<double> w(op->P);
  for (int p = 0; p < op->P; ++p) {
    double tw = op->tw[p];
    if (energy < -0.005) tw = tw * std::exp(2.0 * energy / (4.0 * (op->tp[p] * op->tp[p])));
    w[p] = two_over_sqrtpi * tw;
  }
  return dage_op3d_set_weights(op, op->P, w.data());
}

int dage_op3d_set_coda(dage_op3d *op, double coda) {
  if (!op) return fail(DAGE_E_INVALID, "null handle");
  op->coda = coda;
  return 0;
}

int dage_op3d_get_quadrature(const dage_op3d *op, int *P, double *tp, double *w) {
  if (!op) return fail(DAGE_E_INVALID, "null handle");
  if (P) *P = op->P;
  if (tp) std::memcpy(tp, op->tp.data(), sizeof(double) * op->P);
  if (w) std::memcpy(w, op->w.data(), sizeof(double) * op->P);
  return 0;
}

int dage_op3d_get_matrix(const dage_op3d *op, int axis, double *T_host) {
  clear_error();
  if (!op || !T_host || axis < 0 || axis > 2) return fail(DAGE_E_INVALID, "bad argument");
  const int ni = op->nin[axis], no = op->nout[axis];
  std::vector<double> tmp((size_t)op->P * ni * no);
  DAGE_CUDA_TRY(cudaMemcpy(tmp.data(), op->T(axis), sizeof(double) * tmp.size(),
                           cudaMemcpyDeviceToHost));
  // device layout T[p][i_out][j_in] -> host T(i_out, j_in, p) column-major
  for (int p = 0; p < op->P; ++p)
    for (int i = 0; i < no; ++i)
      for (int j = 0; j < ni; ++j)
        T_host[(size_t)p * no * ni + (size_t)j * no + i] = tmp[((size_t)p * no + i) * ni + j];
  return 0;
}

int dage_op3d_last_time_ms(const dage_op3d *op, float *ms) {
  if (!op || !ms) return fail(DAGE_E_INVALID, "null argument");
  *ms = op->last_ms;
  return 0;
}

namespace {
// Everything of one apply up to (not including) the wait for its stream.
int op3d_enqueue(dage_op3d *op, const double *rho, double *V, unsigned flags, double *energy) {
  if (!op || !rho || !V) return fail(DAGE_E_INVALID, "null argument");
  if ((flags & DAGE_ENERGY) && !energy) return fail(DAGE_E_INVALID, "energy pointer is null");
  DAGE_CUDA_TRY(cudaSetDevice(op->device));
  cudaStream_t s = op->stream;
  const size_t nin = (size_t)op->nin[0] * op->nin[1] * op->nin[2];
  const size_t nout = (size_t)op->nout[0] * op->nout[1] * op->nout[2];
  const bool dev = (flags & DAGE_DEVICE_PTRS) != 0;
  const bool acc = (flags & DAGE_ACCUMULATE) != 0;
  const double *d_rho = rho;
  double *d_V = V;
  DAGE_CUDA_TRY(cudaEventRecord(op->ev0, s));
  if (!dev) {
    DAGE_TRY(op->d_rho.alloc(sizeof(double) * nin));
    DAGE_TRY(op->d_V.alloc(sizeof(double) * nout));
    DAGE_CUDA_TRY(cudaMemcpyAsync(op->d_rho.ptr, rho, sizeof(double) * nin,
                                  cudaMemcpyHostToDevice, s));
    if (acc)
      DAGE_CUDA_TRY(cudaMemcpyAsync(op->d_V.ptr, V, sizeof(double) * nout,
                                    cudaMemcpyHostToDevice, s));
    d_rho = op->d_rho.as<double>();
    d_V = op->d_V.as<double>();
  }
  if (op->precision == DAGE_FP64) {
    DAGE_TRY(apply_fp64(op, d_rho, d_V, acc));
  } else {
    if (acc) return fail(DAGE_E_UNSUPPORTED, "DAGE_ACCUMULATE with a mixed operator");
    DAGE_TRY(mixed_apply(op, d_rho, d_V, s));
  }
  const bool coda = op->same_grid && op->coda != 0.0 && !(flags & DAGE_NO_CODA);
  double *d_res = (flags & DAGE_ENERGY) ? op->partials.as<double>() + finalize_partials_count()
                                        : nullptr;
  const int tf = op->tmark_begin(2);
  DAGE_TRY(launch_finalize(d_rho, d_V, coda ? d_rho : nullptr, op->coda, op->wts[0].as<double>(),
                           op->wts[1].as<double>(), op->wts[2].as<double>(), op->nout[0],
                           op->nout[1], op->nout[2], op->partials.as<double>(),
                           finalize_partials_count(), d_res, s));
  op->tmark_end(tf);
  if (!dev)
    DAGE_CUDA_TRY(cudaMemcpyAsync(V, d_V, sizeof(double) * nout, cudaMemcpyDeviceToHost, s));
  if (d_res) DAGE_CUDA_TRY(cudaMemcpyAsync(energy, d_res, sizeof(double), cudaMemcpyDeviceToHost, s));
  DAGE_CUDA_TRY(cudaEventRecord(op->ev1, s));
  return 0;
}

// Host-pointer applies through a pipeline: two device staging slots per
// operator and copy-in / copy-out streams beside the compute stream.  The
// copy-in into slot k waits for the compute that last read slot k, the
// compute for its copy-in and for the copy-out that last read slot k, the
// copy-out for the compute.  Each copy-in is issued two applies ahead, right
// after the compute that frees its slot, so it is queued before the next
// compute and runs beside it.  With pinned host memory the copies are
// asynchronous (a pageable array makes the host wait for its copy).
int pipe_open(dage_op3d *op) {
  DAGE_CUDA_TRY(cudaSetDevice(op->device));
  if (!op->pipe_h2d[0]) {
    for (int k = 0; k < 2; ++k)
      for (cudaEvent_t *e : {&op->pipe_h2d[k], &op->pipe_comp[k], &op->pipe_d2h[k]})
        DAGE_CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  }
  const size_t nin = (size_t)op->nin[0] * op->nin[1] * op->nin[2];
  const size_t nout = (size_t)op->nout[0] * op->nout[1] * op->nout[2];
  for (int k = 0; k < 2; ++k) {
    DAGE_TRY(op->pipe_rho[k].alloc(sizeof(double) * nin));
    DAGE_TRY(op->pipe_V[k].alloc(sizeof(double) * nout));
  }
  DAGE_CUDA_TRY(cudaEventRecord(op->ev0, op->pipe_in));
  op->pipe_open = true;
  return 0;
}

int pipe_copy_in(dage_op3d *op, int k, const double *rho, const double *V, bool acc) {
  const size_t nin = (size_t)op->nin[0] * op->nin[1] * op->nin[2];
  const size_t nout = (size_t)op->nout[0] * op->nout[1] * op->nout[2];
  DAGE_CUDA_TRY(cudaStreamWaitEvent(op->pipe_in, op->pipe_comp[k], 0));
  if (acc) DAGE_CUDA_TRY(cudaStreamWaitEvent(op->pipe_in, op->pipe_d2h[k], 0));
  DAGE_CUDA_TRY(cudaMemcpyAsync(op->pipe_rho[k].ptr, rho, sizeof(double) * nin,
                                cudaMemcpyHostToDevice, op->pipe_in));
  if (acc)
    DAGE_CUDA_TRY(cudaMemcpyAsync(op->pipe_V[k].ptr, V, sizeof(double) * nout,
                                  cudaMemcpyHostToDevice, op->pipe_in));
  DAGE_CUDA_TRY(cudaEventRecord(op->pipe_h2d[k], op->pipe_in));
  return 0;
}

// d_energy: device pointer (or null) for the apply's energy
int pipe_compute_out(dage_op3d *op, int k, double *V, unsigned flags, double *d_energy) {
  const size_t nout = (size_t)op->nout[0] * op->nout[1] * op->nout[2];
  const bool acc = (flags & DAGE_ACCUMULATE) != 0;
  double *d_rho = op->pipe_rho[k].as<double>(), *d_V = op->pipe_V[k].as<double>();
  cudaStream_t s = op->stream;
  DAGE_CUDA_TRY(cudaStreamWaitEvent(s, op->pipe_h2d[k], 0));
  DAGE_CUDA_TRY(cudaStreamWaitEvent(s, op->pipe_d2h[k], 0));
  if (op->precision == DAGE_FP64)
    DAGE_TRY(apply_fp64(op, d_rho, d_V, acc));
  else
    DAGE_TRY(mixed_enqueue(op, d_rho, d_V, s));
  const bool coda = op->same_grid && op->coda != 0.0 && !(flags & DAGE_NO_CODA);
  const int tf = op->tmark_begin(2);
  DAGE_TRY(launch_finalize(d_rho, d_V, coda ? d_rho : nullptr, op->coda, op->wts[0].as<double>(),
                           op->wts[1].as<double>(), op->wts[2].as<double>(), op->nout[0],
                           op->nout[1], op->nout[2], op->partials.as<double>(),
                           finalize_partials_count(), d_energy, s));
  op->tmark_end(tf);
  DAGE_CUDA_TRY(cudaEventRecord(op->pipe_comp[k], s));
  DAGE_CUDA_TRY(cudaStreamWaitEvent(op->pipe_out, op->pipe_comp[k], 0));
  DAGE_CUDA_TRY(cudaMemcpyAsync(V, d_V, sizeof(double) * nout, cudaMemcpyDeviceToHost,
                                op->pipe_out));
  DAGE_CUDA_TRY(cudaEventRecord(op->pipe_d2h[k], op->pipe_out));
  DAGE_CUDA_TRY(cudaEventRecord(op->ev1, op->pipe_out));
  return 0;
}

// The batch's host-pointer applies: per operator its applies in order,
// slot = position % 2; first copy-ins of every operator, then per apply
// its compute and copy-out followed by the copy-in two places later; then
// one wait per operator.  The energies stay on the device until the end: a
// copy into pageable host memory would block the host behind the copy-out
// queued before it.
int pipe_batch_enqueue(int n, dage_op3d *const *ops, const double *const *rho, double *const *V,
                       unsigned flags, double *d_energies) {
  const bool acc = (flags & DAGE_ACCUMULATE) != 0;
  std::vector<int> pos(n), later(n, -1);  // position in its operator's list; item 2 later
  std::vector<std::pair<dage_op3d *, std::vector<int>>> lists;
  for (int i = 0; i < n; ++i) {
    if (!ops[i] || !rho[i] || !V[i]) return fail(DAGE_E_INVALID, "null argument");
    if (acc && ops[i]->precision != DAGE_FP64)
      return fail(DAGE_E_UNSUPPORTED, "DAGE_ACCUMULATE with a mixed operator");
    size_t l = 0;
    while (l < lists.size() && lists[l].first != ops[i]) ++l;
    if (l == lists.size()) lists.push_back({ops[i], {}});
    std::vector<int> &v = lists[l].second;
    pos[i] = (int)v.size();
    if (v.size() >= 2) later[v[v.size() - 2]] = i;
    v.push_back(i);
  }
  for (auto &l : lists) DAGE_TRY(pipe_open(l.first));
  for (int i = 0; i < n; ++i)
    if (pos[i] < 2) DAGE_TRY(pipe_copy_in(ops[i], pos[i] & 1, rho[i], V[i], acc));
  for (int i = 0; i < n; ++i) {
    DAGE_TRY(pipe_compute_out(ops[i], pos[i] & 1, V[i], flags,
                              d_energies ? d_energies + i : nullptr));
    const int j = later[i];
    if (j >= 0) DAGE_TRY(pipe_copy_in(ops[j], pos[j] & 1, rho[j], V[j], acc));
  }
  return 0;
}

int op3d_pipe_finish(dage_op3d *op);

int pipe_batch(int n, dage_op3d *const *ops, const double *const *rho, double *const *V,
               unsigned flags, double *energies) {
  TmpBuf d_e;
  if ((flags & DAGE_ENERGY) && n > 0) DAGE_TRY(d_e.alloc(sizeof(double) * n));
  int rc = pipe_batch_enqueue(n, ops, rho, V, flags, d_e.as<double>());
  // one wait per distinct operator (also after a failed enqueue: nothing
  // queued is left running)
  for (int i = 0; i < n; ++i) {
    bool seen = false;
    for (int j = 0; j < i && !seen; ++j) seen = ops[j] == ops[i];
    if (seen || !ops[i] || !ops[i]->pipe_open) continue;
    const int r = op3d_pipe_finish(ops[i]);
    if (!rc) rc = r;
  }
  if (!rc && d_e.ptr)
    DAGE_CUDA_TRY(cudaMemcpy(energies, d_e.ptr, sizeof(double) * n, cudaMemcpyDeviceToHost));
  return rc;
}

int op3d_pipe_finish(dage_op3d *op) {
  DAGE_CUDA_TRY(cudaSetDevice(op->device));
  DAGE_CUDA_TRY(cudaStreamSynchronize(op->pipe_out));
  DAGE_CUDA_TRY(cudaStreamSynchronize(op->stream));
  DAGE_CUDA_TRY(cudaStreamSynchronize(op->pipe_in));
  op->pipe_open = false;
  DAGE_CUDA_TRY(cudaEventElapsedTime(&op->last_ms, op->ev0, op->ev1));
  DAGE_TRY(op->tcollect());
  if (op->precision != DAGE_FP64) DAGE_TRY(mixed_check(op, op->stream));
  return 0;
}

int op3d_finish(dage_op3d *op) {
  DAGE_CUDA_TRY(cudaSetDevice(op->device));
  DAGE_CUDA_TRY(cudaStreamSynchronize(op->stream));
  DAGE_CUDA_TRY(cudaEventElapsedTime(&op->last_ms, op->ev0, op->ev1));
  DAGE_TRY(op->tcollect());
  return 0;
}
}  // namespace

int dage_op3d_apply(dage_op3d *op, const double *rho, double *V, unsigned flags,
                    double *energy) {
  clear_error();
  DAGE_TRY(op3d_enqueue(op, rho, V, flags, energy));
  return op3d_finish(op);
}

int dage_op3d_apply_batched(int n, dage_op3d *const *ops, const double *const *rho,
                            double *const *V, unsigned flags, double *energies) {
  clear_error();
  if (n < 0 || (n > 0 && (!ops || !rho || !V))) return fail(DAGE_E_INVALID, "null argument");
  if ((flags & DAGE_ENERGY) && n > 0 && !energies)
    return fail(DAGE_E_INVALID, "energies pointer is null");
  // host pointers go through each operator's copy/compute pipeline
  if (!(flags & DAGE_DEVICE_PTRS)) return pipe_batch(n, ops, rho, V, flags, energies);
  int rc = 0;
  for (int i = 0; i < n && !rc; ++i)
    rc = op3d_enqueue(ops[i], rho[i], V[i], flags, energies ? energies + i : nullptr);
  // one wait per distinct operator, after everything is queued (also after
  // a failed enqueue: nothing queued is left running)
  for (int i = 0; i < n; ++i) {
    bool seen = false;
    for (int j = 0; j < i && !seen; ++j) seen = ops[j] == ops[i];
    if (seen || !ops[i]) continue;
    const int r = op3d_finish(ops[i]);
    if (!rc) rc = r;
  }
  return rc;
}

int dage_op3d_set_timing(dage_op3d *op, int enable) {
  if (!op) return fail(DAGE_E_INVALID, "null handle");
  op->timing = enable != 0;
  for (int k = 0; k < dage_op3d::kKinds; ++k) {
    op->t_launches[k] = 0;
    op->t_ms[k] = 0.0;
  }
  op->tq.clear();
  return 0;
}

int dage_op3d_get_timing(const dage_op3d *op, int kind, long long *launches, double *ms) {
  if (!op || kind < 0 || kind >= dage_op3d::kKinds) return fail(DAGE_E_INVALID, "bad argument");
  if (launches) *launches = op->t_launches[kind];
  if (ms) *ms = op->t_ms[kind];
  return 0;
}

int dage_integrate(const dage_grid1d grid[3], const double *f1, const double *f2,
                   unsigned flags, double *out) {
  clear_error();
  if (!grid || !f1 || !out) return fail(DAGE_E_INVALID, "null argument");
  Axis ax[3];
  for (int d = 0; d < 3; ++d) DAGE_TRY(make_axis(grid[d], ax[d]));
  const size_t n = (size_t)ax[0].n() * ax[1].n() * ax[2].n();
  const bool dev = (flags & DAGE_DEVICE_PTRS) != 0;
  TmpBuf w[3], b1, b2, part;
  for (int d = 0; d < 3; ++d) {
    DAGE_TRY(w[d].alloc(sizeof(double) * ax[d].n()));
    DAGE_CUDA_TRY(cudaMemcpy(w[d].ptr, ax[d].weights.data(), sizeof(double) * ax[d].n(),
                             cudaMemcpyHostToDevice));
  }
  const double *d1 = f1;
  double *d2 = const_cast<double *>(f2);
  if (!dev) {
    DAGE_TRY(b1.alloc(sizeof(double) * n));
    DAGE_CUDA_TRY(cudaMemcpy(b1.ptr, f1, sizeof(double) * n, cudaMemcpyHostToDevice));
    d1 = b1.as<double>();
    if (f2) {
      DAGE_TRY(b2.alloc(sizeof(double) * n));
      DAGE_CUDA_TRY(cudaMemcpy(b2.ptr, f2, sizeof(double) * n, cudaMemcpyHostToDevice));
      d2 = b2.as<double>();
    }
  }
  DAGE_TRY(part.alloc(sizeof(double) * (finalize_partials_count() + 1)));
  double *res = part.as<double>() + finalize_partials_count();
  DAGE_TRY(launch_finalize(d1, d2, nullptr, 0.0, w[0].as<double>(), w[1].as<double>(),
                           w[2].as<double>(), ax[0].n(), ax[1].n(), ax[2].n(),
                           part.as<double>(), finalize_partials_count(), res, 0));
  DAGE_CUDA_TRY(cudaMemcpy(out, res, sizeof(double), cudaMemcpyDeviceToHost));
  return 0;
}

}  // extern "C"
