// gbfmm.cu -- grid-based fast multipole (GBFMM) Coulomb operator on one B200.
//
// The cube is split into an octree level of 2^L boxes per axis (L = maxlevel,
// default 2: 4x4x4 boxes).  For every box b:
//   near field  V(b's points) = sub-operator(rho on b + its 26 neighbours):
//               the tensor-product operator restricted to those input cells
//               and b's output points, FP64, batched over all boxes in one
//               launch per contraction stage and t-point;
//   multipoles  q_lm(b) = sum_{r in b} rho w S_lm(r - c_b)   (FP64);
//   M2L         L(b) = sum_{j in far(b)} T(c_j - c_b) q(j)    (FP64, the
//               interaction matrices of the distinct box displacements are
//               built once on the GPU);
//   L2P         V(r) += sum_lm L_lm(b) S_lm(r - c_b) over b's points.
// Each grid point belongs to one box (a box's last point along an axis
// belongs to the next box unless it is the last grid point), as in the
// reference's CUDA path (src/gbfmm/gbfmm_coulomb3d.cu:478-573,
// gbfmm_coulomb3d.F90:1000-1030).  S_lm are Racah-normalised real regular
// solid harmonics (src/bubbles/harmonics.F90:586-658); the M2L matrices
// follow src/bubbles/multipole.F90:81-303.
//
// Box split.  Boxes get ncell / 2^L cells per axis when that divides; when
// it does not, the first (ncell mod 2^L) boxes along the axis get one extra
// cell (the reference's integer division would leave the trailing cells in
// no box).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <array>
#include <limits>
#include <map>
#include <mutex>
#include <vector>

#include "fp64_stage.cuh"
#include "near_mixed.cuh"
#include "tune.h"
#include "op3d.cuh"

struct dage_gbfmm;

namespace dage {

namespace {

constexpr int kMaxLmax = 15;

// ---------------------------------------------------------------------------
// Real regular solid harmonics by recursion, visiting every (l, m) once.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ int lmi(int l, int m) { return l * (l + 1) + m; }

template <class F>
__host__ __device__ __forceinline__ void solid_harmonics(int lmax, double x, double y, double z,
                                                         F &&f) {
  const double r2 = x * x + y * y + z * z;
  f(0, 1.0);
  if (lmax == 0) return;
  {  // m = 0
    double p2 = 1.0, p1 = z;
    f(lmi(1, 0), z);
    for (int l = 2; l <= lmax; ++l) {
      double cur = (2.0 * l - 1.0) / sqrt((double)(l * l)) * (z * p1);
      cur = cur - sqrt((double)((l - 1) * (l - 1)) / (double)(l * l)) * (r2 * p2);
      f(lmi(l, 0), cur);
      p2 = p1;
      p1 = cur;
    }
  }
  double top = x, bot = y;  // S_{m,m}, S_{m,-m}
  for (int mm = 1; mm <= lmax; ++mm) {
    if (mm >= 2) {
      const double c = sqrt((2.0 * mm - 1.0) / (2.0 * mm));
      const double nb = c * (y * top + x * bot);
      const double nt = c * (x * top - y * bot);
      top = nt;
      bot = nb;
    }
    f(lmi(mm, mm), top);
    f(lmi(mm, -mm), bot);
#pragma unroll 1
    for (int sgn = 0; sgn < 2; ++sgn) {
      const int m = sgn ? -mm : mm;
      double p2 = 0.0, p1 = sgn ? bot : top;
      for (int l = mm + 1; l <= lmax; ++l) {
        double cur = (2.0 * l - 1.0) / sqrt((double)((l + m) * (l - m))) * (z * p1);
        if (l > mm + 1)
          cur = cur - sqrt((double)((l + m - 1) * (l - m - 1)) / (double)((l + m) * (l - m))) *
                          (r2 * p2);
        f(lmi(l, m), cur);
        p2 = p1;
        p1 = cur;
      }
    }
  }
}

struct BoxInfo {
  int p0[3], np[3];     // box sub-grid points (global index, count)
  int own[3];           // owned points (from p0) per axis
  int q0[3], nq[3];     // near-field region points
  int pos[3];           // box position along each axis
  double c[3];          // expansion centre
};

// One density of a batch (a batch of one for dage_gbfmm_apply): its cubes,
// its expansion buffers, and the tables of the plan (grid geometry) it
// shares with every density on the same grid.
struct GInst {
  const double *rho;
  double *V;
  double *q, *L, *partial;  // moments, local expansions (nbox x N), slab sums
  double *epart;            // energy partial sums [kEnergyBlocks]
  const BoxInfo *boxes;     // plan: nbox boxes
  const double *wbox;       // plan: per-position box weights, then coordinates
  int wstride, Nx, Ny, Nz;
  const double *Tm2l;       // plan: M2L matrix per displacement
  const int *ffstart, *ffsrc, *ffdisp;  // plan: far-field lists
  const double *wx, *wy, *wz;           // plan: full-grid integration weights
  double kappa;  // 0: Coulomb; > 0: Helmholtz kernel e^(-kappa r)/r
  // levels: q and L hold every box of levels 2..maxlevel (level 2 first);
  // the finest level starts at box fine_off.  M2M/L2L: translation matrix
  // (packed lower triangle) of box g's displacement from its parent,
  // Wm2m + m2m_disp[g - m2m_base] * Wsize, for boxes of levels >= 3
  int fine_off, m2m_base;
  const double *Wm2m;
  const int *m2m_disp;
  // Helmholtz instances: dense N x N translation matrix per displacement
  // (column k = input lm), Wm2m_h + m2m_disp[g - m2m_base] * N * N
  const double *Wm2m_h;
};

constexpr int kEnergyBlocks = 148 * 6;  // partial sums per density (6 blocks per SM)

// ---------------------------------------------------------------------------
// Modified spherical Bessel functions of the first kind, as the ratios
// f_l(x) = i_l(x) / x^l (finite at x = 0, f_l(0) = 1/(2l+1)!!), l = 0..L:
// the series sum_k (x^2/2)^k / (k! (2l+3)(2l+5)..(2l+2k+1)) / (2l+1)!! for
// l = L and L-1 (positive terms, no cancellation) and the downward
// recursion f_l = (2l+3) f_{l+1} + x^2 f_{l+2} (from i_l = (2l+3)/x i_{l+1}
// + i_{l+2}, src/bubbles/helmholtz3d.F90:879-971; all terms positive).
// ---------------------------------------------------------------------------
// Series terms use tabulated reciprocals 1/(k (2n+2k+1)) (k <= kRcK) and
// 1/(2n+1)!! in place of divisions; uploaded with the harmonic tables.
constexpr int kRcK = 128;
__device__ double d_rc[(kRcK + 1) * 16];
__constant__ double c_dfinv[16];

__device__ __forceinline__ double bessel_ratio_series(double x2h, int n) {
  double term = 1.0, sum = 1.0;
  for (int k = 1; k < 400; ++k) {
    const double rc = k <= kRcK ? d_rc[k * 16 + n] : 1.0 / (k * (2.0 * n + 2 * k + 1));
    term *= x2h * rc;
    sum += term;
    if (term < 1e-17 * sum) break;
  }
  return sum * c_dfinv[n];
}

__device__ __forceinline__ void bessel_ratios(double x, int L, double *f) {
  const double x2 = x * x;
  f[L] = bessel_ratio_series(0.5 * x2, L);
  if (L >= 1) f[L - 1] = bessel_ratio_series(0.5 * x2, L - 1);
  for (int l = L - 2; l >= 0; --l) f[l] = (2 * l + 3) * f[l + 1] + x2 * f[l + 2];
}

// ---------------------------------------------------------------------------
// Recurrence coefficients of solid_harmonics as tables (the same expressions,
// evaluated once on the host, so the values are bit-identical):
//   S_lm = A_lm z S_{l-1,m} - B_lm r^2 S_{l-2,m}    (l > |m|)
//   S_{m,m} = C_m (x S_{m-1,m-1} - y S_{m-1,-(m-1)}) etc. (m >= 2)
// ---------------------------------------------------------------------------
constexpr int kShSize = (kMaxLmax + 1) * (kMaxLmax + 1);
__constant__ double c_shA[kShSize];
__constant__ double c_shB[kShSize];
__constant__ double c_shC[kMaxLmax + 1];

// Uploads the tables to the current device once per process and device
// (called at plan creation, outside any stream capture).
int sh_tables_init() {
  static std::mutex mu;
  static unsigned long long done = 0;  // one bit per device ordinal
  int dev = 0;
  DAGE_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (dev < 64 && (done >> dev) & 1ull) return 0;
  double A[kShSize] = {}, B[kShSize] = {}, C[kMaxLmax + 1] = {};
  for (int l = 1; l <= kMaxLmax; ++l)
    for (int m = -(l - 1); m <= l - 1; ++m) {
      A[lmi(l, m)] = (2.0 * l - 1.0) / sqrt((double)((l + m) * (l - m)));
      B[lmi(l, m)] = sqrt((double)((l + m - 1) * (l - m - 1)) / (double)((l + m) * (l - m)));
    }
  for (int mm = 2; mm <= kMaxLmax; ++mm) C[mm] = sqrt((2.0 * mm - 1.0) / (2.0 * mm));
  DAGE_CUDA_TRY(cudaMemcpyToSymbol(c_shA, A, sizeof(A)));
  DAGE_CUDA_TRY(cudaMemcpyToSymbol(c_shB, B, sizeof(B)));
  DAGE_CUDA_TRY(cudaMemcpyToSymbol(c_shC, C, sizeof(C)));
  std::vector<double> rc((kRcK + 1) * 16, 0.0);
  for (int k = 1; k <= kRcK; ++k)
    for (int n = 0; n < 16; ++n) rc[k * 16 + n] = 1.0 / (k * (2.0 * n + 2 * k + 1));
  double dfinv[16];
  for (int n = 0; n < 16; ++n) {
    double df = 1.0;  // (2n+1)!!
    for (int i = 3; i <= 2 * n + 1; i += 2) df *= i;
    dfinv[n] = 1.0 / df;
  }
  DAGE_CUDA_TRY(cudaMemcpyToSymbol(d_rc, rc.data(), sizeof(double) * rc.size()));
  DAGE_CUDA_TRY(cudaMemcpyToSymbol(c_dfinv, dfinv, sizeof(dfinv)));
  // These copies come from pageable memory on the legacy stream: they may
  // return before the DMA lands, and the kernels that read the tables run on
  // non-blocking streams, which are not ordered after the legacy stream.
  // Without this wait a kernel could read zeros (a Bessel series cut to its
  // leading term, harmonics of zero).
  DAGE_CUDA_TRY(cudaDeviceSynchronize());
  if (dev < 64) done |= 1ull << dev;
  return 0;
}

// solid_harmonics with the coefficient tables (every lane of a warp visits
// the same (l, m) sequence, so the constant-bank reads are uniform).
template <class F>
__device__ __forceinline__ void solid_harmonics_tab(int lmax, double x, double y, double z, F &&f) {
  const double r2 = x * x + y * y + z * z;
  f(0, 1.0);
  if (lmax == 0) return;
  {
    double p2 = 0.0, p1 = 1.0;
    for (int l = 1; l <= lmax; ++l) {
      const double cur = c_shA[lmi(l, 0)] * (z * p1) - c_shB[lmi(l, 0)] * (r2 * p2);
      f(lmi(l, 0), cur);
      p2 = p1;
      p1 = cur;
    }
  }
  double top = x, bot = y;
  for (int mm = 1; mm <= lmax; ++mm) {
    if (mm >= 2) {
      const double c = c_shC[mm];
      const double nb = c * (y * top + x * bot);
      const double nt = c * (x * top - y * bot);
      top = nt;
      bot = nb;
    }
    f(lmi(mm, mm), top);
    f(lmi(mm, -mm), bot);
#pragma unroll 1
    for (int sgn = 0; sgn < 2; ++sgn) {
      const int m = sgn ? -mm : mm;
      double p2 = 0.0, p1 = sgn ? bot : top;
      for (int l = mm + 1; l <= lmax; ++l) {
        const double cur = c_shA[lmi(l, m)] * (z * p1) - c_shB[lmi(l, m)] * (r2 * p2);
        f(lmi(l, m), cur);
        p2 = p1;
        p1 = cur;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Multipole moments q_lm(b) = sum rho w S_lm (Helmholtz: i_l(kappa r) Y_lm).
//
// The (lmax+1)^2 harmonics of a point are split into lmax+1 lane tasks of
// lmax+1 values each: task 0 is the m = 0 chain (l = 0..lmax); the others
// pair the chain of m = +-mm (l = mm..lmax, lmax+1-mm values) with the
// chain of m = +-(lmax+1-mm) of the same sign (mm values); for odd lmax the
// chains m = +h and m = -h, h = (lmax+1)/2, form the last task.  A warp
// evaluates PP = 32/(lmax+1) points at a time, lane p(lmax+1)+t running task
// t for point p, each lane keeping its lmax+1 sums in registers.  Warps walk
// columns of the box (PP neighbouring x, one y, every z); at the end the
// block sums its lanes in a fixed order into one partial per (box, slab).
// ---------------------------------------------------------------------------
constexpr int kMpWarps = 8;

// chains of task t: signed m of the first and second chain (task 0: the
// m = 0 chain alone, m2 unused) and the first chain's length
__device__ __forceinline__ void mp_task(int L, int t, int &m1, int &m2, int &len1) {
  const int h = L / 2;
  if (t == 0) {
    m1 = 0;
    m2 = 0;
    len1 = L + 1;
    return;
  }
  if (t <= h) {
    m1 = t;
    m2 = L + 1 - t;
  } else if (t <= 2 * h) {
    m1 = -(t - h);
    m2 = -(L + 1 - (t - h));
  } else {
    m1 = (L + 1) / 2;
    m2 = -m1;
  }
  len1 = L + 1 - abs(m1);
}

// (l, m) of step k of task t
__device__ __forceinline__ void mp_step(int L, int t, int k, int &l, int &m) {
  int m1, m2, len1;
  mp_task(L, t, m1, m2, len1);
  if (k < len1) {
    m = m1;
    l = abs(m1) + k;
  } else {
    m = m2;
    l = abs(m2) + k - len1;
  }
}

template <bool HELM>
__global__ void __launch_bounds__(kMpWarps * 32, HELM ? 2 : 3)
    multipoles_kernel(const GInst *__restrict__ insts, int lmax, int nslab) {
  __shared__ double sA[16 * 16], sB[16 * 16];  // [k][t]
  __shared__ double red[kMpWarps][32][17];
  const GInst &I = insts[blockIdx.z];
  const int L = lmax, L1 = lmax + 1;
  const int PP = 32 / L1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int e = threadIdx.x; e < L1 * L1; e += blockDim.x) {
    const int t = e / L1, k = e % L1;
    int l, m;
    mp_step(L, t, k, l, m);
    const bool start = l == abs(m);
    sA[k * 16 + t] = start ? 0.0 : c_shA[lmi(l, m)];
    sB[k * 16 + t] = start ? 0.0 : c_shB[lmi(l, m)];
  }
  __syncthreads();
  const int p = lane / L1, t = lane % L1;
  int m1, m2, len1;
  mp_task(L, t, m1, m2, len1);
  const int a1 = abs(m1), a2 = abs(m2), amax = t == 0 ? 0 : max(a1, a2);
  const bool helm = HELM && I.kappa > 0.0;  // a batch may mix kernels
  const BoxInfo b = I.boxes[blockIdx.x];
  const int ws = I.wstride;
  const double *wx = I.wbox + (0 * 64 + b.pos[0]) * ws;
  const double *wy = I.wbox + (1 * 64 + b.pos[1]) * ws;
  const double *wz = I.wbox + (2 * 64 + b.pos[2]) * ws;
  const double *xs = I.wbox + (3 * 64) * ws;  // point coordinates per axis
  const size_t plane = (size_t)I.Nx * I.Ny;

  double acc[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) acc[k] = 0.0;

  const int nib = (b.np[0] + PP - 1) / PP;
  const int nbund = nib * b.np[1];
  for (int u = blockIdx.y * kMpWarps + warp; u < nbund; u += nslab * kMpWarps) {
    const int j = u / nib, i = (u % nib) * PP + p;
    const bool valid = p < PP && i < b.np[0];
    const int ii = valid ? i : 0;
    const double x = xs[b.p0[0] + ii] - b.c[0];
    const double y = xs[ws + b.p0[1] + j] - b.c[1];
    const double wxy = valid ? wx[ii] * wy[j] : 0.0;
    // chain starts S_{a1,+-a1}, S_{a2,+-a2} (task 0: S_00 = 1)
    double s1 = 1.0, s2 = 0.0;
    {
      double top = x, bot = y;
      for (int mm = 1; mm <= amax; ++mm) {
        if (mm >= 2) {
          const double c = c_shC[mm];
          const double nb = c * (y * top + x * bot);
          const double nt = c * (x * top - y * bot);
          top = nt;
          bot = nb;
        }
        if (mm == a1) s1 = m1 > 0 ? top : bot;
        if (mm == a2) s2 = m2 > 0 ? top : bot;
      }
    }
    const double *rcol = I.rho + (size_t)(b.p0[0] + ii) + (size_t)I.Nx * (b.p0[1] + j) +
                         plane * b.p0[2];
    // Helmholtz: i_l(kappa r) Y_lm(rhat) = kappa^l f_l(kappa r) S_lm(r).  The
    // factors g_l = kappa^l f_l of the bundle's next CZ z values of each of
    // its PP columns come first, one lane per point (series for L and L - 1,
    // downward recursion), into this warp's rows of `red` (free until the
    // final reduction).
    if constexpr (!HELM) {
      for (int kz = 0; kz < b.np[2]; ++kz) {
        const double v = valid ? rcol[plane * kz] * (wxy * wz[kz]) : 0.0;
        const double z = xs[2 * ws + b.p0[2] + kz] - b.c[2];
        const double r2 = x * x + y * y + z * z;
        double p1 = 0.0, p2 = 0.0;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          if (k > L) break;
          const bool st = k == 0 || k == len1;
          const double rec = sA[k * 16 + t] * (z * p1) - sB[k * 16 + t] * (r2 * p2);
          const double cur = st ? (k == 0 ? s1 : s2) : rec;
          p2 = st ? 0.0 : p1;
          p1 = cur;
          acc[k] += v * cur;
        }
      }
      continue;
    }
    const int CZ = 32 / PP;
    const int pi = p < PP ? p : 0;
    for (int kz0 = 0; kz0 < b.np[2]; kz0 += CZ) {
      if (helm) {
        const int ic = min((u % nib) * PP + lane / CZ, b.np[0] - 1);
        const int kc = min(kz0 + lane % CZ, b.np[2] - 1);
        const double xc = xs[b.p0[0] + ic] - b.c[0], zc = xs[2 * ws + b.p0[2] + kc] - b.c[2];
        const double x2 = (I.kappa * I.kappa) * (xc * xc + y * y + zc * zc);
        double *g = red[warp][lane];
        g[L] = bessel_ratio_series(0.5 * x2, L);
        if (L >= 1) g[L - 1] = bessel_ratio_series(0.5 * x2, L - 1);
        for (int l = L - 2; l >= 0; --l) g[l] = (2 * l + 3) * g[l + 1] + x2 * g[l + 2];
        double kp = 1.0;
        for (int l = 0; l <= L; ++l) {
          g[l] *= kp;
          kp *= I.kappa;
        }
        __syncwarp();
      }
      const int kzend = min(kz0 + CZ, b.np[2]);
      for (int kz = kz0; kz < kzend; ++kz) {
        const double v = valid ? rcol[plane * kz] * (wxy * wz[kz]) : 0.0;
        const double z = xs[2 * ws + b.p0[2] + kz] - b.c[2];
        const double r2 = x * x + y * y + z * z;
        const double *gp = red[warp][pi * CZ + (kz - kz0)];
        double p1 = 0.0, p2 = 0.0;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          if (k > L) break;
          const bool st = k == 0 || k == len1;
          const double rec = sA[k * 16 + t] * (z * p1) - sB[k * 16 + t] * (r2 * p2);
          const double cur = st ? (k == 0 ? s1 : s2) : rec;
          p2 = st ? 0.0 : p1;
          p1 = cur;
          const double f = helm ? v * gp[k < len1 ? a1 + k : a2 + k - len1] : v;
          acc[k] += f * cur;
        }
      }
      // Required before the next chunk's factors overwrite `red` and before
      // the final store below overwrites it with this lane's sums: every
      // lane of the warp must be done reading the factor rows.
      if (helm) __syncwarp();
    }
  }
  // (Helmholtz: ordered after the last reads of the factor rows by the
  // __syncwarp at the end of the chunk loop above.)
#pragma unroll
  for (int k = 0; k < 16; ++k)
    if (k <= L) red[warp][lane][k] = acc[k];
  __syncthreads();
  const int N = L1 * L1;
  for (int e = threadIdx.x; e < N; e += blockDim.x) {
    const int tt = e / L1, k = e % L1;
    int l, m;
    mp_step(L, tt, k, l, m);
    double sum = 0.0;
    for (int w = 0; w < kMpWarps; ++w)
      for (int pp = 0; pp < PP; ++pp) sum += red[w][pp * L1 + tt][k];
    I.partial[((size_t)blockIdx.x * nslab + blockIdx.y) * N + lmi(l, m)] = sum;
  }
}

// q(box, lm) = sum over slabs, fixed order; grid (., density)
__global__ void reduce_slabs_kernel(const GInst *__restrict__ insts, int nslab, int N, int nbox) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nbox * N) return;
  const GInst &I = insts[blockIdx.y];
  const int b = idx / N, s = idx % N;
  double acc = 0.0;
  for (int k = 0; k < nslab; ++k) acc += I.partial[((size_t)b * nslab + k) * N + s];
  I.q[(size_t)(I.fine_off + b) * N + s] = acc;
}

// ---------------------------------------------------------------------------
// M2L matrices of the distinct displacements (multipole.F90:265-303):
//   I_lm(d) = S_lm(d) / |d|^(2l+1), l <= 2 lmax
//   T(i, s) = c1 I[lm1] + c2 I[lm2] (i >= s),  T(s, i) = (-1)^(l_i - l_s) T(i, s)
// stored column-major, T[s*N + i], so a warp reading one column is coalesced.
// ---------------------------------------------------------------------------
__global__ void m2l_matrices_kernel(const double *__restrict__ disp, int lmax,
                                    const double *__restrict__ c1, const double *__restrict__ c2,
                                    const int *__restrict__ lm1, const int *__restrict__ lm2,
                                    const int *__restrict__ prow, const int *__restrict__ pcol,
                                    double *Tall) {
  extern __shared__ double I[];
  const int L2 = 2 * lmax;
  const int NI = (L2 + 1) * (L2 + 1);
  const int N = (lmax + 1) * (lmax + 1);
  const int M = N * (N + 1) / 2;
  const double *d = disp + 3 * blockIdx.x;
  if (threadIdx.x == 0) solid_harmonics(L2, d[0], d[1], d[2], [&](int lm, double s) { I[lm] = s; });
  __syncthreads();
  const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  for (int lm = threadIdx.x; lm < NI; lm += blockDim.x) {
    int l = (int)sqrt((double)lm);
    while ((l + 1) * (l + 1) <= lm) ++l;
    while (l * l > lm) --l;
    double rp = 1.0;
    for (int e = 0; e < 2 * l + 1; ++e) rp *= r;
    I[lm] = I[lm] / rp;
  }
  __syncthreads();
  double *T = Tall + (size_t)blockIdx.x * N * N;
  for (int e = threadIdx.x; e < M; e += blockDim.x) {
    const int i = prow[e], s = pcol[e];  // 0-based row (l,m) >= column (j,k)
    const double w = c1[e] * I[lm1[e]] + c2[e] * I[lm2[e]];
    int li = (int)sqrt((double)i), ls = (int)sqrt((double)s);
    while ((li + 1) * (li + 1) <= i) ++li;
    while (li * li > i) --li;
    while ((ls + 1) * (ls + 1) <= s) ++ls;
    while (ls * ls > s) --ls;
    T[(size_t)s * N + i] = w;
    T[(size_t)i * N + s] = ((li - ls) & 1) ? -w : w;
  }
}

// Helmholtz M2L matrices (src/bubbles/helmholtz_multipole_tools.F90:172-278:
// Racah -> orthonormal scaling, rotation to the translation axis, coaxial
// translation, rotation back, orthonormal -> Racah):
//   T[(n,m') -> (l,m)] = s_out(l) sum_mu R_l[mu][m] C(l, n, |mu|) R_n[mu][m'] s_in(n)
// with per-displacement rotation blocks R (rblk doubles each, block l at
// roff(l)) and coaxial coefficients C[(l (L+1) + n) (L+1) + m].  Stored like
// the Coulomb matrices, T[k N + i] (column k = input (n,m')).
__global__ void helm_m2l_matrices_kernel(const double *__restrict__ R, int rblk,
                                         const double *__restrict__ C, int L, double *Tall) {
  const int N = (L + 1) * (L + 1);
  const double *Rd = R + (size_t)blockIdx.x * rblk;
  const double *Cd = C + (size_t)blockIdx.x * (L + 1) * (L + 1) * (L + 1);
  double *T = Tall + (size_t)blockIdx.x * N * N;
  const double four_pi = 4.0 * 3.141592653589793238;
  for (int e = threadIdx.x; e < N * N; e += blockDim.x) {
    const int k = e / N, i = e % N;
    int l = (int)sqrtf((float)i + 0.5f), n = (int)sqrtf((float)k + 0.5f);
    const int m = i - l * (l + 1), mp = k - n * (n + 1);
    const int roff_l = (2 * l - 1) * l * (2 * l + 1) / 3, roff_n = (2 * n - 1) * n * (2 * n + 1) / 3;
    const int wl = 2 * l + 1, wn = 2 * n + 1;
    const int mu_max = l < n ? l : n;
    double acc = 0.0;
    for (int mu = -mu_max; mu <= mu_max; ++mu)
      acc += Rd[roff_l + (mu + l) * wl + (m + l)] * Cd[((size_t)l * (L + 1) + n) * (L + 1) + abs(mu)] *
             Rd[roff_n + (mu + n) * wn + (mp + n)];
    T[(size_t)k * N + i] = sqrt(four_pi / (2 * l + 1)) * acc * sqrt((2 * n + 1) / four_pi);
  }
}

// L(b) = sum over the far field of b of T(disp) q(src); block (box, density).
// G = blockDim.x / npad thread groups of npad (N rounded up to warps)
// threads share a target box: group h takes the sources e = start + h,
// start + h + G, ... and the groups' sums are added in group order
// (deterministic).
__global__ void m2l_apply_kernel(const GInst *__restrict__ insts, int N, int npad) {
  extern __shared__ double qs[];  // [G][N] sources, then [G][N] sums
  const GInst &I = insts[blockIdx.y];
  const int b = blockIdx.x;
  const int kM2LGroups = blockDim.x / npad;
  const int h = threadIdx.x / npad, i = threadIdx.x % npad;
  double *q = qs + (size_t)h * N;
  double acc = 0.0;
  const int e0 = I.ffstart[b], e1 = I.ffstart[b + 1];
  for (int base = e0; base < e1; base += kM2LGroups) {
    const int e = base + h;
    __syncthreads();
    if (e < e1)
      for (int k = i; k < N; k += npad) q[k] = I.q[(size_t)I.ffsrc[e] * N + k];
    __syncthreads();
    if (e < e1 && i < N) {
      const double *T = I.Tm2l + (size_t)I.ffdisp[e] * N * N;
      for (int k = 0; k < N; ++k) acc += T[(size_t)k * N + i] * q[k];
    }
  }
  double *sums = qs + (size_t)kM2LGroups * N;
  if (i < N) sums[(size_t)h * N + i] = acc;
  __syncthreads();
  if (h == 0 && i < N) {
    double t = sums[i];
    for (int g = 1; g < kM2LGroups; ++g) t += sums[(size_t)g * N + i];
    I.L[(size_t)b * N + i] = t;
  }
}

// Translation matrices W(d) of the distinct child-to-parent displacements
// (TranslationMatrix_eval, multipole.F90:443-476): packed lower triangle,
// column by column, W[r] = c1[r] S[lm1[r]] + c2[r] S[lm2[r]] (absent: -1).
__global__ void translation_matrices_kernel(const double *__restrict__ disp, int lmax,
                                            const double *__restrict__ c1,
                                            const double *__restrict__ c2,
                                            const int *__restrict__ lm1,
                                            const int *__restrict__ lm2, int M, double *Wall) {
  extern __shared__ double S[];
  const double *d = disp + 3 * blockIdx.x;
  if (threadIdx.x == 0) solid_harmonics(lmax, d[0], d[1], d[2], [&](int lm, double v) { S[lm] = v; });
  __syncthreads();
  double *W = Wall + (size_t)blockIdx.x * M;
  for (int r = threadIdx.x; r < M; r += blockDim.x) {
    double w = 0.0;
    if (lm1[r] >= 0) w = c1[r] * S[lm1[r]];
    if (lm2[r] >= 0) w = w + c2[r] * S[lm2[r]];
    W[r] = w;
  }
}

// packed (column-major lower) position of W(i, j), i >= j
__device__ __forceinline__ size_t wpos(int i, int j, int N) {
  return (size_t)j * N - (size_t)j * (j - 1) / 2 + (i - j);
}

// Upward pass, one level: q(parent) = sum over the 8 children c of
// W(c_c - c_parent) q(c), W applied with a unit diagonal (dtpmv 'L','N','U',
// gbfmm_coulomb3d.F90:1502-1562).  Block (parent, density); parents of this
// level start at box `poff`, their children at `coff` (children of parent p
// are coff + 8 p .. +7).
__global__ void m2m_kernel(const GInst *__restrict__ insts, int N, int poff, int coff) {
  const GInst &I = insts[blockIdx.y];
  const int p = blockIdx.x;
  if (I.kappa > 0.0) {
    // Helmholtz: the dense translation of the regular basis i_l Y_lm
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
      double acc = 0.0;
      for (int c = 0; c < 8; ++c) {
        const int gc = coff + 8 * p + c;
        const double *qc = I.q + (size_t)gc * N;
        const double *W = I.Wm2m_h + (size_t)I.m2m_disp[gc - I.m2m_base] * N * N;
        for (int j = 0; j < N; ++j) acc += W[(size_t)j * N + i] * qc[j];
      }
      I.q[(size_t)(poff + p) * N + i] = acc;
    }
    return;
  }
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    double acc = 0.0;
    for (int c = 0; c < 8; ++c) {
      const int gc = coff + 8 * p + c;
      const double *qc = I.q + (size_t)gc * N;
      const double *W = I.Wm2m + (size_t)I.m2m_disp[gc - I.m2m_base] * ((size_t)N * (N + 1) / 2);
      double t = qc[i];
      for (int j = 0; j < i; ++j) t += W[wpos(i, j, N)] * qc[j];
      acc += t;
    }
    I.q[(size_t)(poff + p) * N + i] = acc;
  }
}

// Downward pass, one level: L(child) += W(c_child - c_parent)^T L(parent)
// with a unit diagonal (translate_potential, gbfmm_coulomb3d.F90:1565-1621).
// Block (child, density); children of this level start at box `coff`,
// their parents at `poff`.
__global__ void l2l_kernel(const GInst *__restrict__ insts, int N, int poff, int coff) {
  const GInst &I = insts[blockIdx.y];
  const int c = blockIdx.x, gc = coff + c;
  const double *Lp = I.L + (size_t)(poff + c / 8) * N;
  if (I.kappa > 0.0) {
    // Helmholtz: the local expansion multiplies (2l+1) i_l Y_lm and the
    // moments i_l Y_lm, so with q(parent) = W q(child) the child's expansion
    // is L(child)_i = sum_j W_ji (2 l_j + 1) L(parent)_j / (2 l_i + 1)
    const double *W = I.Wm2m_h + (size_t)I.m2m_disp[gc - I.m2m_base] * N * N;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
      double t = 0.0;
      for (int j = 0; j < N; ++j) {
        const int lj = (int)sqrtf((float)j + 0.5f);
        t += W[(size_t)i * N + j] * (2 * lj + 1) * Lp[j];
      }
      const int li = (int)sqrtf((float)i + 0.5f);
      I.L[(size_t)gc * N + i] += t / (2 * li + 1);
    }
    return;
  }
  const double *W = I.Wm2m + (size_t)I.m2m_disp[gc - I.m2m_base] * ((size_t)N * (N + 1) / 2);
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    double t = Lp[i];
    for (int j = i + 1; j < N; ++j) t += W[wpos(j, i, N)] * Lp[j];
    I.L[(size_t)gc * N + i] += t;
  }
}

// V(r) += sum_lm L_lm S_lm(r - c) over the owned points of every box; block
// (chunk, box, density).  L = the density's own local expansions unless
// Lext is given (evaluation of caller-supplied expansions).
__global__ void l2p_kernel(const GInst *__restrict__ insts, const double *__restrict__ Lext,
                           int lmax) {
  extern __shared__ double Ls[];
  const GInst &I = insts[blockIdx.z];
  if (I.kappa > 0.0) return;  // Helmholtz instances: l2p_helm_kernel
  const int N = (lmax + 1) * (lmax + 1);
  const BoxInfo b = I.boxes[blockIdx.y];
  const double *L = Lext ? Lext : I.L + (size_t)I.fine_off * N;
  for (int k = threadIdx.x; k < N; k += blockDim.x) Ls[k] = L[(size_t)blockIdx.y * N + k];
  __syncthreads();
  const double *xs = I.wbox + (3 * 64) * I.wstride;
  const int ws = I.wstride;
  const long long n = (long long)b.own[0] * b.own[1] * b.own[2];
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % b.own[0]);
    const long long r = e / b.own[0];
    const int j = (int)(r % b.own[1]), k = (int)(r / b.own[1]);
    const int gx = b.p0[0] + i, gy = b.p0[1] + j, gz = b.p0[2] + k;
    double v = 0.0;
    const double x = xs[gx] - b.c[0], y = xs[ws + gy] - b.c[1], z = xs[2 * ws + gz] - b.c[2];
    solid_harmonics_tab(lmax, x, y, z, [&](int lm, double s) { v += Ls[lm] * s; });
    I.V[(size_t)gx + (size_t)I.Nx * gy + (size_t)I.Nx * I.Ny * gz] += v;
  }
}

// Helmholtz L2P, V(r) += 8 kappa sum (2l+1)/(4 pi) i_l(kappa r) Y_lm L_lm
// (src/gbfmm/gbfmm_helmholtz3d.F90:1019-1105), with the multipole kernel's
// lane tasks: lane p(lmax+1)+t evaluates task t's harmonics of point p and
// the point's lanes sum their terms with a segmented shuffle reduction.  The
// Bessel ratios f_l(kappa r), l = 0..lmax, come first for 32 points per
// warp, one lane per point (series for lmax and lmax - 1, then the downward
// recursion f_l = (2l+3) f_{l+1} + (kappa r)^2 f_{l+2}), into shared memory.
// Block (chunk, box, density); Coulomb instances return.
constexpr int kL2pHelmWarps = 8;
constexpr int kL2pHelmThreads = kL2pHelmWarps * 32;  // sF has one row block per warp

__global__ void __launch_bounds__(kL2pHelmThreads)
    l2p_helm_kernel(const GInst *__restrict__ insts, const double *__restrict__ Lext, int lmax) {
  __shared__ double sA[16 * 16], sB[16 * 16], sLt[16 * 16];  // [k][t]
  __shared__ double sF[kL2pHelmWarps][32][17];              // [warp][point][l]
  const GInst &I = insts[blockIdx.z];
  if (!(I.kappa > 0.0)) return;
  const int L = lmax, L1 = lmax + 1, N = L1 * L1;
  const int PP = 32 / L1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const BoxInfo b = I.boxes[blockIdx.y];
  const double *Lb = (Lext ? Lext : I.L + (size_t)I.fine_off * N) + (size_t)blockIdx.y * N;
  const double kappa = I.kappa;
  for (int e = threadIdx.x; e < N; e += blockDim.x) {
    const int t = e / L1, k = e % L1;
    int l, m;
    mp_step(L, t, k, l, m);
    const bool start = l == abs(m);
    sA[k * 16 + t] = start ? 0.0 : c_shA[lmi(l, m)];
    sB[k * 16 + t] = start ? 0.0 : c_shB[lmi(l, m)];
    double kp = 8.0 * kappa / (4.0 * 3.141592653589793238);  // 8 kappa^(l+1) (2l+1) / (4 pi)
    for (int i = 0; i < l; ++i) kp *= kappa;
    sLt[k * 16 + t] = Lb[lmi(l, m)] * ((2 * l + 1) * kp);
  }
  __syncthreads();
  const int p = lane / L1, t = lane % L1;
  int m1, m2, len1;
  mp_task(L, t, m1, m2, len1);
  const int a1 = abs(m1), a2 = abs(m2), amax = t == 0 ? 0 : max(a1, a2);
  const double *xs = I.wbox + (3 * 64) * I.wstride;
  const int ws = I.wstride;
  const long long n = (long long)b.own[0] * b.own[1] * b.own[2];
  double(*F)[17] = sF[warp];
  const long long stride32 = (long long)gridDim.x * (blockDim.x >> 5) * 32;
  for (long long base32 = ((long long)blockIdx.x * (blockDim.x >> 5) + warp) * 32; base32 < n;
       base32 += stride32) {
  {  // Bessel ratios of the 32 points, lane = point
    const long long e = min(base32 + lane, n - 1);
    const int i = (int)(e % b.own[0]);
    const long long r = e / b.own[0];
    const int j = (int)(r % b.own[1]), k = (int)(r / b.own[1]);
    const double x = xs[b.p0[0] + i] - b.c[0], y = xs[ws + b.p0[1] + j] - b.c[1],
                 z = xs[2 * ws + b.p0[2] + k] - b.c[2];
    const double x2 = (kappa * kappa) * (x * x + y * y + z * z);
    double *f = F[lane];
    f[L] = bessel_ratio_series(0.5 * x2, L);
    if (L >= 1) f[L - 1] = bessel_ratio_series(0.5 * x2, L - 1);
    for (int l = L - 2; l >= 0; --l) f[l] = (2 * l + 3) * f[l + 1] + x2 * f[l + 2];
  }
  __syncwarp();
  for (int sub = 0; sub < 32; sub += PP) {
    const long long e = base32 + sub + p;
    const bool valid = p < PP && sub + p < 32 && e < n;
    const long long ee = valid ? e : 0;
    const int i = (int)(ee % b.own[0]);
    const long long r = ee / b.own[0];
    const int j = (int)(r % b.own[1]), k = (int)(r / b.own[1]);
    const int gx = b.p0[0] + i, gy = b.p0[1] + j, gz = b.p0[2] + k;
    const double x = xs[gx] - b.c[0], y = xs[ws + gy] - b.c[1], z = xs[2 * ws + gz] - b.c[2];
    const double r2 = x * x + y * y + z * z;
    double s1 = 1.0, s2 = 0.0;
    {
      double top = x, bot = y;
      for (int mm = 1; mm <= amax; ++mm) {
        if (mm >= 2) {
          const double c = c_shC[mm];
          const double nb = c * (y * top + x * bot);
          const double nt = c * (x * top - y * bot);
          top = nt;
          bot = nb;
        }
        if (mm == a1) s1 = m1 > 0 ? top : bot;
        if (mm == a2) s2 = m2 > 0 ? top : bot;
      }
    }
    const double *fp = F[valid ? sub + p : 0];
    double acc = 0.0, p1 = 0.0, p2 = 0.0;
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      if (kk > L) break;
      const bool st = kk == 0 || kk == len1;
      const double rec = sA[kk * 16 + t] * (z * p1) - sB[kk * 16 + t] * (r2 * p2);
      const double cur = st ? (kk == 0 ? s1 : s2) : rec;
      p2 = st ? 0.0 : p1;
      p1 = cur;
      const double f = fp[kk < len1 ? a1 + kk : a2 + kk - len1];
      acc += (sLt[kk * 16 + t] * f) * cur;
    }
    // segmented sum over the point's lanes t = 0..L (fixed order)
#pragma unroll
    for (int off = 1; off < 16; off <<= 1) {
      const double o = __shfl_down_sync(0xffffffffu, acc, off);
      if (t + off < L1) acc += o;
    }
    if (valid && t == 0) I.V[(size_t)gx + (size_t)I.Nx * gy + (size_t)I.Nx * I.Ny * gz] += acc;
  }
  __syncwarp();
  }
}

// Energy int rho V with the LIP weights: kEnergyBlocks fixed blocks per
// density, then one fixed-order sum per density (deterministic).
__global__ void energy_kernel(const GInst *__restrict__ insts) {
  __shared__ double sh[32];
  const GInst &I = insts[blockIdx.y];
  // one warp per x row (y, z): its weight wy wz once, lanes over x
  const int lane = threadIdx.x & 31;
  const long long rows = (long long)I.Ny * I.Nz;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  double acc = 0.0;
  for (long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows;
       r += nwarps) {
    const size_t base = (size_t)r * I.Nx;
    double srow = 0.0;
    // four independent elements per lane per pass (loads in flight together)
    for (int x0 = lane; x0 < I.Nx; x0 += 128) {
      double p[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int x = x0 + 32 * u;
        p[u] = x < I.Nx ? I.rho[base + x] * I.V[base + x] * I.wx[x] : 0.0;
      }
      srow += (p[0] + p[1]) + (p[2] + p[3]);
    }
    acc += srow * (I.wy[r % I.Ny] * I.wz[r / I.Ny]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    I.epart[blockIdx.x] = t;
  }
}

__global__ void energy_sum_kernel(const GInst *__restrict__ insts, double *out) {
  if (threadIdx.x != 0) return;
  const GInst &I = insts[blockIdx.x];
  double t = 0.0;
  for (int k = 0; k < kEnergyBlocks; ++k) t += I.epart[k];
  out[blockIdx.x] = t;
}

// ---------------------------------------------------------------------------
// Host-side M2L coefficient tables (multipole.F90:106-187), built once per
// lmax: entries of the packed lower triangle of T.
// ---------------------------------------------------------------------------
double fprod(int n) {
  double p = 1.0;
  for (int i = 1; i <= n; ++i) p = p * (1.0 * i);
  return p;
}
double sg(int k) { return (k & 1) ? -1.0 : 1.0; }
double Ccf(int l, int m) {
  if (m == 0) return 1.0 / fprod(l);
  if (m > 0) return sg(m) / std::sqrt(2.0 * fprod(l - m) * fprod(l + m));
  return sg(m) * Ccf(l, -m);
}
double Csf(int l, int m) {
  if (m == 0) return 0.0;
  if (m > 0) return sg(m) / std::sqrt(2.0 * fprod(l - m) * fprod(l + m));
  return -sg(m) * Csf(l, -m);
}
double Cstf(int l, int m) { return fprod(l - m) * fprod(l + m) * Csf(l, m); }
double Cctf(int l, int m) { return fprod(l - m) * fprod(l + m) * Ccf(l, m); }
double Df(int l, int m) { return std::sqrt(fprod(l + m) * fprod(l - m) * (2.0 - (m == 0))); }

struct M2LTables {
  std::vector<double> c1, c2;
  std::vector<int> lm1, lm2, prow, pcol;
};

void m2l_tables(int lmax, M2LTables &t) {
  const int N = (lmax + 1) * (lmax + 1);
  const double ij[3] = {1.0, 0.5, 0.25};
  auto lm_of = [](int s, int &l, int &m) {
    l = 0;
    while ((l + 1) * (l + 1) <= s) ++l;
    m = s - l * l - l;
  };
  for (int s = 0; s < N; ++s) {
    int j, k;
    lm_of(s, j, k);
    for (int i = s; i < N; ++i) {
      int l, m;
      lm_of(i, l, m);
      const double c = 2 * sg(j) * ij[(m == 0) + (k == 0)];
      int L1 = l + j, M1, M2;
      double a, b;
      if (m >= 0 && k >= 0) {
        M1 = std::abs(m + k); a = Cctf(L1, m + k);
        M2 = std::abs(m - k); b = sg(k) * Cctf(L1, m - k);
      } else if (m >= 0 && k < 0) {
        M1 = -std::abs(m + k); a = Cstf(L1, m + k);
        M2 = -std::abs(m - k); b = -sg(k) * Cstf(L1, m - k);
        a = -a * sg(k); b = -b * sg(k);
      } else if (m < 0 && k >= 0) {
        M1 = -std::abs(m + k); a = Cstf(L1, m + k);
        M2 = -std::abs(m - k); b = sg(k) * Cstf(L1, m - k);
        a = -a * sg(m); b = -b * sg(m);
      } else {
        M1 = std::abs(m + k); a = -Cctf(L1, m + k);
        M2 = std::abs(m - k); b = sg(k) * Cctf(L1, m - k);
        a = a * sg(m + k); b = b * sg(m + k);
      }
      a = a * c; b = b * c;
      a = sg(m) * a / Df(l, m); b = sg(m) * b / Df(l, m);
      a = sg(k) * a / Df(j, k); b = sg(k) * b / Df(j, k);
      t.c1.push_back(a);
      t.c2.push_back(b);
      t.lm1.push_back(L1 * (L1 + 1) + M1);
      t.lm2.push_back(L1 * (L1 + 1) + M2);
      t.prow.push_back(i);
      t.pcol.push_back(s);
    }
  }
}

// Host-side translation (M2M/L2L) coefficient tables
// (TranslationMatrix_compute_coeffs, multipole.F90:372-440): entry r of the
// packed lower triangle (column s = (j,k), row i = (l,m) >= s) is
// c1 S_{l-j, m1} + c2 S_{l-j, m2} of the displacement's regular solid
// harmonics; a term whose order |m1| or |m2| exceeds l - j is absent.
struct TransTables {
  std::vector<double> c1, c2;
  std::vector<int> lm1, lm2;
};

void translation_tables(int lmax, TransTables &t) {
  const int N = (lmax + 1) * (lmax + 1);
  auto lm_of = [](int s, int &l, int &m) {
    l = 0;
    while ((l + 1) * (l + 1) <= s) ++l;
    m = s - l * l - l;
  };
  for (int s = 0; s < N; ++s) {
    int j, k;
    lm_of(s, j, k);
    const double hk = k == 0 ? 0.5 : 1.0;  // the reference's ij(delta(0,k))
    for (int i = s; i < N; ++i) {
      int l, m;
      lm_of(i, l, m);
      const int Lo = l - j;
      double a = 0.0, b = 0.0;
      int ma = 0, mb = 0;
      bool ha = false, hb = false;
      const int dm = std::abs(m - k), sm = std::abs(m + k);
      if (m >= 0 && k >= 0) {
        if (Lo >= 0 && dm <= Lo) ha = true, ma = dm, a = Ccf(Lo, m - k) * hk;
        if (Lo >= 0 && sm <= Lo) hb = true, mb = sm, b = sg(k) * Ccf(Lo, m + k) * hk;
      } else if (m >= 0) {  // k < 0
        if (Lo >= 0 && dm <= Lo) ha = true, ma = -dm, a = Csf(Lo, m - k) * sg(k);
        if (Lo >= 0 && sm <= Lo) hb = true, mb = -sm, b = -Csf(Lo, m + k);
      } else if (k >= 0) {  // m < 0
        if (Lo >= 0 && dm <= Lo) ha = true, ma = -dm, a = -Csf(Lo, m - k) * sg(m) * hk;
        if (Lo >= 0 && sm <= Lo) hb = true, mb = -sm, b = -Csf(Lo, m + k) * hk * sg(m + k);
      } else {
        if (Lo >= 0 && dm <= Lo) ha = true, ma = dm, a = Ccf(Lo, m - k) * sg(m - k);
        if (Lo >= 0 && sm <= Lo) hb = true, mb = sm, b = -Ccf(Lo, m + k) * sg(m);
      }
      const double scale = Df(l, m) * sg(m - k) / Df(j, k);
      t.c1.push_back(a * scale);
      t.c2.push_back(b * scale);
      t.lm1.push_back(ha ? Lo * (Lo + 1) + ma : -1);
      t.lm2.push_back(hb ? Lo * (Lo + 1) + mb : -1);
    }
  }
}

// octree box index <-> vector (gbfmm_parallel_info.F90:1128-1194)
void box_vector(int ibox, int level, int v[3]) {
  int vv[3] = {0, 0, 0}, rem;
  if (level > 1) {
    box_vector((ibox - 1) / 8 + 1, level - 1, vv);
    for (int d = 0; d < 3; ++d) vv[d] *= 2;
    rem = (ibox - 1) % 8;
  } else {
    rem = ibox - 1;
  }
  const int iz = rem / 4;
  rem -= iz * 4;
  const int iy = rem / 2;
  rem -= iy * 2;
  v[0] = vv[0] + rem;
  v[1] = vv[1] + iy;
  v[2] = vv[2] + iz;
}
int box_index(const int v[3], int level) {
  int idx, rem[3];
  if (level > 1) {
    int pv[3] = {v[0] / 2, v[1] / 2, v[2] / 2};
    idx = (box_index(pv, level - 1) - 1) * 8 + 1;
    for (int d = 0; d < 3; ++d) rem[d] = v[d] - pv[d] * 2;
  } else {
    idx = 1;
    for (int d = 0; d < 3; ++d) rem[d] = v[d];
  }
  return idx + rem[0] + rem[1] * 2 + rem[2] * 4;
}
std::vector<int> neighbours(int ibox, int level) {
  const int lim = 1 << level;
  int v[3];
  box_vector(ibox, level, v);
  std::vector<int> out;
  for (int iz = -1; iz <= 1; ++iz)
    for (int iy = -1; iy <= 1; ++iy)
      for (int ix = -1; ix <= 1; ++ix) {
        if (!ix && !iy && !iz) continue;
        const int w[3] = {v[0] + ix, v[1] + iy, v[2] + iz};
        if (w[0] < 0 || w[1] < 0 || w[2] < 0 || w[0] >= lim || w[1] >= lim || w[2] >= lim)
          continue;
        out.push_back(box_index(w, level));
      }
  return out;
}
std::vector<int> local_farfield(int ibox, int level) {
  std::vector<int> out;
  if (level < 2) return out;
  const auto pnn = neighbours((ibox - 1) / 8 + 1, level - 1);
  const auto nn = neighbours(ibox, level);
  for (int p : pnn)
    for (int c = 1; c <= 8; ++c) {
      const int child = (p - 1) * 8 + c;
      if (std::find(nn.begin(), nn.end(), child) == nn.end()) out.push_back(child);
    }
  return out;
}

// Adaptive mode (GBFMMParallelInfo_get_local_farfield_indices evaluation
// types 1 and 2, gbfmm_parallel_info.F90:827-983, as gbfmm_coulomb3d.F90:
// 1386-1433 uses them): of the neighbours of ibox's parent, those with a
// child among ibox's nearest neighbours contribute their other children
// (`partial`, boxes of `level`); the others contribute as whole boxes of
// level - 1 (`whole`).
void local_farfield_adaptive(int ibox, int level, std::vector<int> &partial,
                             std::vector<int> &whole) {
  partial.clear();
  whole.clear();
  if (level < 2) return;
  const auto pnn = neighbours((ibox - 1) / 8 + 1, level - 1);
  const auto nn = neighbours(ibox, level);
  for (int p : pnn) {
    bool has_nn = false;
    for (int c = 1; c <= 8 && !has_nn; ++c)
      has_nn = std::find(nn.begin(), nn.end(), (p - 1) * 8 + c) != nn.end();
    if (!has_nn) {
      whole.push_back(p);
      continue;
    }
    for (int c = 1; c <= 8; ++c) {
      const int child = (p - 1) * 8 + c;
      if (std::find(nn.begin(), nn.end(), child) == nn.end()) partial.push_back(child);
    }
  }
}

}  // namespace
}  // namespace dage

using namespace dage;

struct dage_gbfmm {
  int device = 0;
  double energy = 0.0, kappa = 0.0;  // kernel: Coulomb (energy 0) or e^(-kappa r)/r
  std::vector<double> disp;          // distinct far-field displacements (x, y, z)
  int level = 2, lmax = 12, nbox = 0, N = 0, P = 0, precision = DAGE_FP64;
  int lev0 = 2;  // coarsest level with multipoles: 1 in the adaptive mode
  Axis ax[3];
  int npts[3];
  dage_quad quad{};
  std::vector<double> tp, tw, w;
  std::vector<BoxInfo> boxes;
  int axis_pos_count[3];
  // per axis, per box position: near-field operator matrix (P x own x near)
  std::vector<DevBuf> Tnear[3];
  std::vector<DevBuf> band_near[3];  // K band per (t-point, 128-row tile) of Tnear
  DevBuf d_boxes, d_wbox, d_q, d_L, d_partial, d_Tm2l, d_ffstart, d_ffsrc, d_ffdisp;
  // levels 2..level: box offsets (lev_off[l], l = 2..level+1), expansion
  // centres of every box, M2M/L2L translation matrices per distinct
  // child-to-parent displacement
  std::vector<int> lev_off;
  int nbtot = 0, fine_off = 0, nm2m = 0;
  std::vector<double> centers;
  DevBuf d_Wm2m, d_m2m_disp;
  std::vector<double> m2m_dvec;  // child - parent of each distinct M2M displacement
  DevBuf d_Wm2m_h;               // Helmholtz M2M matrices for the current kappa
  int wstride = 0, nslab = 16, ndisp = 0;
  DevBuf d_U, d_W, d_desc[3];
  size_t U_per_box = 0, W_per_box = 0;
  std::vector<StageDesc> desc[3];
  int tile_n[3] = {64, 64, 64};  // near-field stage tile widths (autotuned)
  // fp16x3 near field on the tensor cores (near_mixed.cu): FP16 matrix
  // parts of the plan, the single-density set, the weights on the device
  NearF16Plan *near16 = nullptr;
  NearF16Set *near16set = nullptr;
  DevBuf d_wn;
  DevBuf wts[3], d_epart, d_energy, d_inst, d_rho, d_V;
  cudaStream_t own_stream = nullptr, stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_ms = 0.f;
};

namespace {

int split_axis(int ncell, int nb, int v, int &c0, int &nc) {
  const int base = ncell / nb, rem = ncell % nb;
  c0 = v * base + std::min(v, rem);  // 0-based first cell
  nc = base + (v < rem ? 1 : 0);
  return 0;
}

// ---------------------------------------------------------------------------
// Helmholtz M2L coefficient tables (host; assembled into matrices on the GPU)
// ---------------------------------------------------------------------------
// k_0..k_L(x), k_0 = (pi/2) e^-x / x, upward recursion
// (src/bubbles/helmholtz3d.F90:1133-1174; long double as the reference's
// REAL128 evaluation is closer to it than double).
void bessel_k_host(double x, int L, std::vector<double> &out) {
  typedef long double ext;
  const ext X = x, pi = 3.14159265358979323846264338327950288L;
  std::vector<ext> k(L + 2, 0.0L);
  k[0] = std::exp(-X) / X * pi / 2;
  if (L >= 1) k[1] = std::exp(-X) * (X + 1) / (X * X) * pi / 2;
  for (int l = 2; l <= L; ++l) k[l] = (2 * l - 1) * k[l - 1] / X + k[l - 2];
  out.assign(k.begin(), k.begin() + L + 1);
}

// Coaxial multipole-to-local coefficients C(l, n, m), l, n, m <= L, from
// k_0..k_{L+1}(kappa d): the recurrence of src/bubbles/
// helmholtz_multipole_tools.F90:428-511 (a/b coefficients :591-607, zero for
// n < 0), which seeds (l, 0, 0) and (0, n, 0) up to L+1 and leaves the
// entries it never fills at zero, exactly as the reference does.
void coaxial_ml(const std::vector<double> &k, int L, std::vector<double> &out) {
  const int D = L + 3;  // indices -1 .. L+1
  std::vector<double> C((size_t)D * D * D, 0.0);
  auto c = [&](int l, int n, int m) -> double & {
    return C[((size_t)(l + 1) * D + (n + 1)) * D + (m + 1)];
  };
  auto A = [](int n, int m) {
    if (n < 0) return 0.0;
    const int am = std::abs(m);
    return std::sqrt((double)((n + 1 + am) * (n + 1 - am)) / ((2 * n + 1) * (2 * n + 3)));
  };
  auto B = [](int n, int m) {
    if (n < 0 || std::abs(m) > n) return 0.0;
    const double b = std::sqrt((double)((n - m - 1) * (n - m)) / ((2 * n - 1) * (2 * n + 1)));
    return m < 0 ? -b : b;
  };
  c(0, 0, 0) = k[0];
  for (int n = 1; n <= L + 1; ++n) {
    c(n, 0, 0) = ((n & 1) ? -1.0 : 1.0) * std::sqrt(2.0 * n + 1) * k[n];
    c(0, n, 0) = std::sqrt(2.0 * n + 1) * k[n];
  }
  for (int n = 1; n <= L; ++n) {
    c(1, n, 0) = (-A(n, 0) * c(0, n + 1, 0) - A(n - 1, 0) * c(0, n - 1, 0)) / A(0, 0);
    c(n, 1, 0) = (((1 + n) & 1) ? -1.0 : 1.0) * c(1, n, 0);
  }
  for (int m = 0; m <= L; ++m) {
    for (int n = m; n <= L; ++n)
      for (int l = m; l <= L; ++l)
        c(l, n + 1, m) = (-A(l, m) * c(l + 1, n, m) - A(l - 1, m) * c(l - 1, n, m) -
                          A(n - 1, m) * c(l, n - 1, m)) /
                         A(n, m);
    for (int l = m; l <= L; ++l)
      c(l, m + 1, m + 1) = (-B(l, -m - 1) * c(l - 1, m, m) - B(l + 1, m) * c(l + 1, m, m)) /
                           B(m + 1, -m - 1);
  }
  out.resize((size_t)(L + 1) * (L + 1) * (L + 1));
  for (int l = 0; l <= L; ++l)
    for (int n = 0; n <= L; ++n)
      for (int m = 0; m <= L; ++m) out[((size_t)l * (L + 1) + n) * (L + 1) + m] = c(l, n, m);
}

// i_0..i_L(x), modified spherical Bessel functions of the first kind, by
// their all-positive series x^l sum_k (x^2/2)^k / (k! (2l+1)(2l+3)..(2l+2k+1))
// in long double.
void bessel_i_host(double x, int L, std::vector<double> &out) {
  typedef long double ext;
  out.assign(L + 1, 0.0);
  const ext X = x, h = X * X / 2;
  ext lead = 1;  // x^l / (2l+1)!!
  for (int l = 0; l <= L; ++l) {
    if (l > 0) lead *= X / (2 * l + 1);
    ext term = lead, sum = lead;
    for (int k = 1; k < 1000 && term > sum * 1e-22L; ++k) {
      term *= h / (k * (ext)(2 * l + 2 * k + 1));
      sum += term;
    }
    out[l] = (double)sum;
  }
}

// Coaxial multipole-to-multipole coefficients C(l, n, m), l, n, m <= L, from
// i_0..i_{L+1}(kappa d): the recurrence of src/bubbles/
// helmholtz_multipole_tools.F90:513-588 (get_all_aligned_translation_
// coefficients; a/b coefficients :591-607, zero for n < 0).
void coaxial_mm(const std::vector<double> &ib, int L, std::vector<double> &out) {
  const int D = L + 3;  // indices -1 .. L+1
  std::vector<double> C((size_t)D * D * D, 0.0);
  auto c = [&](int l, int n, int m) -> double & {
    return C[((size_t)(l + 1) * D + (n + 1)) * D + (m + 1)];
  };
  auto A = [](int n, int m) {
    if (n < 0) return 0.0;
    const int am = std::abs(m);
    return std::sqrt((double)((n + 1 + am) * (n + 1 - am)) / ((2 * n + 1) * (2 * n + 3)));
  };
  auto B = [](int n, int m) {
    if (n < 0 || std::abs(m) > n) return 0.0;
    const double b = std::sqrt((double)((n - m - 1) * (n - m)) / ((2 * n - 1) * (2 * n + 1)));
    return m < 0 ? -b : b;
  };
  for (int n = 0; n <= L + 1; ++n) {
    c(n, 0, 0) = ((n & 1) ? -1.0 : 1.0) * std::sqrt(2.0 * n + 1) * ib[n];
    c(0, n, 0) = ((n & 1) ? -1.0 : 1.0) * c(n, 0, 0);
  }
  for (int n = 1; n <= L; ++n) {
    c(1, n, 0) = (A(n, 0) * c(0, n + 1, 0) + A(n - 1, 0) * c(0, n - 1, 0)) / A(0, 0);
    c(n, 1, 0) = (((1 + n) & 1) ? -1.0 : 1.0) * c(1, n, 0);
  }
  for (int m = 0; m <= L; ++m) {
    for (int n = m; n <= L; ++n)
      for (int l = m; l <= L; ++l)
        c(l, n + 1, m) = (A(l, m) * c(l + 1, n, m) + A(l - 1, m) * c(l - 1, n, m) -
                          A(n - 1, m) * c(l, n - 1, m)) /
                         A(n, m);
    for (int l = m; l <= L; ++l)
      c(l, m + 1, m + 1) = (B(l, -m - 1) * c(l - 1, m, m) + B(l + 1, m) * c(l + 1, m, m)) /
                           B(m + 1, -m - 1);
  }
  out.resize((size_t)(L + 1) * (L + 1) * (L + 1));
  for (int l = 0; l <= L; ++l)
    for (int n = 0; n <= L; ++n)
      for (int m = 0; m <= L; ++m) out[((size_t)l * (L + 1) + n) * (L + 1) + m] = c(l, n, m);
}

// Rotation blocks R_l[m'][m] (l = 0..L, block l at (2l-1)l(2l+1)/3) taking
// real-harmonic expansions to the frame whose z axis is dhat: the unique
// matrices with S_lm(Q^T r') = sum_m' R_l[m'][m] S_lm'(r'), solved from
// 3(2l+1) sample directions by the normal equations.
void rotation_blocks(const double *dhat, int L, std::vector<double> &out) {
  double z[3] = {dhat[0], dhat[1], dhat[2]};
  const double nz = std::sqrt(z[0] * z[0] + z[1] * z[1] + z[2] * z[2]);
  for (double &v : z) v /= nz;
  const double t[3] = {std::fabs(z[0]) > 0.9 ? 0.0 : 1.0, std::fabs(z[0]) > 0.9 ? 1.0 : 0.0, 0.0};
  double x[3] = {t[1] * z[2] - t[2] * z[1], t[2] * z[0] - t[0] * z[2], t[0] * z[1] - t[1] * z[0]};
  const double nx = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  for (double &v : x) v /= nx;
  const double y[3] = {z[1] * x[2] - z[2] * x[1], z[2] * x[0] - z[0] * x[2],
                       z[0] * x[1] - z[1] * x[0]};
  out.assign((size_t)(L + 1) * (2 * L + 1) * (2 * L + 3) / 3, 0.0);  // sum of (2l+1)^2
  for (int l = 0; l <= L; ++l) {
    const int w = 2 * l + 1, np = 3 * w;
    std::vector<double> Bm((size_t)np * w), Gm((size_t)np * w);
    for (int q = 0; q < np; ++q) {
      const double u = 1.0 - 2.0 * (q + 0.5) / np, ph = 2.399963229728653 * q;
      const double sr = std::sqrt(1.0 - u * u);
      const double rp[3] = {sr * std::cos(ph), sr * std::sin(ph), u};
      const double ro[3] = {x[0] * rp[0] + y[0] * rp[1] + z[0] * rp[2],
                            x[1] * rp[0] + y[1] * rp[1] + z[1] * rp[2],
                            x[2] * rp[0] + y[2] * rp[1] + z[2] * rp[2]};
      solid_harmonics(l, rp[0], rp[1], rp[2], [&](int lm, double v) {
        if (lm >= l * l) Bm[(size_t)q * w + lm - l * l] = v;
      });
      solid_harmonics(l, ro[0], ro[1], ro[2], [&](int lm, double v) {
        if (lm >= l * l) Gm[(size_t)q * w + lm - l * l] = v;
      });
    }
    std::vector<double> M((size_t)w * 2 * w, 0.0);
    for (int i = 0; i < w; ++i)
      for (int j = 0; j < w; ++j)
        for (int q = 0; q < np; ++q) {
          M[(size_t)i * 2 * w + j] += Bm[(size_t)q * w + i] * Bm[(size_t)q * w + j];
          M[(size_t)i * 2 * w + w + j] += Bm[(size_t)q * w + i] * Gm[(size_t)q * w + j];
        }
    for (int cc = 0; cc < w; ++cc) {
      int pv = cc;
      for (int r = cc + 1; r < w; ++r)
        if (std::fabs(M[(size_t)r * 2 * w + cc]) > std::fabs(M[(size_t)pv * 2 * w + cc])) pv = r;
      for (int j = 0; j < 2 * w; ++j) std::swap(M[(size_t)cc * 2 * w + j], M[(size_t)pv * 2 * w + j]);
      const double dv = M[(size_t)cc * 2 * w + cc];
      for (int j = 0; j < 2 * w; ++j) M[(size_t)cc * 2 * w + j] /= dv;
      for (int r = 0; r < w; ++r)
        if (r != cc) {
          const double f = M[(size_t)r * 2 * w + cc];
          for (int j = 0; j < 2 * w; ++j) M[(size_t)r * 2 * w + j] -= f * M[(size_t)cc * 2 * w + j];
        }
    }
    const size_t off = (size_t)(2 * l - 1) * l * (2 * l + 1) / 3;
    for (int i = 0; i < w; ++i)
      for (int j = 0; j < w; ++j) out[off + (size_t)i * w + j] = M[(size_t)i * 2 * w + w + j];
  }
}

// M2L matrix of every distinct displacement for the plan's kernel.
// M2L matrix of every distinct displacement of a plan for the kernel with
// parameter kappa (0: Coulomb), into T.
int build_m2l_into(const dage_gbfmm *g, double kappa, DevBuf &T) {
  if (g->ndisp == 0) return 0;
  cudaStream_t s = g->stream;
  const int lmax = g->lmax;
  DAGE_TRY(T.alloc(sizeof(double) * (size_t)g->ndisp * g->N * g->N));
  if (kappa > 0.0) {
    const int rblk = (lmax + 1) * (2 * lmax + 1) * (2 * lmax + 3) / 3;
    const size_t cblk = (size_t)(lmax + 1) * (lmax + 1) * (lmax + 1);
    std::vector<double> R((size_t)g->ndisp * rblk), C(g->ndisp * cblk), r, c, k;
    for (int d = 0; d < g->ndisp; ++d) {
      // translation from the source box to the target box: target - source
      const double *dv = &g->disp[3 * d];  // source - target
      const double dir[3] = {-dv[0], -dv[1], -dv[2]};
      rotation_blocks(dir, lmax, r);
      std::copy(r.begin(), r.begin() + rblk, R.begin() + (size_t)d * rblk);
      bessel_k_host(kappa * std::sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]),
                    lmax + 1, k);
      coaxial_ml(k, lmax, c);
      std::copy(c.begin(), c.end(), C.begin() + (size_t)d * cblk);
    }
    TmpBuf dR, dC;
    DAGE_TRY(dR.alloc(sizeof(double) * R.size()));
    DAGE_TRY(dC.alloc(sizeof(double) * C.size()));
    DAGE_CUDA_TRY(cudaMemcpyAsync(dR.ptr, R.data(), sizeof(double) * R.size(), cudaMemcpyHostToDevice, s));
    DAGE_CUDA_TRY(cudaMemcpyAsync(dC.ptr, C.data(), sizeof(double) * C.size(), cudaMemcpyHostToDevice, s));
    helm_m2l_matrices_kernel<<<g->ndisp, 256, 0, s>>>(dR.as<double>(), rblk, dC.as<double>(), lmax,
                                                       T.as<double>());
    DAGE_CUDA_TRY(cudaGetLastError());
    DAGE_CUDA_TRY(cudaStreamSynchronize(s));
    return 0;
  }
  M2LTables t;
  m2l_tables(lmax, t);
  TmpBuf dd, c1, c2, l1, l2, pr, pc;
  const size_t M = t.c1.size();
  DAGE_TRY(dd.alloc(sizeof(double) * g->disp.size()));
  DAGE_TRY(c1.alloc(sizeof(double) * M));
  DAGE_TRY(c2.alloc(sizeof(double) * M));
  DAGE_TRY(l1.alloc(sizeof(int) * M));
  DAGE_TRY(l2.alloc(sizeof(int) * M));
  DAGE_TRY(pr.alloc(sizeof(int) * M));
  DAGE_TRY(pc.alloc(sizeof(int) * M));
  DAGE_CUDA_TRY(cudaMemcpyAsync(dd.ptr, g->disp.data(), sizeof(double) * g->disp.size(), cudaMemcpyHostToDevice, s));
  DAGE_CUDA_TRY(cudaMemcpyAsync(c1.ptr, t.c1.data(), sizeof(double) * M, cudaMemcpyHostToDevice, s));
  DAGE_CUDA_TRY(cudaMemcpyAsync(c2.ptr, t.c2.data(), sizeof(double) * M, cudaMemcpyHostToDevice, s));
  DAGE_CUDA_TRY(cudaMemcpyAsync(l1.ptr, t.lm1.data(), sizeof(int) * M, cudaMemcpyHostToDevice, s));
  DAGE_CUDA_TRY(cudaMemcpyAsync(l2.ptr, t.lm2.data(), sizeof(int) * M, cudaMemcpyHostToDevice, s));
  DAGE_CUDA_TRY(cudaMemcpyAsync(pr.ptr, t.prow.data(), sizeof(int) * M, cudaMemcpyHostToDevice, s));
  DAGE_CUDA_TRY(cudaMemcpyAsync(pc.ptr, t.pcol.data(), sizeof(int) * M, cudaMemcpyHostToDevice, s));
  const int NI = (2 * lmax + 1) * (2 * lmax + 1);
  m2l_matrices_kernel<<<g->ndisp, 256, sizeof(double) * NI, s>>>(
      dd.as<double>(), lmax, c1.as<double>(), c2.as<double>(), l1.as<int>(), l2.as<int>(),
      pr.as<int>(), pc.as<int>(), T.as<double>());
  DAGE_CUDA_TRY(cudaGetLastError());
  DAGE_CUDA_TRY(cudaStreamSynchronize(s));
  return 0;
}

int build_m2l(dage_gbfmm *g) { return build_m2l_into(g, g->kappa, g->d_Tm2l); }

// Helmholtz M2M matrices of the plan's child-to-parent displacements for
// kappa: the HelmholtzMultipoleTranslator (helmholtz_multipole_tools.F90:
// 172-278 with :338-378: rotation to the axis parent - child, coaxial
// translation by i_l(kappa d), rotation back), assembled like the M2L
// converter (the same scalings and real-basis coaxial action), into W.
int build_helm_m2m_into(const dage_gbfmm *g, double kappa, DevBuf &W) {
  if (g->nm2m == 0 || kappa <= 0.0) return 0;
  cudaStream_t s = g->stream;
  const int lmax = g->lmax;
  const int rblk = (lmax + 1) * (2 * lmax + 1) * (2 * lmax + 3) / 3;
  const size_t cblk = (size_t)(lmax + 1) * (lmax + 1) * (lmax + 1);
  std::vector<double> R((size_t)g->nm2m * rblk), C(g->nm2m * cblk), r, c, ib;
  for (int d = 0; d < g->nm2m; ++d) {
    const double *dv = &g->m2m_dvec[3 * d];  // child - parent
    const double dir[3] = {-dv[0], -dv[1], -dv[2]};
    rotation_blocks(dir, lmax, r);
    std::copy(r.begin(), r.begin() + rblk, R.begin() + (size_t)d * rblk);
    bessel_i_host(kappa * std::sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]), lmax + 1, ib);
    coaxial_mm(ib, lmax, c);
    std::copy(c.begin(), c.end(), C.begin() + (size_t)d * cblk);
  }
  TmpBuf dR, dC;
  DAGE_TRY(W.alloc(sizeof(double) * (size_t)g->nm2m * g->N * g->N));
  DAGE_TRY(dR.alloc(sizeof(double) * R.size()));
  DAGE_TRY(dC.alloc(sizeof(double) * C.size()));
  DAGE_CUDA_TRY(cudaMemcpyAsync(dR.ptr, R.data(), sizeof(double) * R.size(), cudaMemcpyHostToDevice, s));
  DAGE_CUDA_TRY(cudaMemcpyAsync(dC.ptr, C.data(), sizeof(double) * C.size(), cudaMemcpyHostToDevice, s));
  helm_m2l_matrices_kernel<<<g->nm2m, 256, 0, s>>>(dR.as<double>(), rblk, dC.as<double>(), lmax,
                                                    W.as<double>());
  DAGE_CUDA_TRY(cudaGetLastError());
  DAGE_CUDA_TRY(cudaStreamSynchronize(s));
  return 0;
}

// Near-field weights w_p = 2/sqrt(pi) tw_p, times e^(2E/(4 t_p^2)) for the
// Helmholtz kernel when E < -0.005 (src/gbfmm/gbfmm_helmholtz3d.F90:478-516).
void weights_for(const dage_gbfmm *g, double energy, std::vector<double> &w) {
  const double two_over_sqrtpi = 2.0 / std::sqrt(std::acos(-1.0));
  w.resize(g->P);
  for (int p = 0; p < g->P; ++p) {
    double tw = g->tw[p];
    if (energy < -0.005) tw *= std::exp(2.0 * energy / (4.0 * g->tp[p] * g->tp[p]));
    w[p] = two_over_sqrtpi * tw;
  }
}

void set_weights(dage_gbfmm *g) { weights_for(g, g->energy, g->w); }

int gbfmm_create_impl(dage_gbfmm *g, const dage_grid1d grid[3], int maxlevel, int lmax,
                      const dage_quad *quad) {
  DAGE_TRY(sh_tables_init());
  if (!grid || !quad) return fail(DAGE_E_INVALID, "null argument");
  // levels 2..maxlevel: M2L at every level (the local far field of a level-2
  // box is every box outside its neighbourhood), M2M/L2L between levels
  if (maxlevel < 2 || maxlevel > 5) return fail(DAGE_E_UNSUPPORTED, "maxlevel must be 2..5");
  if (lmax < 0 || lmax > kMaxLmax) return fail(DAGE_E_UNSUPPORTED, "lmax must be 0..%d", kMaxLmax);
  g->level = maxlevel;
  g->lmax = lmax;
  g->N = (lmax + 1) * (lmax + 1);
  g->quad = *quad;
  g->P = quad->nlin + quad->nlog;
  if (g->P < 1) return fail(DAGE_E_INVALID, "quadrature needs t-points");
  DAGE_CUDA_TRY(cudaGetDevice(&g->device));
  const int nb = 1 << maxlevel;
  g->nbox = nb * nb * nb;
  for (int d = 0; d < 3; ++d) {
    DAGE_TRY(make_axis(grid[d], g->ax[d]));
    g->npts[d] = g->ax[d].n();
    if (g->ax[d].ncell < nb) return fail(DAGE_E_INVALID, "fewer cells than boxes along an axis");
  }
  DAGE_CUDA_TRY(cudaStreamCreateWithFlags(&g->own_stream, cudaStreamNonBlocking));
  g->stream = g->own_stream;
  DAGE_CUDA_TRY(cudaEventCreate(&g->ev0));
  DAGE_CUDA_TRY(cudaEventCreate(&g->ev1));
  cudaStream_t s = g->stream;
  const int nlip = g->ax[0].nlip;

  // --- boxes ---------------------------------------------------------------
  g->boxes.resize(g->nbox);
  std::vector<int> pos_near0[3], pos_nearn[3], pos_p0[3], pos_np[3], pos_own[3];
  for (int d = 0; d < 3; ++d) {
    const Axis &a = g->ax[d];
    for (int v = 0; v < nb; ++v) {
      int c0, nc;
      split_axis(a.ncell, nb, v, c0, nc);
      const int p0 = c0 * (nlip - 1), np = nc * (nlip - 1) + 1;
      const bool last = (c0 + nc == a.ncell);
      int nc0, ncn, cc0, ccn;
      split_axis(a.ncell, nb, std::max(v - 1, 0), nc0, ncn);
      split_axis(a.ncell, nb, std::min(v + 1, nb - 1), cc0, ccn);
      const int near_c0 = nc0, near_c1 = cc0 + ccn;  // [near_c0, near_c1)
      pos_p0[d].push_back(p0);
      pos_np[d].push_back(np);
      pos_own[d].push_back(last ? np : np - 1);
      pos_near0[d].push_back(near_c0 * (nlip - 1));
      pos_nearn[d].push_back((near_c1 - near_c0) * (nlip - 1) + 1);
    }
  }
  for (int b = 0; b < g->nbox; ++b) {
    int v[3];
    box_vector(b + 1, maxlevel, v);
    BoxInfo &B = g->boxes[b];
    for (int d = 0; d < 3; ++d) {
      B.pos[d] = v[d];
      B.p0[d] = pos_p0[d][v[d]];
      B.np[d] = pos_np[d][v[d]];
      B.own[d] = pos_own[d][v[d]];
      B.q0[d] = pos_near0[d][v[d]];
      B.nq[d] = pos_nearn[d][v[d]];
      const Axis &a = g->ax[d];
      if (a.ncell % nb == 0) {  // the reference's centre (gbfmm_parallel_info.F90:1290-1299)
        const double qmin = a.points.front(), qmax = a.points.back();
        B.c[d] = qmin + (v[d] + 0.5) * ((qmax - qmin) / (nb + 0.0));
      } else {
        B.c[d] = 0.5 * (a.points[B.p0[d]] + a.points[B.p0[d] + B.np[d] - 1]);
      }
    }
  }
  DAGE_TRY(g->d_boxes.alloc(sizeof(BoxInfo) * g->nbox));
  DAGE_CUDA_TRY(cudaMemcpyAsync(g->d_boxes.ptr, g->boxes.data(), sizeof(BoxInfo) * g->nbox,
                                cudaMemcpyHostToDevice, s));

  // --- per-position box weights + point coordinates -------------------------
  int maxn = 0;
  for (int d = 0; d < 3; ++d) maxn = std::max(maxn, g->npts[d]);
  g->wstride = maxn;
  if (nb > 64) return fail(DAGE_E_UNSUPPORTED, "too many boxes per axis");
  std::vector<double> wbox((size_t)(3 * 64 + 3) * maxn, 0.0);
  for (int d = 0; d < 3; ++d) {
    LipBasis L;
    DAGE_TRY(make_lip_basis(nlip, g->ax[d].grid_type, L));
    for (int v = 0; v < nb; ++v) {
      int c0, nc;
      split_axis(g->ax[d].ncell, nb, v, c0, nc);
      double *w = wbox.data() + (size_t)(d * 64 + v) * maxn;
      for (int c = 0; c < nc; ++c)
        for (int i = 0; i < nlip; ++i) w[c * (nlip - 1) + i] += L.integrals[i] * g->ax[d].h[c0 + c];
    }
    std::copy(g->ax[d].points.begin(), g->ax[d].points.end(),
              wbox.begin() + (size_t)(3 * 64 + d) * maxn);
  }
  DAGE_TRY(g->d_wbox.alloc(sizeof(double) * wbox.size()));
  DAGE_CUDA_TRY(cudaMemcpyAsync(g->d_wbox.ptr, wbox.data(), sizeof(double) * wbox.size(),
                                cudaMemcpyHostToDevice, s));

  // --- levels: box offsets and expansion centres ------------------------------
  // A box of a coarser level is the union of its descendants at the finest
  // level (so the levels nest also for uneven splits); centres follow the
  // reference on evenly divisible axes, else the midpoint of the box's points.
  g->lev_off.assign(maxlevel + 2, 0);
  for (int l = g->lev0; l <= maxlevel; ++l) g->lev_off[l + 1] = g->lev_off[l] + (1 << (3 * l));
  g->nbtot = g->lev_off[maxlevel + 1];
  g->fine_off = g->lev_off[maxlevel];
  g->centers.assign(3 * (size_t)g->nbtot, 0.0);
  for (int l = g->lev0; l <= maxlevel; ++l) {
    const int nbl = 1 << l, f = 1 << (maxlevel - l);
    for (int i = 1; i <= (1 << (3 * l)); ++i) {
      int v[3];
      box_vector(i, l, v);
      double *c = &g->centers[3 * (size_t)(g->lev_off[l] + i - 1)];
      for (int d = 0; d < 3; ++d) {
        const Axis &a = g->ax[d];
        if (l == maxlevel) {
          c[d] = g->boxes[box_index(v, l) - 1].c[d];
        } else if (a.ncell % nb == 0) {
          const double qmin = a.points.front(), qmax = a.points.back();
          c[d] = qmin + (v[d] + 0.5) * ((qmax - qmin) / (nbl + 0.0));
        } else {
          const int first = pos_p0[d][v[d] * f];
          const int last = pos_p0[d][v[d] * f + f - 1] + pos_np[d][v[d] * f + f - 1] - 1;
          c[d] = 0.5 * (a.points[first] + a.points[last]);
        }
      }
    }
  }

  // --- far-field lists of every level, grouped by displacement ----------------
  // displacements keyed by (level, integer box-vector difference) on a regular
  // box lattice (all axes divide evenly), else by the exact centre differences
  bool regular = true;
  for (int d = 0; d < 3; ++d) regular = regular && (g->ax[d].ncell % nb == 0);
  std::map<std::vector<long long>, int> disp_index;
  std::vector<double> &disp = g->disp;
  std::vector<int> ffstart(1, 0), ffsrc, ffdisp;
  std::vector<int> partial, whole;
  for (int l = g->lev0; l <= maxlevel; ++l)
    for (int b = 1; b <= (1 << (3 * l)); ++b) {
      int vb[3];
      box_vector(b, l, vb);
      const double *cb = &g->centers[3 * (size_t)(g->lev_off[l] + b - 1)];
      // sources: (box, level) pairs
      std::vector<std::pair<int, int>> srcs;
      if (g->lev0 == 1) {
        local_farfield_adaptive(b, l, partial, whole);
        for (int j : partial) srcs.emplace_back(j, l);
        for (int j : whole) srcs.emplace_back(j, l - 1);
      } else {
        for (int j : local_farfield(b, l)) srcs.emplace_back(j, l);
      }
      for (const auto &src : srcs) {
        const int j = src.first, lj = src.second;
        int vj[3];
        box_vector(j, lj, vj);
        const double *cj = &g->centers[3 * (size_t)(g->lev_off[lj] + j - 1)];
        double dv[3];
        std::vector<long long> key(4);
        // same level: the box-vector difference; a level - 1 source: the
        // centre difference in half boxes of level l (4 vj - 2 vb + 1)
        key[3] = regular ? (lj == l ? l : -l) : 0;
        for (int d = 0; d < 3; ++d) {
          dv[d] = cj[d] - cb[d];
          if (regular)
            key[d] = lj == l ? vj[d] - vb[d] : 4LL * vj[d] - 2LL * vb[d] + 1;
          else
            std::memcpy(&key[d], &dv[d], 8);
        }
        auto it = disp_index.find(key);
        int di;
        if (it == disp_index.end()) {
          di = (int)disp_index.size();
          disp_index[key] = di;
          disp.insert(disp.end(), dv, dv + 3);
        } else {
          di = it->second;
        }
        ffsrc.push_back(g->lev_off[lj] + j - 1);
        ffdisp.push_back(di);
      }
      ffstart.push_back((int)ffsrc.size());
    }
  if ((double)disp_index.size() * g->N * g->N * 8.0 > 6.0 * (1ull << 30))
    return fail(DAGE_E_UNSUPPORTED,
                "%zu distinct far-field displacements (uneven box split at level %d): the M2L "
                "matrices would exceed 6 GiB; use an evenly divisible grid or fewer levels",
                disp_index.size(), maxlevel);

  // --- M2M/L2L translation displacements (boxes of levels >= 3) ---------------
  {
    std::map<std::vector<long long>, int> tindex;
    std::vector<double> tdisp;
    std::vector<int> m2m_disp;
    for (int l = g->lev0 + 1; l <= maxlevel; ++l)
      for (int i = 1; i <= (1 << (3 * l)); ++i) {
        const double *cc = &g->centers[3 * (size_t)(g->lev_off[l] + i - 1)];
        const double *cp = &g->centers[3 * (size_t)(g->lev_off[l - 1] + (i - 1) / 8)];
        double dv[3];
        std::vector<long long> key(4);
        key[3] = regular ? l : 0;
        for (int d = 0; d < 3; ++d) {
          dv[d] = cc[d] - cp[d];
          if (regular)
            key[d] = (i - 1) % 8;  // the child octant: the displacement of a regular lattice
          else
            std::memcpy(&key[d], &dv[d], 8);
        }
        if (regular) key[1] = key[2] = 0;
        auto it = tindex.find(key);
        int ti;
        if (it == tindex.end()) {
          ti = (int)tindex.size();
          tindex[key] = ti;
          tdisp.insert(tdisp.end(), dv, dv + 3);
        } else {
          ti = it->second;
        }
        m2m_disp.push_back(ti);
      }
    g->nm2m = (int)tindex.size();
    g->m2m_dvec = tdisp;
    if (g->nm2m > 0) {
      const int M = g->N * (g->N + 1) / 2;
      TransTables t;
      translation_tables(lmax, t);
      TmpBuf dd, c1, c2, l1, l2;
      DAGE_TRY(dd.alloc(sizeof(double) * tdisp.size()));
      DAGE_TRY(c1.alloc(sizeof(double) * M));
      DAGE_TRY(c2.alloc(sizeof(double) * M));
      DAGE_TRY(l1.alloc(sizeof(int) * M));
      DAGE_TRY(l2.alloc(sizeof(int) * M));
      DAGE_TRY(g->d_Wm2m.alloc(sizeof(double) * (size_t)g->nm2m * M));
      DAGE_TRY(g->d_m2m_disp.alloc(sizeof(int) * m2m_disp.size()));
      DAGE_CUDA_TRY(cudaMemcpyAsync(dd.ptr, tdisp.data(), sizeof(double) * tdisp.size(), cudaMemcpyHostToDevice, s));
      DAGE_CUDA_TRY(cudaMemcpyAsync(c1.ptr, t.c1.data(), sizeof(double) * M, cudaMemcpyHostToDevice, s));
      DAGE_CUDA_TRY(cudaMemcpyAsync(c2.ptr, t.c2.data(), sizeof(double) * M, cudaMemcpyHostToDevice, s));
      DAGE_CUDA_TRY(cudaMemcpyAsync(l1.ptr, t.lm1.data(), sizeof(int) * M, cudaMemcpyHostToDevice, s));
      DAGE_CUDA_TRY(cudaMemcpyAsync(l2.ptr, t.lm2.data(), sizeof(int) * M, cudaMemcpyHostToDevice, s));
      DAGE_CUDA_TRY(cudaMemcpyAsync(g->d_m2m_disp.ptr, m2m_disp.data(), sizeof(int) * m2m_disp.size(),
                                    cudaMemcpyHostToDevice, s));
      translation_matrices_kernel<<<g->nm2m, 256, sizeof(double) * g->N, s>>>(
          dd.as<double>(), lmax, c1.as<double>(), c2.as<double>(), l1.as<int>(), l2.as<int>(), M,
          g->d_Wm2m.as<double>());
      DAGE_CUDA_TRY(cudaGetLastError());
      DAGE_CUDA_TRY(cudaStreamSynchronize(s));
    }
  }
  g->ndisp = (int)disp_index.size();
  DAGE_TRY(g->d_ffstart.alloc(sizeof(int) * ffstart.size()));
  DAGE_TRY(g->d_ffsrc.alloc(sizeof(int) * std::max<size_t>(1, ffsrc.size())));
  DAGE_TRY(g->d_ffdisp.alloc(sizeof(int) * std::max<size_t>(1, ffdisp.size())));
  DAGE_CUDA_TRY(cudaMemcpyAsync(g->d_ffstart.ptr, ffstart.data(), sizeof(int) * ffstart.size(),
                                cudaMemcpyHostToDevice, s));
  if (!ffsrc.empty()) {
    DAGE_CUDA_TRY(cudaMemcpyAsync(g->d_ffsrc.ptr, ffsrc.data(), sizeof(int) * ffsrc.size(),
                                  cudaMemcpyHostToDevice, s));
    DAGE_CUDA_TRY(cudaMemcpyAsync(g->d_ffdisp.ptr, ffdisp.data(), sizeof(int) * ffdisp.size(),
                                  cudaMemcpyHostToDevice, s));
  }
  DAGE_TRY(build_m2l(g));
  DAGE_TRY(g->d_q.alloc(sizeof(double) * g->nbtot * g->N));
  DAGE_TRY(g->d_L.alloc(sizeof(double) * g->nbtot * g->N));
  DAGE_TRY(g->d_partial.alloc(sizeof(double) * (size_t)g->nbox * g->nslab * g->N));

  // --- near-field sub-operator matrices per axis position --------------------
  TmpBuf d_tp;
  DAGE_TRY(build_quadrature(g->quad, g->tp, g->tw, d_tp, s));
  set_weights(g);
  for (int d = 0; d < 3; ++d) {
    g->Tnear[d].resize(nb);
    g->band_near[d].resize(nb);
    for (int v = 0; v < nb; ++v) {
      const int q0 = pos_near0[d][v], nq = pos_nearn[d][v];
      dage_grid1d sub;
      sub.ncell = (nq - 1) / (nlip - 1);
      sub.nlip = nlip;
      sub.grid_type = g->ax[d].grid_type;
      sub.qmin = g->ax[d].points[q0];
      sub.cell_scales = g->ax[d].h.data() + q0 / (nlip - 1);
      Axis ain;
      DAGE_TRY(make_axis(sub, ain));
      // identical coordinates to the global grid's points: copy them over
      for (int i = 0; i < nq; ++i) ain.points[i] = g->ax[d].points[q0 + i];
      for (int c = 0; c < ain.ncell; ++c) ain.celld[c] = g->ax[d].celld[q0 / (nlip - 1) + c];
      const int own = pos_own[d][v];
      DAGE_TRY(g->Tnear[d][v].alloc(sizeof(double) * (size_t)g->P * own * nq));
      DAGE_TRY(build_axis_matrix(ain, g->ax[d].points.data() + pos_p0[d][v], own,
                                 d_tp.as<double>(), g->P, g->Tnear[d][v].as<double>(), s));
      DAGE_TRY(g->band_near[d][v].alloc(sizeof(int2) * (size_t)g->P * ceil_div(own, kFp64TileN)));
      DAGE_TRY(launch_band(g->Tnear[d][v].as<double>(), nq, own, g->P,
                           g->band_near[d][v].as<int2>(), s));
    }
  }
  // intermediates and stage descriptors
  size_t maxU = 0, maxW = 0;
  for (const auto &B : g->boxes) {
    maxU = std::max(maxU, (size_t)B.nq[1] * B.nq[2] * B.own[0]);
    maxW = std::max(maxW, (size_t)B.nq[2] * B.own[0] * B.own[1]);
  }
  g->U_per_box = maxU;
  g->W_per_box = maxW;
  if (g->precision == DAGE_FP64) {  // the FP64 near field's intermediates
    DAGE_TRY(g->d_U.alloc(sizeof(double) * maxU * g->nbox));
    DAGE_TRY(g->d_W.alloc(sizeof(double) * maxW * g->nbox));
  }
  for (int d = 0; d < 3; ++d) {
    DAGE_TRY(g->wts[d].alloc(sizeof(double) * g->npts[d]));
    DAGE_CUDA_TRY(cudaMemcpyAsync(g->wts[d].ptr, g->ax[d].weights.data(),
                                  sizeof(double) * g->npts[d], cudaMemcpyHostToDevice, s));
    DAGE_TRY(g->d_desc[d].alloc(sizeof(StageDesc) * g->nbox));
  }
  DAGE_TRY(g->d_epart.alloc(sizeof(double) * kEnergyBlocks));
  DAGE_TRY(g->d_energy.alloc(sizeof(double)));
  DAGE_TRY(g->d_inst.alloc(sizeof(GInst)));
  DAGE_CUDA_TRY(cudaStreamSynchronize(s));
  return 0;
}


// ---------------------------------------------------------------------------
// Pipeline pieces shared by the single-density and batched applies
// ---------------------------------------------------------------------------
GInst plan_inst(const dage_gbfmm *g, const double *rho, double *V, double *q, double *L,
                double *partial, double *epart) {
  GInst I{};
  I.rho = rho;
  I.V = V;
  I.q = q;
  I.L = L;
  I.partial = partial;
  I.epart = epart;
  I.boxes = g->d_boxes.as<BoxInfo>();
  I.wbox = g->d_wbox.as<double>();
  I.wstride = g->wstride;
  I.Nx = g->npts[0];
  I.Ny = g->npts[1];
  I.Nz = g->npts[2];
  I.Tm2l = g->d_Tm2l.as<double>();
  I.ffstart = g->d_ffstart.as<int>();
  I.ffsrc = g->d_ffsrc.as<int>();
  I.ffdisp = g->d_ffdisp.as<int>();
  I.wx = g->wts[0].as<double>();
  I.wy = g->wts[1].as<double>();
  I.wz = g->wts[2].as<double>();
  I.kappa = g->kappa;
  I.fine_off = g->fine_off;
  I.m2m_base = g->level > g->lev0 ? g->lev_off[g->lev0 + 1] : 0;
  I.Wm2m = g->d_Wm2m.as<double>();
  I.m2m_disp = g->d_m2m_disp.as<int>();
  I.Wm2m_h = g->d_Wm2m_h.as<double>();
  return I;
}

// Appends the near-field stage descriptors of one density (one per box and
// stage; t-point p reads its matrices at T + p * t_ps) with intermediates
// U (U_per_box per box) and W (W_per_box per box).
void near_descs(const dage_gbfmm *g, const double *rho, double *V, double *U0, double *W0,
                std::vector<StageDesc> ds[3]) {
  const int Nx = g->npts[0], Ny = g->npts[1];
  for (int b = 0; b < g->nbox; ++b) {
    const BoxInfo &B = g->boxes[b];
    double *U = U0 + g->U_per_box * b;
    double *W = W0 + g->W_per_box * b;
    StageDesc x{}, y{}, z{};
    // stage x: rho near region (a: x, rows (b: y, c: z)) -> U(R=(y,z), n=x_own)
    x.M = B.nq[1] * B.nq[2];
    x.N = B.own[0];
    x.K = B.nq[0];
    x.X = rho + B.q0[0] + (size_t)Nx * B.q0[1] + (size_t)Nx * Ny * B.q0[2];
    x.a_d0 = B.nq[1];
    x.a_s1 = Nx;
    x.a_s2 = (long long)Nx * Ny;
    x.T = g->Tnear[0][B.pos[0]].as<double>();
    x.krange = g->band_near[0][B.pos[0]].as<int2>();
    x.kr_ps = ceil_div(B.own[0], kFp64TileN);
    x.t_ps = (long long)B.own[0] * B.nq[0];
    x.ldt = B.nq[0];
    x.out = U;
    x.o_d0 = x.M;
    x.o_s1 = 1;
    x.o_s2 = 0;
    x.o_sn = x.M;
    // stage y: U (K = y near, rows (z near, x own)) -> W(R=(z, x), n=y_own)
    y.M = B.nq[2] * B.own[0];
    y.N = B.own[1];
    y.K = B.nq[1];
    y.X = U;
    y.a_d0 = y.M;
    y.a_s1 = B.nq[1];
    y.a_s2 = 0;
    y.T = g->Tnear[1][B.pos[1]].as<double>();
    y.krange = g->band_near[1][B.pos[1]].as<int2>();
    y.kr_ps = ceil_div(B.own[1], kFp64TileN);
    y.t_ps = (long long)B.own[1] * B.nq[1];
    y.ldt = B.nq[1];
    y.out = W;
    y.o_d0 = y.M;
    y.o_s1 = 1;
    y.o_s2 = 0;
    y.o_sn = y.M;
    // stage z: W (K = z near, rows (x own, y own)) -> V box (owned points)
    z.M = B.own[0] * B.own[1];
    z.N = B.own[2];
    z.K = B.nq[2];
    z.X = W;
    z.a_d0 = z.M;
    z.a_s1 = B.nq[2];
    z.a_s2 = 0;
    z.T = g->Tnear[2][B.pos[2]].as<double>();
    z.krange = g->band_near[2][B.pos[2]].as<int2>();
    z.kr_ps = ceil_div(B.own[2], kFp64TileN);
    z.t_ps = (long long)B.own[2] * B.nq[2];
    z.ldt = B.nq[2];
    z.out = V + B.p0[0] + (size_t)Nx * B.p0[1] + (size_t)Nx * Ny * B.p0[2];
    z.o_d0 = B.own[0];
    z.o_s1 = 1;
    z.o_s2 = Nx;
    z.o_sn = (long long)Nx * Ny;
    ds[0].push_back(x);
    ds[1].push_back(y);
    ds[2].push_back(z);
  }
}

// Largest 128-row tile count and column count of each near-field stage over
// the boxes of a plan (a batched launch's grid bounds).
void near_bounds(const dage_gbfmm *g, int mt[3], int nt[3]) {
  const int TM = kFp64TileM;
  for (const auto &B : g->boxes) {
    mt[0] = std::max(mt[0], ceil_div((long long)B.nq[1] * B.nq[2], TM));
    nt[0] = std::max(nt[0], B.own[0]);
    mt[1] = std::max(mt[1], ceil_div((long long)B.nq[2] * B.own[0], TM));
    nt[1] = std::max(nt[1], B.own[1]);
    mt[2] = std::max(mt[2], ceil_div((long long)B.own[0] * B.own[1], TM));
    nt[2] = std::max(nt[2], B.own[2]);
  }
}

int max_owned(const dage_gbfmm *g) {
  int m = 0;
  for (const auto &B : g->boxes) m = std::max(m, B.own[0] * B.own[1] * B.own[2]);
  return m;
}

int run_multipoles(const GInst *d_inst, int ninst, int nbox, int lmax, int nslab, bool helm,
                   cudaStream_t s) {
  const int N = (lmax + 1) * (lmax + 1);
  if (helm)
    multipoles_kernel<true><<<dim3(nbox, nslab, ninst), kMpWarps * 32, 0, s>>>(d_inst, lmax, nslab);
  else
    multipoles_kernel<false><<<dim3(nbox, nslab, ninst), kMpWarps * 32, 0, s>>>(d_inst, lmax, nslab);
  DAGE_CUDA_TRY(cudaGetLastError());
  reduce_slabs_kernel<<<dim3((nbox * N + 255) / 256, ninst), 256, 0, s>>>(d_inst, nslab, N, nbox);
  DAGE_CUDA_TRY(cudaGetLastError());
  return 0;
}

int run_m2l(const GInst *d_inst, int ninst, int nbox, int N, cudaStream_t s) {
  const int npad = ((N + 31) / 32) * 32;           // N <= 256
  const int groups = std::max(1, std::min(8, 1024 / npad));
  m2l_apply_kernel<<<dim3(nbox, ninst), npad * groups, sizeof(double) * N * 2 * groups, s>>>(
      d_inst, N, npad);
  DAGE_CUDA_TRY(cudaGetLastError());
  return 0;
}

// Upward pass from the finest level to level 2 (1 in the adaptive mode).
int run_m2m(const GInst *d_inst, int ninst, const dage_gbfmm *g, cudaStream_t s) {
  const int threads = std::min(256, ((g->N + 31) / 32) * 32);
  for (int l = g->level - 1; l >= g->lev0; --l) {
    m2m_kernel<<<dim3(1 << (3 * l), ninst), threads, 0, s>>>(d_inst, g->N, g->lev_off[l],
                                                            g->lev_off[l + 1]);
    DAGE_CUDA_TRY(cudaGetLastError());
  }
  return 0;
}

// Downward pass from level 3 to the finest level, after the M2L of all levels.
int run_l2l(const GInst *d_inst, int ninst, const dage_gbfmm *g, cudaStream_t s) {
  const int threads = std::min(256, ((g->N + 31) / 32) * 32);
  for (int l = 3; l <= g->level; ++l) {
    l2l_kernel<<<dim3(1 << (3 * l), ninst), threads, 0, s>>>(d_inst, g->N, g->lev_off[l - 1],
                                                            g->lev_off[l]);
    DAGE_CUDA_TRY(cudaGetLastError());
  }
  return 0;
}

// Coulomb instances run l2p_kernel, Helmholtz instances (when `helm`)
// l2p_helm_kernel; each kernel returns at once on the other kind.
int run_l2p(const GInst *d_inst, int ninst, int nbox, int lmax, int maxown, const double *Lext,
            bool helm, cudaStream_t s) {
  const int N = (lmax + 1) * (lmax + 1);
  const int bx = std::min((maxown + 127) / 128, 64);
  l2p_kernel<<<dim3(bx, nbox, ninst), 128, sizeof(double) * N, s>>>(d_inst, Lext, lmax);
  DAGE_CUDA_TRY(cudaGetLastError());
  if (helm) {
    const int pts = kL2pHelmThreads;  // points per block pass (one per thread)
    const int hx = std::min((maxown + pts - 1) / pts, 256);
    l2p_helm_kernel<<<dim3(hx, nbox, ninst), kL2pHelmThreads, 0, s>>>(d_inst, Lext, lmax);
    DAGE_CUDA_TRY(cudaGetLastError());
  }
  return 0;
}

int run_near(const StageDesc *const d_desc[3], int njobs, const int mt[3], const int nt[3], int P,
             const std::vector<double> &w, const int tile_n[3], cudaStream_t s) {
  for (int p = 0; p < P; ++p)
    for (int st = 0; st < 3; ++st)
      DAGE_TRY(launch_fp64_stages(d_desc[st], njobs, mt[st], nt[st], p, st < 2 ? 1.0 : w[p],
                                  st == 2 && p > 0, s, tile_n[st]));
  return 0;
}

int run_energy(const GInst *d_inst, int ninst, double *d_out, cudaStream_t s) {
  energy_kernel<<<dim3(kEnergyBlocks, ninst), 256, 0, s>>>(d_inst);
  DAGE_CUDA_TRY(cudaGetLastError());
  energy_sum_kernel<<<ninst, 32, 0, s>>>(d_inst, d_out);
  DAGE_CUDA_TRY(cudaGetLastError());
  return 0;
}

// Autotuner: the tile width (32, 64 or 128 columns) of each near-field
// stage, chosen by timing every candidate on a batched launch of t-point 0
// (one warm-up, three timed launches; the launches write the intermediates
// and the output cubes of the descriptors, which the caller overwrites).
int autotune_tiles(const StageDesc *const d_desc[3], int njobs, const int mt[3], const int nt[3],
                   cudaStream_t s, int tile_n[3]) {
  cudaEvent_t e0, e1;
  DAGE_CUDA_TRY(cudaEventCreate(&e0));
  DAGE_CUDA_TRY(cudaEventCreate(&e1));
  const int cand[3] = {32, 64, 128};
  int rc = 0;
  for (int st = 0; st < 3 && !rc; ++st) {
    float best = std::numeric_limits<float>::max();
    for (int tn : cand) {
      for (int r = 0; r < 4 && !rc; ++r) {
        if (r == 1) cudaEventRecord(e0, s);
        rc = launch_fp64_stages(d_desc[st], njobs, mt[st], nt[st], 0, 1.0, false, s, tn);
      }
      if (rc) break;
      cudaEventRecord(e1, s);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best) {
        best = ms;
        tile_n[st] = tn;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

// Key of a plan in the tune cache: device, points per axis, t-points, boxes.
std::string plan_key(const dage_gbfmm *g, const char *what) {
  return tune_device_key() + "/" + what + "/" + std::to_string(g->npts[0]) + "x" +
         std::to_string(g->npts[1]) + "x" + std::to_string(g->npts[2]) + ",P" +
         std::to_string(g->P) + ",boxes" + std::to_string(g->nbox);
}

// The plan's own tiles, from the tune cache or tuned on scratch input and
// output cubes.
int gbfmm_autotune(dage_gbfmm *g) {
  const std::string key = plan_key(g, "gbfmm_near_fp64");
  std::vector<int> v;
  if (tune_lookup(key, v) && v.size() == 3) {
    for (int d = 0; d < 3; ++d) g->tile_n[d] = v[d];
    return 0;
  }
  cudaStream_t s = g->stream;
  const size_t n = (size_t)g->npts[0] * g->npts[1] * g->npts[2];
  TmpBuf rho, V;
  DAGE_TRY(rho.alloc(sizeof(double) * n));
  DAGE_TRY(V.alloc(sizeof(double) * n));
  DAGE_CUDA_TRY(cudaMemsetAsync(rho.ptr, 0, sizeof(double) * n, s));
  std::vector<StageDesc> ds[3];
  near_descs(g, rho.as<double>(), V.as<double>(), g->d_U.as<double>(), g->d_W.as<double>(), ds);
  for (int d = 0; d < 3; ++d)
    DAGE_CUDA_TRY(cudaMemcpyAsync(g->d_desc[d].ptr, ds[d].data(), sizeof(StageDesc) * g->nbox,
                                  cudaMemcpyHostToDevice, s));
  int mt[3] = {0, 0, 0}, nt[3] = {0, 0, 0};
  near_bounds(g, mt, nt);
  const StageDesc *dd[3] = {g->d_desc[0].as<StageDesc>(), g->d_desc[1].as<StageDesc>(),
                            g->d_desc[2].as<StageDesc>()};
  const int rc = autotune_tiles(dd, g->nbox, mt, nt, s, g->tile_n);
  DAGE_CUDA_TRY(cudaStreamSynchronize(s));
  rho.release();
  V.release();
  if (rc) return rc;
  tune_store(key, {g->tile_n[0], g->tile_n[1], g->tile_n[2]});
  return 0;
}

// --- fp16x3 near field (near_mixed.cu) ---------------------------------------
NearGeom near_geom(const dage_gbfmm *g) {
  NearGeom G;
  G.P = g->P;
  const int nb = 1 << g->level;
  for (int d = 0; d < 3; ++d) {
    G.npts[d] = g->npts[d];
    G.q0[d].assign(nb, 0);
    G.nq[d].assign(nb, 0);
    G.own[d].assign(nb, 0);
    G.p0[d].assign(nb, 0);
    for (const auto &B : g->boxes) {
      const int v = B.pos[d];
      G.q0[d][v] = B.q0[d];
      G.nq[d][v] = B.nq[d];
      G.own[d][v] = B.own[d];
      G.p0[d][v] = B.p0[d];
    }
    for (int v = 0; v < nb; ++v) {
      G.T[d].push_back(g->Tnear[d][v].as<double>());
      G.band[d].push_back(g->band_near[d][v].as<int2>());
    }
  }
  return G;
}

std::vector<NearBox> near_boxes(const dage_gbfmm *g) {
  std::vector<NearBox> v;
  for (const auto &B : g->boxes) v.push_back(NearBox{{B.pos[0], B.pos[1], B.pos[2]}});
  return v;
}

// the near-field weights w_p on the device
int upload_near_w(dage_gbfmm *g) {
  DAGE_TRY(g->d_wn.alloc(sizeof(double) * g->P));
  DAGE_CUDA_TRY(cudaMemcpyAsync(g->d_wn.ptr, g->w.data(), sizeof(double) * g->P,
                                cudaMemcpyHostToDevice, g->stream));
  DAGE_CUDA_TRY(cudaStreamSynchronize(g->stream));
  return 0;
}

// Tile width of the fp16x3 near field (64 or 128 output columns), chosen by
// timing one near-field pass of each on scratch cubes; kept in the tune
// cache per (device, points per axis, t-points, boxes).
int near16_tune(dage_gbfmm *g, int *tile) {
  // DAGE_NEAR16_TILE=64|128 fixes the width (tests of both code paths)
  if (const char *e = std::getenv("DAGE_NEAR16_TILE")) {
    *tile = std::atoi(e) == 128 ? 128 : 64;
    return 0;
  }
  const std::string key = plan_key(g, "gbfmm_near_fp16x3");
  std::vector<int> v;
  if (tune_lookup(key, v) && v.size() == 1) {
    *tile = v[0];
    return 0;
  }
  cudaStream_t s = g->stream;
  const size_t n = (size_t)g->npts[0] * g->npts[1] * g->npts[2];
  TmpBuf rho, V;
  DAGE_TRY(rho.alloc(sizeof(double) * n));
  DAGE_TRY(V.alloc(sizeof(double) * n));
  DAGE_CUDA_TRY(cudaMemsetAsync(rho.ptr, 0, sizeof(double) * n, s));
  cudaEvent_t e0, e1;
  DAGE_CUDA_TRY(cudaEventCreate(&e0));
  DAGE_CUDA_TRY(cudaEventCreate(&e1));
  const auto boxes = near_boxes(g);
  float best = std::numeric_limits<float>::max();
  int rc = 0;
  for (int tn : {64, 128}) {
    NearF16Set *set = nullptr;
    rc = near_f16_set_create(&set, g->near16, boxes, 1, tn, s);
    const double *rr[1] = {rho.as<double>()};
    double *vv[1] = {V.as<double>()};
    const double *ww[1] = {g->d_wn.as<double>()};
    if (!rc) rc = near_f16_set_bind(set, rr, vv, ww, s);
    for (int r = 0; r < 3 && !rc; ++r) {
      if (r == 1) cudaEventRecord(e0, s);
      rc = near_f16_set_run(set, s);
    }
    if (!rc) {
      cudaEventRecord(e1, s);
      rc = near_f16_set_check(set, s);
    }
    float ms = 0.f;
    if (!rc) cudaEventElapsedTime(&ms, e0, e1);
    near_f16_set_destroy(set);
    if (rc) break;
    if (ms < best) {
      best = ms;
      *tile = tn;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  tune_store(key, {*tile});
  return 0;
}

// FP16 matrix parts, weights and tile width; with `single`, the set of the
// single-density apply.
int near16_init(dage_gbfmm *g, bool single) {
  DAGE_TRY(near_f16_prepare());
  DAGE_TRY(near_f16_plan_create(&g->near16, near_geom(g), g->stream));
  DAGE_TRY(upload_near_w(g));
  int tile = 64;
  DAGE_TRY(near16_tune(g, &tile));
  for (int d = 0; d < 3; ++d) g->tile_n[d] = tile;
  if (single) DAGE_TRY(near_f16_set_create(&g->near16set, g->near16, near_boxes(g), 1, tile, g->stream));
  return 0;
}

// Uploads the single-density instance table and, for a full apply, the
// near-field descriptors.
int single_setup(dage_gbfmm *g, const double *rho, double *V, bool near) {
  const GInst I = plan_inst(g, rho, V, g->d_q.as<double>(), g->d_L.as<double>(),
                            g->d_partial.as<double>(), g->d_epart.as<double>());
  DAGE_CUDA_TRY(cudaMemcpyAsync(g->d_inst.ptr, &I, sizeof(GInst), cudaMemcpyHostToDevice, g->stream));
  if (near) {
    std::vector<StageDesc> ds[3];
    near_descs(g, rho, V, g->d_U.as<double>(), g->d_W.as<double>(), ds);
    for (int d = 0; d < 3; ++d)
      DAGE_CUDA_TRY(cudaMemcpyAsync(g->d_desc[d].ptr, ds[d].data(), sizeof(StageDesc) * g->nbox,
                                    cudaMemcpyHostToDevice, g->stream));
  }
  // the host copies above are pageable: finish them before the vectors go
  DAGE_CUDA_TRY(cudaStreamSynchronize(g->stream));
  return 0;
}

void gbfmm_destroy_impl(dage_gbfmm *g) {
  if (!g) return;
  if (g->stream) cudaStreamSynchronize(g->stream);
  near_f16_set_destroy(g->near16set);
  near_f16_plan_destroy(g->near16);
  g->d_wn.release();
  g->d_Wm2m_h.release();
  for (int d = 0; d < 3; ++d) {
    for (auto &b : g->Tnear[d]) b.release();
    for (auto &b : g->band_near[d]) b.release();
    g->d_desc[d].release();
    g->wts[d].release();
  }
  for (DevBuf *b : {&g->d_boxes, &g->d_wbox, &g->d_q, &g->d_L, &g->d_partial, &g->d_Tm2l,
                    &g->d_ffstart, &g->d_ffsrc, &g->d_ffdisp, &g->d_U, &g->d_W, &g->d_epart,
                    &g->d_energy, &g->d_inst, &g->d_rho, &g->d_V})
    b->release();
  if (g->ev0) cudaEventDestroy(g->ev0);
  if (g->ev1) cudaEventDestroy(g->ev1);
  if (g->own_stream) cudaStreamDestroy(g->own_stream);
  delete g;
}

// device pointers for rho / V (staging host buffers when needed)
int stage_io(dage_gbfmm *g, const double *rho, double *V, unsigned flags, const double **d_rho,
             double **d_V) {
  const size_t n = (size_t)g->npts[0] * g->npts[1] * g->npts[2];
  if (flags & DAGE_DEVICE_PTRS) {
    *d_rho = rho;
    *d_V = V;
    return 0;
  }
  DAGE_TRY(g->d_rho.alloc(sizeof(double) * n));
  DAGE_TRY(g->d_V.alloc(sizeof(double) * n));
  if (rho)
    DAGE_CUDA_TRY(cudaMemcpyAsync(g->d_rho.ptr, rho, sizeof(double) * n, cudaMemcpyHostToDevice,
                                  g->stream));
  *d_rho = g->d_rho.as<double>();
  *d_V = g->d_V.as<double>();
  return 0;
}

}  // namespace

// ---------------------------------------------------------------------------
// Batch of independent densities (grids of any sizes): densities on equal
// grids share one plan; every pipeline stage is one launch over all of them,
// except the near field, whose intermediates are processed in chunks of
// densities that fit a memory budget.
// ---------------------------------------------------------------------------
struct dage_gbfmm_batch {
  int device = 0, n = 0, lmax = 0, N = 0, P = 0, nbox = 0, nslab = 8;
  std::vector<dage_gbfmm *> plans;
  std::vector<int> plan_of;
  std::vector<size_t> npts;   // points of each density
  std::vector<double> w;      // t-point weights (shared quadrature)
  DevBuf q, L, partial, epart, energy, inst;
  struct Chunk {
    int i0 = 0, i1 = 0, njobs = 0;
    DevBuf desc[3];
    std::vector<size_t> uoff, woff;  // per density: offsets into U, W
  };
  std::vector<Chunk> chunks;
  DevBuf U, W;
  // fp16x3 near field: sets of densities of one plan each, within the budget
  int precision = DAGE_FP64;
  struct MSet {
    int plan = 0;
    std::vector<int> dens;
    NearF16Set *set = nullptr;
  };
  std::vector<MSet> msets;
  DevBuf ws16[3];  // the sets' shared workspace: split input, U, W
  int mt[3] = {0, 0, 0}, nt[3] = {0, 0, 0}, maxown = 0;
  int tile_n[3] = {64, 64, 64};
  bool tuned = false;
  DevBuf stage_rho, stage_V;  // host-pointer mode
  std::vector<size_t> stage_off;
  cudaStream_t own_stream = nullptr, stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_ms = 0.f;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  size_t graph_nodes = 0;
  std::vector<const void *> graph_key;  // rho/V pointers the graph was captured for
  // Helmholtz kernels: one per distinct (plan, energy < 0); densities with
  // energy 0 use their plan's Coulomb matrices and the Coulomb weights
  struct Kern {
    int plan = 0;
    double energy = 0.0;
    DevBuf T, w;  // M2L matrices of the plan's displacements; near-field weights
    DevBuf Wh;    // Helmholtz M2M matrices (maxlevel >= 3)
  };
  std::vector<Kern> kerns;
  std::vector<int> kern_of;  // per density, -1: Coulomb
  // optional first pipeline stage: rho_i += inject_factor[i] * bubbles
  const dage_bubbles *bubbles = nullptr;
  int inject_lmin = 0;
  std::vector<double> inject_factor;
};

namespace dage {
namespace {

bool same_grid(const dage_gbfmm *g, const dage_grid1d grid[3]) {
  for (int d = 0; d < 3; ++d) {
    Axis a;
    if (make_axis(grid[d], a)) return false;
    if (!same_axis(a, g->ax[d])) return false;
  }
  return true;
}

void batch_destroy_impl(dage_gbfmm_batch *b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (auto &m : b->msets) near_f16_set_destroy(m.set);
  for (auto *g : b->plans) gbfmm_destroy_impl(g);
  for (auto &c : b->chunks)
    for (auto &d : c.desc) d.release();
  for (auto &k : b->kerns) {
    k.T.release();
    k.w.release();
    k.Wh.release();
  }
  for (DevBuf *d : {&b->q, &b->L, &b->partial, &b->epart, &b->energy, &b->inst, &b->U, &b->W,
                    &b->ws16[0], &b->ws16[1], &b->ws16[2], &b->stage_rho, &b->stage_V})
    d->release();
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->own_stream) cudaStreamDestroy(b->own_stream);
  delete b;
}

int batch_create_impl(dage_gbfmm_batch *b, int n, const dage_grid1d *grids, int maxlevel, int lmax,
                      const dage_quad *quad, int precision, size_t budget) {
  DAGE_CUDA_TRY(cudaGetDevice(&b->device));
  DAGE_CUDA_TRY(cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking));
  b->stream = b->own_stream;
  DAGE_CUDA_TRY(cudaEventCreate(&b->ev0));
  DAGE_CUDA_TRY(cudaEventCreate(&b->ev1));
  b->n = n;
  b->plan_of.resize(n);
  b->kern_of.assign(n, -1);
  for (int i = 0; i < n; ++i) {
    const dage_grid1d *gi = grids + 3 * i;
    int found = -1;
    for (size_t k = 0; k < b->plans.size() && found < 0; ++k)
      if (same_grid(b->plans[k], gi)) found = (int)k;
    if (found < 0) {
      auto *g = new dage_gbfmm();
      g->precision = precision;
      int rc = gbfmm_create_impl(g, gi, maxlevel, lmax, quad);
      if (!rc && precision != DAGE_FP64) rc = near16_init(g, false);
      if (rc) {
        gbfmm_destroy_impl(g);
        return rc;
      }
      b->plans.push_back(g);
      found = (int)b->plans.size() - 1;
    }
    b->plan_of[i] = found;
    const dage_gbfmm *g = b->plans[found];
    b->npts.push_back((size_t)g->npts[0] * g->npts[1] * g->npts[2]);
  }
  const dage_gbfmm *g0 = b->plans[0];
  b->lmax = lmax;
  b->N = g0->N;
  b->P = g0->P;
  b->nbox = g0->nbox;
  b->nslab = n >= 8 ? 4 : g0->nslab;  // many densities fill the GPU with fewer slabs
  b->w = g0->w;
  for (const auto *g : b->plans) {
    near_bounds(g, b->mt, b->nt);
    b->maxown = std::max(b->maxown, max_owned(g));
  }
  const size_t per = (size_t)g0->nbtot * b->N;  // every level's boxes
  DAGE_TRY(b->q.alloc(sizeof(double) * per * n));
  DAGE_TRY(b->L.alloc(sizeof(double) * per * n));
  DAGE_TRY(b->partial.alloc(sizeof(double) * (size_t)b->nbox * b->N * b->nslab * n));
  DAGE_TRY(b->epart.alloc(sizeof(double) * kEnergyBlocks * n));
  DAGE_TRY(b->energy.alloc(sizeof(double) * n));
  DAGE_TRY(b->inst.alloc(sizeof(GInst) * n));
  b->precision = precision;
  if (precision != DAGE_FP64) {
    // per plan: consecutive densities of the plan while the set fits the budget
    for (size_t k = 0; k < b->plans.size(); ++k) {
      const auto boxes = near_boxes(b->plans[k]);
      dage_gbfmm_batch::MSet cur;
      cur.plan = (int)k;
      for (int i = 0; i < n; ++i) {
        if (b->plan_of[i] != (int)k) continue;
        if (!cur.dens.empty() &&
            near_f16_set_bytes(b->plans[k]->near16, boxes, (int)cur.dens.size() + 1) > budget) {
          b->msets.push_back(cur);
          cur.dens.clear();
        }
        cur.dens.push_back(i);
      }
      if (!cur.dens.empty()) b->msets.push_back(cur);
    }
    // one workspace for all sets (they run one after another on the stream)
    size_t wsb[3] = {0, 0, 0};
    for (auto &m : b->msets) {
      const dage_gbfmm *g = b->plans[m.plan];
      size_t sb[3];
      near_f16_set_sizes(g->near16, near_boxes(g), (int)m.dens.size(), sb);
      for (int k = 0; k < 3; ++k) wsb[k] = std::max(wsb[k], sb[k]);
    }
    void *ws[3];
    for (int k = 0; k < 3; ++k) {
      DAGE_TRY(b->ws16[k].alloc(wsb[k]));
      DAGE_CUDA_TRY(cudaMemsetAsync(b->ws16[k].ptr, 0, wsb[k], b->stream));
      ws[k] = b->ws16[k].ptr;
    }
    for (auto &m : b->msets) {
      const dage_gbfmm *g = b->plans[m.plan];
      DAGE_TRY(near_f16_set_create(&m.set, g->near16, near_boxes(g), (int)m.dens.size(),
                                   g->tile_n[0], b->stream, ws));
    }
    for (int d = 0; d < 3; ++d) b->tile_n[d] = b->plans[0]->tile_n[d];
    b->tuned = true;
    for (auto *g : b->plans) g->stream = b->stream;
    return 0;
  }
  // near-field chunks: consecutive densities while their intermediates fit
  size_t umax = 0, wmax = 0, ucur = 0, wcur = 0;
  dage_gbfmm_batch::Chunk cur;
  for (int i = 0; i < n; ++i) {
    const dage_gbfmm *g = b->plans[b->plan_of[i]];
    const size_t ui = g->U_per_box * b->nbox, wi = g->W_per_box * b->nbox;
    const bool full = cur.i1 > cur.i0 &&
                      ((ucur + ui + wcur + wi) * sizeof(double) > budget ||
                       (long long)(cur.i1 - cur.i0 + 1) * b->nbox > 65535);
    if (full) {
      b->chunks.push_back(std::move(cur));
      cur = dage_gbfmm_batch::Chunk();
      cur.i0 = cur.i1 = i;
      ucur = wcur = 0;
    }
    cur.uoff.push_back(ucur);
    cur.woff.push_back(wcur);
    ucur += ui;
    wcur += wi;
    cur.i1 = i + 1;
    umax = std::max(umax, ucur);
    wmax = std::max(wmax, wcur);
  }
  b->chunks.push_back(std::move(cur));
  DAGE_TRY(b->U.alloc(sizeof(double) * std::max<size_t>(umax, 1)));
  DAGE_TRY(b->W.alloc(sizeof(double) * std::max<size_t>(wmax, 1)));
  for (auto &c : b->chunks) {
    c.njobs = (c.i1 - c.i0) * b->nbox;
    for (auto &d : c.desc) DAGE_TRY(d.alloc(sizeof(StageDesc) * c.njobs));
  }
  // plans share the batch's stream
  for (auto *g : b->plans) g->stream = b->stream;
  return 0;
}

// Instance tables and near-field descriptors for a set of device cubes.
int batch_tables(dage_gbfmm_batch *b, const double *const *rho, double *const *V) {
  const size_t per = (size_t)b->plans[0]->nbtot * b->N;  // every level's boxes
  std::vector<GInst> ins(b->n);
  for (int i = 0; i < b->n; ++i) {
    ins[i] = plan_inst(b->plans[b->plan_of[i]], rho[i], V[i], b->q.as<double>() + per * i,
                       b->L.as<double>() + per * i,
                       b->partial.as<double>() + (size_t)b->nbox * b->N * b->nslab * i,
                       b->epart.as<double>() + (size_t)kEnergyBlocks * i);
    if (b->kern_of[i] >= 0) {
      const auto &k = b->kerns[b->kern_of[i]];
      ins[i].kappa = std::sqrt(-2.0 * k.energy);
      ins[i].Tm2l = k.T.as<double>();
      ins[i].Wm2m_h = k.Wh.as<double>();
    }
  }
  DAGE_CUDA_TRY(cudaMemcpyAsync(b->inst.ptr, ins.data(), sizeof(GInst) * b->n,
                                cudaMemcpyHostToDevice, b->stream));
  for (auto &m : b->msets) {
    std::vector<const double *> rr, ww;
    std::vector<double *> vv;
    for (int i : m.dens) {
      rr.push_back(rho[i]);
      vv.push_back(V[i]);
      ww.push_back(b->kern_of[i] >= 0 ? b->kerns[b->kern_of[i]].w.as<double>()
                                      : b->plans[m.plan]->d_wn.as<double>());
    }
    DAGE_TRY(near_f16_set_bind(m.set, rr.data(), vv.data(), ww.data(), b->stream));
  }
  std::vector<std::vector<StageDesc>> keep;
  for (auto &c : b->chunks) {
    std::vector<StageDesc> ds[3];
    for (int i = c.i0; i < c.i1; ++i) {
      const size_t z0 = ds[2].size();
      near_descs(b->plans[b->plan_of[i]], rho[i], V[i], b->U.as<double>() + c.uoff[i - c.i0],
                 b->W.as<double>() + c.woff[i - c.i0], ds);
      if (b->kern_of[i] >= 0)  // this density's own t-point weights in the z stage
        for (size_t e = z0; e < ds[2].size(); ++e) ds[2][e].wp = b->kerns[b->kern_of[i]].w.as<double>();
    }
    for (int d = 0; d < 3; ++d)
      DAGE_CUDA_TRY(cudaMemcpyAsync(c.desc[d].ptr, ds[d].data(), sizeof(StageDesc) * c.njobs,
                                    cudaMemcpyHostToDevice, b->stream));
    for (int d = 0; d < 3; ++d) keep.push_back(std::move(ds[d]));
  }
  // the host copies are pageable: finish them before the vectors go
  DAGE_CUDA_TRY(cudaStreamSynchronize(b->stream));
  return 0;
}

// The whole pipeline for the current tables, as stream work (captured into
// the graph or launched directly).
int batch_launch(dage_gbfmm_batch *b, const double *const *rho, double *const *V) {
  cudaStream_t s = b->stream;
  const GInst *d_inst = b->inst.as<GInst>();
  if (b->bubbles)
    for (int i = 0; i < b->n; ++i) {
      if (b->inject_factor[i] == 0.0) continue;
      const dage_gbfmm *g = b->plans[b->plan_of[i]];
      const double *xs = g->d_wbox.as<double>() + (size_t)3 * 64 * g->wstride;
      DAGE_TRY(bubbles_inject_launch(b->bubbles, xs, g->npts[0], xs + g->wstride, g->npts[1],
                                     xs + 2 * g->wstride, g->npts[2], b->inject_lmin,
                                     b->inject_factor[i], const_cast<double *>(rho[i]), s));
    }
  for (int i = 0; i < b->n; ++i)
    DAGE_CUDA_TRY(cudaMemsetAsync(V[i], 0, sizeof(double) * b->npts[i], s));
  bool any_helm = false;
  for (int i = 0; i < b->n; ++i) any_helm |= b->kern_of[i] >= 0;
  DAGE_TRY(run_multipoles(d_inst, b->n, b->nbox, b->lmax, b->nslab, any_helm, s));
  DAGE_TRY(run_m2m(d_inst, b->n, b->plans[0], s));
  DAGE_TRY(run_m2l(d_inst, b->n, b->plans[0]->nbtot, b->N, s));
  DAGE_TRY(run_l2l(d_inst, b->n, b->plans[0], s));
  for (auto &c : b->chunks) {
    const StageDesc *dd[3] = {c.desc[0].as<StageDesc>(), c.desc[1].as<StageDesc>(),
                              c.desc[2].as<StageDesc>()};
    DAGE_TRY(run_near(dd, c.njobs, b->mt, b->nt, b->P, b->w, b->tile_n, s));
  }
  for (auto &m : b->msets) DAGE_TRY(near_f16_set_run(m.set, s));
  DAGE_TRY(run_l2p(d_inst, b->n, b->nbox, b->lmax, b->maxown, nullptr, any_helm, s));
  DAGE_TRY(run_energy(d_inst, b->n, b->energy.as<double>(), s));
  return 0;
}

}  // namespace
}  // namespace dage

extern "C" {

int dage_gbfmm_create(const dage_grid1d grid[3], int maxlevel, int lmax, const dage_quad *quad,
                      int precision, dage_gbfmm **out) {
  clear_error();
  if (!out) return fail(DAGE_E_INVALID, "null output handle pointer");
  *out = nullptr;
  if (precision != DAGE_FP64 && precision != DAGE_MIXED_FP16X3)
    return fail(DAGE_E_UNSUPPORTED,
                "the GBFMM operator runs in DAGE_FP64 or DAGE_MIXED_FP16X3 (near field)");
  auto *g = new dage_gbfmm();
  g->precision = precision;
  int rc = gbfmm_create_impl(g, grid, maxlevel, lmax, quad);
  if (!rc) rc = precision == DAGE_FP64 ? gbfmm_autotune(g) : near16_init(g, true);
  if (rc) {
    gbfmm_destroy_impl(g);
    return rc;
  }
  *out = g;
  return 0;
}

int dage_gbfmm_create_adaptive(const dage_grid1d grid[3], int maxlevel, int lmax,
                               const dage_quad *quad, int precision, dage_gbfmm **out) {
  clear_error();
  if (!out) return fail(DAGE_E_INVALID, "null output handle pointer");
  *out = nullptr;
  if (precision != DAGE_FP64 && precision != DAGE_MIXED_FP16X3)
    return fail(DAGE_E_UNSUPPORTED,
                "the GBFMM operator runs in DAGE_FP64 or DAGE_MIXED_FP16X3 (near field)");
  auto *g = new dage_gbfmm();
  g->precision = precision;
  g->lev0 = 1;
  int rc = gbfmm_create_impl(g, grid, maxlevel, lmax, quad);
  if (!rc) rc = precision == DAGE_FP64 ? gbfmm_autotune(g) : near16_init(g, true);
  if (rc) {
    gbfmm_destroy_impl(g);
    return rc;
  }
  *out = g;
  return 0;
}

int dage_gbfmm_destroy(dage_gbfmm *g) {
  clear_error();
  gbfmm_destroy_impl(g);
  return 0;
}

int dage_gbfmm_set_stream(dage_gbfmm *g, void *stream) {
  if (!g) return fail(DAGE_E_INVALID, "null handle");
  g->stream = stream ? (cudaStream_t)stream : g->own_stream;
  return 0;
}

int dage_gbfmm_set_energy(dage_gbfmm *g, double energy) {
  clear_error();
  if (!g) return fail(DAGE_E_INVALID, "null handle");
  if (!(energy <= 0.0)) return fail(DAGE_E_INVALID, "energy must be <= 0 (got %g)", energy);
  DAGE_CUDA_TRY(cudaSetDevice(g->device));
  g->energy = energy;
  g->kappa = energy < 0.0 ? std::sqrt(-2.0 * energy) : 0.0;
  set_weights(g);
  if (g->near16) DAGE_TRY(upload_near_w(g));
  DAGE_TRY(build_helm_m2m_into(g, g->kappa, g->d_Wm2m_h));
  return build_m2l(g);
}

int dage_gbfmm_tiles(const dage_gbfmm *g, int tile_n[3]) {
  if (!g || !tile_n) return fail(DAGE_E_INVALID, "null argument");
  for (int d = 0; d < 3; ++d) tile_n[d] = g->tile_n[d];
  return 0;
}

int dage_gbfmm_box_count(const dage_gbfmm *g, int *nbox, int *nlm) {
  if (!g) return fail(DAGE_E_INVALID, "null handle");
  if (nbox) *nbox = g->nbox;
  if (nlm) *nlm = g->N;
  return 0;
}

int dage_gbfmm_apply(dage_gbfmm *g, const double *rho, double *V, unsigned flags,
                     double *energy) {
  clear_error();
  if (!g || !rho || !V) return fail(DAGE_E_INVALID, "null argument");
  if ((flags & DAGE_ENERGY) && !energy) return fail(DAGE_E_INVALID, "energy pointer is null");
  DAGE_CUDA_TRY(cudaSetDevice(g->device));
  cudaStream_t s = g->stream;
  const size_t n = (size_t)g->npts[0] * g->npts[1] * g->npts[2];
  DAGE_CUDA_TRY(cudaEventRecord(g->ev0, s));
  const double *d_rho;
  double *d_V;
  DAGE_TRY(stage_io(g, rho, V, flags, &d_rho, &d_V));
  if (g->near16set) {
    const double *rr[1] = {d_rho};
    double *vv[1] = {d_V};
    const double *ww[1] = {g->d_wn.as<double>()};
    DAGE_TRY(near_f16_set_bind(g->near16set, rr, vv, ww, s));
  }
  DAGE_TRY(single_setup(g, d_rho, d_V, g->near16set == nullptr));
  const GInst *d_inst = g->d_inst.as<GInst>();
  DAGE_CUDA_TRY(cudaMemsetAsync(d_V, 0, sizeof(double) * n, s));
  DAGE_TRY(run_multipoles(d_inst, 1, g->nbox, g->lmax, g->nslab, g->kappa > 0.0, s));
  DAGE_TRY(run_m2m(d_inst, 1, g, s));
  DAGE_TRY(run_m2l(d_inst, 1, g->nbtot, g->N, s));
  DAGE_TRY(run_l2l(d_inst, 1, g, s));
  if (g->near16set) {
    DAGE_TRY(near_f16_set_run(g->near16set, s));
  } else {
    int mt[3] = {0, 0, 0}, nt[3] = {0, 0, 0};
    near_bounds(g, mt, nt);
    const StageDesc *dd[3] = {g->d_desc[0].as<StageDesc>(), g->d_desc[1].as<StageDesc>(),
                              g->d_desc[2].as<StageDesc>()};
    DAGE_TRY(run_near(dd, g->nbox, mt, nt, g->P, g->w, g->tile_n, s));
  }
  DAGE_TRY(run_l2p(d_inst, 1, g->nbox, g->lmax, max_owned(g), nullptr, g->kappa > 0.0, s));
  if (flags & DAGE_ENERGY) DAGE_TRY(run_energy(d_inst, 1, g->d_energy.as<double>(), s));
  if (!(flags & DAGE_DEVICE_PTRS))
    DAGE_CUDA_TRY(cudaMemcpyAsync(V, d_V, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  if (flags & DAGE_ENERGY)
    DAGE_CUDA_TRY(cudaMemcpyAsync(energy, g->d_energy.ptr, sizeof(double), cudaMemcpyDeviceToHost, s));
  DAGE_CUDA_TRY(cudaEventRecord(g->ev1, s));
  DAGE_CUDA_TRY(cudaStreamSynchronize(s));
  DAGE_CUDA_TRY(cudaEventElapsedTime(&g->last_ms, g->ev0, g->ev1));
  if (g->near16set) DAGE_TRY(near_f16_set_check(g->near16set, s));
  return 0;
}

int dage_gbfmm_multipole_moments(dage_gbfmm *g, const double *rho, unsigned flags,
                                 double *moments) {
  clear_error();
  if (!g || !rho || !moments) return fail(DAGE_E_INVALID, "null argument");
  DAGE_CUDA_TRY(cudaSetDevice(g->device));
  const double *d_rho;
  double *d_V;
  DAGE_TRY(stage_io(g, rho, nullptr, flags & DAGE_DEVICE_PTRS, &d_rho, &d_V));
  DAGE_TRY(single_setup(g, d_rho, nullptr, false));
  DAGE_TRY(run_multipoles(g->d_inst.as<GInst>(), 1, g->nbox, g->lmax, g->nslab, g->kappa > 0.0,
                          g->stream));
  DAGE_CUDA_TRY(cudaMemcpyAsync(moments, g->d_q.as<double>() + (size_t)g->fine_off * g->N,
                                sizeof(double) * g->nbox * g->N,
                                cudaMemcpyDeviceToHost, g->stream));
  DAGE_CUDA_TRY(cudaStreamSynchronize(g->stream));
  return 0;
}

int dage_gbfmm_local_expansions(dage_gbfmm *g, double *L) {
  clear_error();
  if (!g || !L) return fail(DAGE_E_INVALID, "null argument");
  DAGE_CUDA_TRY(cudaMemcpy(L, g->d_L.as<double>() + (size_t)g->fine_off * g->N,
                           sizeof(double) * g->nbox * g->N, cudaMemcpyDeviceToHost));
  return 0;
}

int dage_gbfmm_evaluate_le(dage_gbfmm *g, const double *local_expansions, double *V,
                           unsigned flags) {
  clear_error();
  if (!g || !local_expansions || !V) return fail(DAGE_E_INVALID, "null argument");
  DAGE_CUDA_TRY(cudaSetDevice(g->device));
  cudaStream_t s = g->stream;
  const size_t n = (size_t)g->npts[0] * g->npts[1] * g->npts[2];
  TmpBuf dL;
  DAGE_TRY(dL.alloc(sizeof(double) * g->nbox * g->N));
  DAGE_CUDA_TRY(cudaMemcpyAsync(dL.ptr, local_expansions, sizeof(double) * g->nbox * g->N,
                                cudaMemcpyHostToDevice, s));
  double *d_V = V;
  if (!(flags & DAGE_DEVICE_PTRS)) {
    DAGE_TRY(g->d_V.alloc(sizeof(double) * n));
    DAGE_CUDA_TRY(cudaMemcpyAsync(g->d_V.ptr, V, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    d_V = g->d_V.as<double>();
  }
  DAGE_TRY(single_setup(g, nullptr, d_V, false));
  DAGE_TRY(run_l2p(g->d_inst.as<GInst>(), 1, g->nbox, g->lmax, max_owned(g), dL.as<double>(),
                   g->kappa > 0.0, s));
  if (!(flags & DAGE_DEVICE_PTRS))
    DAGE_CUDA_TRY(cudaMemcpyAsync(V, d_V, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  DAGE_CUDA_TRY(cudaStreamSynchronize(s));
  return 0;
}

int dage_gbfmm_last_time_ms(const dage_gbfmm *g, float *ms) {
  if (!g || !ms) return fail(DAGE_E_INVALID, "null argument");
  *ms = g->last_ms;
  return 0;
}

// ----------------------------------------------------------------- batch
int dage_gbfmm_batch_create(int n, const dage_grid1d *grids, int maxlevel, int lmax,
                            const dage_quad *quad, int precision, size_t near_budget_bytes,
                            dage_gbfmm_batch **out) {
  clear_error();
  if (!out) return fail(DAGE_E_INVALID, "null output handle pointer");
  *out = nullptr;
  if (n < 1 || n > 65535 || !grids || !quad)
    return fail(DAGE_E_INVALID, "need 1..65535 densities, grids and a quadrature");
  if (precision != DAGE_FP64 && precision != DAGE_MIXED_FP16X3)
    return fail(DAGE_E_UNSUPPORTED,
                "the GBFMM batch runs in DAGE_FP64 or DAGE_MIXED_FP16X3 (near field)");
  auto *b = new dage_gbfmm_batch();
  const size_t budget = near_budget_bytes ? near_budget_bytes : ((size_t)8 << 30);
  const int rc = batch_create_impl(b, n, grids, maxlevel, lmax, quad, precision, budget);
  if (rc) {
    batch_destroy_impl(b);
    return rc;
  }
  *out = b;
  return 0;
}

int dage_gbfmm_batch_apply(dage_gbfmm_batch *b, const double *const *rho, double *const *V,
                           unsigned flags, double *energies) {
  clear_error();
  if (!b || !rho || !V) return fail(DAGE_E_INVALID, "null argument");
  if ((flags & DAGE_ENERGY) && !energies) return fail(DAGE_E_INVALID, "energies pointer is null");
  for (int i = 0; i < b->n; ++i)
    if (!rho[i] || !V[i]) return fail(DAGE_E_INVALID, "null cube for density %d", i);
  DAGE_CUDA_TRY(cudaSetDevice(b->device));
  cudaStream_t s = b->stream;
  DAGE_CUDA_TRY(cudaEventRecord(b->ev0, s));
  // device cubes
  std::vector<const double *> dr(b->n);
  std::vector<double *> dv(b->n);
  if (flags & DAGE_DEVICE_PTRS) {
    for (int i = 0; i < b->n; ++i) {
      dr[i] = rho[i];
      dv[i] = V[i];
    }
  } else {
    if (b->stage_off.empty()) {
      size_t off = 0;
      for (int i = 0; i < b->n; ++i) {
        b->stage_off.push_back(off);
        off += b->npts[i];
      }
      DAGE_TRY(b->stage_rho.alloc(sizeof(double) * off));
      DAGE_TRY(b->stage_V.alloc(sizeof(double) * off));
    }
    for (int i = 0; i < b->n; ++i) {
      dr[i] = b->stage_rho.as<double>() + b->stage_off[i];
      dv[i] = b->stage_V.as<double>() + b->stage_off[i];
      DAGE_CUDA_TRY(cudaMemcpyAsync(const_cast<double *>(dr[i]), rho[i],
                                    sizeof(double) * b->npts[i], cudaMemcpyHostToDevice, s));
    }
  }
  std::vector<const void *> key;
  for (int i = 0; i < b->n; ++i) {
    key.push_back(dr[i]);
    key.push_back(dv[i]);
  }
  const bool use_graph = !(flags & DAGE_NO_GRAPH);
  if (!use_graph || key != b->graph_key || !b->exec) {
    DAGE_TRY(batch_tables(b, dr.data(), dv.data()));
    if (!b->tuned) {
      // keyed on the batch: device, t-points, the densities' points per axis
      std::map<std::string, int> sizes;  // grid -> densities on it
      for (int i = 0; i < b->n; ++i) {
        const dage_gbfmm *g = b->plans[b->plan_of[i]];
        ++sizes[std::to_string(g->npts[0]) + "x" + std::to_string(g->npts[1]) + "x" +
                std::to_string(g->npts[2])];
      }
      std::string key = tune_device_key() + "/gbfmm_batch_fp64/P" + std::to_string(b->P);
      for (const auto &kv : sizes) key += "," + kv.first + "*" + std::to_string(kv.second);
      std::vector<int> v;
      if (tune_lookup(key, v) && v.size() == 3) {
        for (int d = 0; d < 3; ++d) b->tile_n[d] = v[d];
      } else {
        const auto &c = b->chunks[0];
        const StageDesc *dd[3] = {c.desc[0].as<StageDesc>(), c.desc[1].as<StageDesc>(),
                                  c.desc[2].as<StageDesc>()};
        DAGE_TRY(autotune_tiles(dd, c.njobs, b->mt, b->nt, s, b->tile_n));
        tune_store(key, {b->tile_n[0], b->tile_n[1], b->tile_n[2]});
      }
      b->tuned = true;
    }
    if (use_graph) {
      if (b->exec) cudaGraphExecDestroy(b->exec);
      if (b->graph) cudaGraphDestroy(b->graph);
      b->exec = nullptr;
      b->graph = nullptr;
      b->graph_key.clear();
      // kernel attributes are set before capture
      DAGE_TRY(prepare_fp64_stages());
      DAGE_TRY(near_f16_prepare());
      DAGE_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      const int rc = batch_launch(b, dr.data(), dv.data());
      cudaGraph_t graph = nullptr;
      const cudaError_t ce = cudaStreamEndCapture(s, &graph);
      if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
      }
      if (ce != cudaSuccess) return fail(DAGE_E_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
      b->graph = graph;
      DAGE_CUDA_TRY(cudaGraphGetNodes(graph, nullptr, &b->graph_nodes));
      DAGE_CUDA_TRY(cudaGraphInstantiate(&b->exec, graph, 0));
      b->graph_key = key;
    }
  }
  if (use_graph)
    DAGE_CUDA_TRY(cudaGraphLaunch(b->exec, s));
  else
    DAGE_TRY(batch_launch(b, dr.data(), dv.data()));
  if (!(flags & DAGE_DEVICE_PTRS))
    for (int i = 0; i < b->n; ++i)
      DAGE_CUDA_TRY(cudaMemcpyAsync(V[i], dv[i], sizeof(double) * b->npts[i],
                                    cudaMemcpyDeviceToHost, s));
  if (flags & DAGE_ENERGY)
    DAGE_CUDA_TRY(cudaMemcpyAsync(energies, b->energy.ptr, sizeof(double) * b->n,
                                  cudaMemcpyDeviceToHost, s));
  DAGE_CUDA_TRY(cudaEventRecord(b->ev1, s));
  DAGE_CUDA_TRY(cudaStreamSynchronize(s));
  DAGE_CUDA_TRY(cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1));
  for (auto &m : b->msets) DAGE_TRY(near_f16_set_check(m.set, s));
  return 0;
}

int dage_gbfmm_batch_set_energies(dage_gbfmm_batch *b, const double *energies) {
  clear_error();
  if (!b || !energies) return fail(DAGE_E_INVALID, "null argument");
  for (int i = 0; i < b->n; ++i)
    if (!(energies[i] <= 0.0)) return fail(DAGE_E_INVALID, "energy %d must be <= 0", i);
  DAGE_CUDA_TRY(cudaSetDevice(b->device));
  DAGE_CUDA_TRY(cudaStreamSynchronize(b->stream));
  for (auto &k : b->kerns) {
    k.T.release();
    k.w.release();
    k.Wh.release();
  }
  b->kerns.clear();
  for (int i = 0; i < b->n; ++i) {
    b->kern_of[i] = -1;
    if (energies[i] == 0.0) continue;
    for (size_t k = 0; k < b->kerns.size() && b->kern_of[i] < 0; ++k)
      if (b->kerns[k].plan == b->plan_of[i] && b->kerns[k].energy == energies[i])
        b->kern_of[i] = (int)k;
    if (b->kern_of[i] >= 0) continue;
    b->kerns.emplace_back();
    auto &k = b->kerns.back();
    k.plan = b->plan_of[i];
    k.energy = energies[i];
    const dage_gbfmm *g = b->plans[k.plan];
    DAGE_TRY(build_m2l_into(g, std::sqrt(-2.0 * k.energy), k.T));
    DAGE_TRY(build_helm_m2m_into(g, std::sqrt(-2.0 * k.energy), k.Wh));
    std::vector<double> w;
    weights_for(g, k.energy, w);
    DAGE_TRY(k.w.alloc(sizeof(double) * w.size()));
    DAGE_CUDA_TRY(cudaMemcpyAsync(k.w.ptr, w.data(), sizeof(double) * w.size(),
                                  cudaMemcpyHostToDevice, b->stream));
    DAGE_CUDA_TRY(cudaStreamSynchronize(b->stream));
    b->kern_of[i] = (int)b->kerns.size() - 1;
  }
  b->graph_key.clear();  // the tables change: capture again on the next apply
  return 0;
}

int dage_gbfmm_batch_set_bubbles(dage_gbfmm_batch *b, const dage_bubbles *bubbles,
                                 const double *factors, int lmin) {
  clear_error();
  if (!b) return fail(DAGE_E_INVALID, "null handle");
  if (bubbles && !factors) return fail(DAGE_E_INVALID, "factors are null");
  b->bubbles = bubbles;
  b->inject_lmin = lmin;
  b->inject_factor.assign(b->n, 0.0);
  if (bubbles)
    for (int i = 0; i < b->n; ++i) b->inject_factor[i] = factors[i];
  b->graph_key.clear();  // the pipeline changes: capture again on the next apply
  return 0;
}

int dage_gbfmm_batch_info(const dage_gbfmm_batch *b, int *nplans, int *nchunks, int tile_n[3],
                          long long *graph_nodes) {
  if (!b) return fail(DAGE_E_INVALID, "null handle");
  if (nplans) *nplans = (int)b->plans.size();
  if (nchunks) *nchunks = (int)(b->precision == DAGE_FP64 ? b->chunks.size() : b->msets.size());
  if (tile_n)
    for (int d = 0; d < 3; ++d) tile_n[d] = b->tile_n[d];
  if (graph_nodes) *graph_nodes = (long long)b->graph_nodes;
  return 0;
}

int dage_gbfmm_batch_set_stream(dage_gbfmm_batch *b, void *stream) {
  if (!b) return fail(DAGE_E_INVALID, "null handle");
  b->stream = stream ? (cudaStream_t)stream : b->own_stream;
  for (auto *g : b->plans) g->stream = b->stream;
  return 0;
}

int dage_gbfmm_batch_last_time_ms(const dage_gbfmm_batch *b, float *ms) {
  if (!b || !ms) return fail(DAGE_E_INVALID, "null argument");
  *ms = b->last_ms;
  return 0;
}

int dage_gbfmm_batch_destroy(dage_gbfmm_batch *b) {
  clear_error();
  batch_destroy_impl(b);
  return 0;
}

}  // extern "C"
