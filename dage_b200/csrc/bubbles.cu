// bubbles.cu -- bubbles -> cube injection on one B200.
//
//   cube(r) += factor * sum_atoms sum_{l >= lmin} sum_m [r^k f_lm](|r - R|) Y_lm(r - R)
//
// The radial functions live on per-atom LIP grids (7-point cells starting at
// r = 0).  At creation each cell's LIP values are turned into monomial
// coefficients in the cell coordinate (the reference's calc_cf,
// src/bubbles/bubbles_cuda.cu:197-300), on the GPU, once per bubble set.  The
// injection is ONE kernel over all atoms: every thread owns cube points
// (8 x 8 x 4 bricks per block, so a warp's lanes share radial cells), loops
// over the atoms (centres, radial cell starts and steps staged in
// shared memory), finds the radial cell by the same binary search as
// Grid1D_get_icell (src/bubbles/grid.F90:1212-1245, valid for any radial
// grid, not only the reference GPU path's closed-form cell index), evaluates
// the radial polynomial by Horner and the Racah-normalised real spherical
// harmonics of the unit vector by recursion (YBundle,
// src/bubbles/harmonic.F90:612-660), and adds to the cube once.  The
// reference launches one kernel per atom per stream
// (src/bubbles/bubbles_cuda.cu:3090-3350).
#include <algorithm>
#include <cmath>
#include <vector>

#include "bubbles.cuh"

namespace dage {
namespace {

constexpr int kMaxAtomsSmem = 256;

// Two points' values side by side: the harmonics recursion below runs on
// both at once, each lane of the pair with exactly the single-point
// arithmetic.
struct Pair {
  double a, b;
  __device__ Pair() {}
  __device__ Pair(double v) : a(v), b(v) {}
  __device__ Pair(double x, double y) : a(x), b(y) {}
};
__device__ __forceinline__ Pair operator*(Pair x, Pair y) { return Pair(x.a * y.a, x.b * y.b); }
__device__ __forceinline__ Pair operator*(double s, Pair x) { return Pair(s * x.a, s * x.b); }
__device__ __forceinline__ Pair operator*(Pair x, double s) { return Pair(x.a * s, x.b * s); }
__device__ __forceinline__ Pair operator+(Pair x, Pair y) { return Pair(x.a + y.a, x.b + y.b); }
__device__ __forceinline__ Pair operator-(Pair x, Pair y) { return Pair(x.a - y.a, x.b - y.b); }

// The same recursion for a compile-time lmax, fully unrolled, so that every
// callback sees a constant lm; T = double (one point) or Pair (two).
template <int LS, class T, class F>
__device__ __forceinline__ void unit_harmonics_fixed(T x, T y, T z, F &&f) {
  f(0, T(1.0));
  if constexpr (LS > 0) {
    T p2 = T(1.0), p1 = z;
    f(2, z);
#pragma unroll
    for (int l = 2; l <= LS; ++l) {
      T cur = (2.0 * l - 1.0) * (z * p1) - sqrt((double)((l - 1) * (l - 1))) * p2;
      cur = cur * (1.0 / sqrt((double)(l * l)));
      f(l * (l + 1), cur);
      p2 = p1;
      p1 = cur;
    }
    T top = x, bot = y;
#pragma unroll
    for (int mm = 1; mm <= LS; ++mm) {
      if (mm >= 2) {
        const double c = sqrt(1.0 - 0.5 / mm);
        const T nb = c * (top * y + bot * x);
        const T nt = c * (top * x - bot * y);
        top = nt;
        bot = nb;
      }
      f(mm * (mm + 1) + mm, top);
      f(mm * (mm + 1) - mm, bot);
#pragma unroll
      for (int sg = 0; sg < 2; ++sg) {
        const int m = sg ? -mm : mm;
        T q2 = T(0.0), q1 = sg ? bot : top;
#pragma unroll
        for (int l = mm + 1; l <= LS; ++l) {
          T cur = (2.0 * l - 1.0) * (q1 * z);
          if (l - mm > 1) cur = cur - sqrt((l + m - 1.0) * (l - m - 1.0)) * q2;
          cur = (1.0 / sqrt(1.0 * (l - m) * (l + m))) * cur;
          f(l * (l + 1) + m, cur);
          q2 = q1;
          q1 = cur;
        }
      }
    }
  }
}

// A 7-point cell's polynomial (coefficients highest power first, padded to
// 8) at t, the coefficients read as four 16-byte loads.
__device__ __forceinline__ double horner7(const double *c, double t) {
  const double2 *q = reinterpret_cast<const double2 *>(c);
  const double2 a = __ldg(q), b = __ldg(q + 1), e = __ldg(q + 2), g = __ldg(q + 3);
  double v = a.x;
  v = v * t + a.y;
  v = v * t + b.x;
  v = v * t + b.y;
  v = v * t + e.x;
  v = v * t + e.y;
  return v * t + g.x;
}

// The same polynomial at two cell coordinates, its coefficients read once.
__device__ __forceinline__ Pair horner7_pair(const double *c, double t0, double t1) {
  const double2 *q = reinterpret_cast<const double2 *>(c);
  const double2 a = __ldg(q), b = __ldg(q + 1), e = __ldg(q + 2), g = __ldg(q + 3);
  double v = a.x, w = a.x;
  v = v * t0 + a.y;
  w = w * t1 + a.y;
  v = v * t0 + b.x;
  w = w * t1 + b.x;
  v = v * t0 + b.y;
  w = w * t1 + b.y;
  v = v * t0 + e.x;
  w = w * t1 + e.x;
  v = v * t0 + e.y;
  w = w * t1 + e.y;
  return Pair(v * t0 + g.x, w * t1 + g.x);
}

// LIP values of one cell -> monomial coefficients in the cell coordinate
// (highest power first), padded to 8 per (cell, lm).
__global__ void bubble_coeffs_kernel(const double *__restrict__ rf, const int *__restrict__ atom_np,
                                     const int *__restrict__ atom_foff,
                                     const int *__restrict__ atom_cell0, int natom, int N,
                                     const double *__restrict__ lipc, int nlip, double *coef) {
  // one thread per (global cell, lm)
  const int total_cells = atom_cell0[natom];
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total_cells * N) return;
  const int gcell = idx / N, lm = idx % N;
  int a = 0;
  while (atom_cell0[a + 1] <= gcell) ++a;
  const int c = gcell - atom_cell0[a];
  const double *vals = rf + atom_foff[a] + (size_t)lm * atom_np[a] + c * (nlip - 1);
  double *o = coef + ((size_t)gcell * N + lm) * 8;
  for (int kk = 0; kk < 8; ++kk) {
    double s = 0.0;
    if (kk < nlip)
      for (int j = 0; j < nlip; ++j) s += lipc[kk * nlip + j] * vals[j];
    o[kk] = s;
  }
}

// Cube points in 8 x 8 x 4 bricks, one brick per 256-thread block and step:
// a warp holds 8 x 4 neighbouring (x, y) points, so its lanes mostly share
// each atom's radial cell (one coefficient block, little divergence in the
// cell search), and a block's points are 0.8 x 0.8 x 0.4 cells apart at most
// instead of a 256-point line.  Requires blockDim.x == 256.
struct BrickGrid {
  int nx, ny, nz, nbx, nby;
  long long count;
  __device__ BrickGrid(int nx_, int ny_, int nz_)
      : nx(nx_), ny(ny_), nz(nz_), nbx((nx_ + 7) / 8), nby((ny_ + 7) / 8),
        count((long long)((nx_ + 7) / 8) * ((ny_ + 7) / 8) * ((nz_ + 3) / 4)) {}
  __device__ bool point(long long bk, int &ix, int &iy, int &iz) const {
    const int bx = (int)(bk % nbx);
    const long long r = bk / nbx;
    const int by = (int)(r % nby), bz = (int)(r / nby);
    ix = bx * 8 + (threadIdx.x & 7);
    iy = by * 8 + ((threadIdx.x >> 3) & 7);
    iz = bz * 4 + (threadIdx.x >> 6);
    return ix < nx && iy < ny && iz < nz;
  }
};

// 8 x 8 x 8 bricks for two points per thread: thread t holds (x, y) =
// (t % 8, (t / 8) % 8) and z = t / 64 and t / 64 + 4 of the brick.
struct BrickGrid2 {
  int nx, ny, nz, nbx, nby;
  long long count;
  __device__ BrickGrid2(int nx_, int ny_, int nz_)
      : nx(nx_), ny(ny_), nz(nz_), nbx((nx_ + 7) / 8), nby((ny_ + 7) / 8),
        count((long long)((nx_ + 7) / 8) * ((ny_ + 7) / 8) * ((nz_ + 7) / 8)) {}
  __device__ void point(long long bk, int &ix, int &iy, int &iz) const {
    const int bx = (int)(bk % nbx);
    const long long r = bk / nbx;
    const int by = (int)(r % nby), bz = (int)(r / nby);
    ix = bx * 8 + (threadIdx.x & 7);
    iy = by * 8 + ((threadIdx.x >> 3) & 7);
    iz = bz * 8 + (threadIdx.x >> 6);
  }
};


// LS >= 0: lmax <= LS and 7-point cells (harmonics unrolled, 16-byte
// coefficient loads); LS = -1: any lmax and cell size.
template <int LS>
__global__ void __launch_bounds__(256)
    inject_kernel(const AtomTab *__restrict__ atoms, int natom, const double *__restrict__ celld,
                  const double *__restrict__ hcell, const double *__restrict__ coef, int N,
                  int lmax, int lmin, int nlip, double first, const double *__restrict__ xs,
                  int nx, const double *__restrict__ ys, int ny, const double *__restrict__ zs,
                  int nz, double factor, double *cube) {
  __shared__ AtomTab sa[kMaxAtomsSmem];
  for (int a = threadIdx.x; a < natom && a < kMaxAtomsSmem; a += blockDim.x) sa[a] = atoms[a];
  __syncthreads();
  const int lm0 = lmin * lmin;
  const BrickGrid B(nx, ny, nz);
  for (long long bk = blockIdx.x; bk < B.count; bk += gridDim.x) {
    int ix, iy, iz;
    if (!B.point(bk, ix, iy, iz)) continue;
    const long long i = ix + (long long)nx * (iy + (long long)ny * iz);
    const double px = xs[ix], py = ys[iy], pz = zs[iz];
    double acc = 0.0;
    for (int a = 0; a < natom; ++a) {
      const AtomTab A = a < kMaxAtomsSmem ? sa[a] : atoms[a];
      const double dx = px - A.cx, dy = py - A.cy, dz = pz - A.cz;
      const double d = sqrt(dx * dx + dy * dy + dz * dz);
      if (d > A.rmax) continue;
      // Grid1D_get_icell: binary search on the cell starts (1-based cells)
      const double *cd = celld + A.cell0;
      int ic;
      if (cd[A.ncell - 1] <= d) {
        ic = A.ncell;
      } else {
        int icell = A.ncell / 2, maxi = A.ncell - 1, mini = 1;
        ic = 0;
        for (int it = 0; it < 64 && !ic; ++it) {
          if (d >= cd[icell]) {
            if (d < cd[icell + 1]) {
              ic = icell + 1;
            } else {
              mini = icell + 2;
              icell = (mini + maxi) / 2;
            }
          } else {
            if (d >= cd[icell - 1]) {
              ic = icell;
            } else {
              maxi = icell - 1;
              icell = (mini + maxi) / 2;
            }
          }
        }
        if (!ic) continue;
      }
      const double t = (d - cd[ic - 1]) / hcell[A.cell0 + ic - 1] + first;
      const double *cf = coef + ((size_t)(A.cell0 + ic - 1) * N) * 8;
      double ux = 0.0, uy = 0.0, uz = 0.0;
      const bool at_centre = !(d > 0.0);
      if (!at_centre) {
        const double inv = 1.0 / d;
        ux = dx * inv;
        uy = dy * inv;
        uz = dz * inv;
      }
      if constexpr (LS >= 0) {
        unit_harmonics_fixed<LS>(ux, uy, uz, [&](int lm, double Y) {
          if (lm < lm0 || lm >= N) return;
          if (at_centre && lm > 0) return;
          acc += horner7(cf + (size_t)lm * 8, t) * Y;
        });
      } else {
        unit_harmonics(lmax, ux, uy, uz, [&](int lm, double Y) {
          if (lm < lm0) return;
          if (at_centre && lm > 0) return;
          const double *c = cf + (size_t)lm * 8;
          double v = c[0];
          for (int kk = 1; kk < nlip; ++kk) v = v * t + c[kk];
          acc += v * Y;
        });
      }
    }
    cube[i] += factor * acc;
  }
}

// inject_kernel with two points per thread (z and z + 4 of an 8 x 8 x 8
// brick), each radial polynomial's coefficients read once for both points
// when they share the atom's radial cell; each point keeps the
// single-point kernel's arithmetic.  7-point cells, lmax <= LS.
template <int LS>
__global__ void __launch_bounds__(256)
    inject_pair_kernel(const AtomTab *__restrict__ atoms, int natom,
                       const double *__restrict__ celld, const double *__restrict__ hcell,
                       const double *__restrict__ coef, int N, int lmin, double first,
                       const double *__restrict__ xs, int nx, const double *__restrict__ ys,
                       int ny, const double *__restrict__ zs, int nz, double factor,
                       double *cube) {
  __shared__ AtomTab sa[kMaxAtomsSmem];
  for (int a = threadIdx.x; a < natom && a < kMaxAtomsSmem; a += blockDim.x) sa[a] = atoms[a];
  __syncthreads();
  const int lm0 = lmin * lmin;
  const BrickGrid2 B(nx, ny, nz);
  for (long long bk = blockIdx.x; bk < B.count; bk += gridDim.x) {
    int ix, iy, iz0;
    B.point(bk, ix, iy, iz0);
    const int iz1 = iz0 + 4;
    if (ix >= nx || iy >= ny || iz0 >= nz) continue;
    const bool has1 = iz1 < nz;
    const double px = xs[ix], py = ys[iy], pz0 = zs[iz0], pz1 = has1 ? zs[iz1] : pz0;
    Pair acc(0.0);
    for (int a = 0; a < natom; ++a) {
      const AtomTab A = a < kMaxAtomsSmem ? sa[a] : atoms[a];
      const double dx = px - A.cx, dy = py - A.cy, dz0 = pz0 - A.cz, dz1 = pz1 - A.cz;
      const double d0 = sqrt(dx * dx + dy * dy + dz0 * dz0);
      const double d1 = sqrt(dx * dx + dy * dy + dz1 * dz1);
      const bool in0 = d0 <= A.rmax, in1 = has1 && d1 <= A.rmax;
      if (!in0 && !in1) continue;
      const double *cd = celld + A.cell0;
      const int ic0 = in0 ? radial_cell(cd, A.ncell, d0) : 0;
      const int ic1 = in1 ? radial_cell(cd, A.ncell, d1) : 0;
      if (!ic0 && !ic1) continue;
      const double t0 = ic0 ? (d0 - cd[ic0 - 1]) / hcell[A.cell0 + ic0 - 1] + first : 0.0;
      const double t1 = ic1 ? (d1 - cd[ic1 - 1]) / hcell[A.cell0 + ic1 - 1] + first : 0.0;
      const bool ctr0 = !(d0 > 0.0), ctr1 = !(d1 > 0.0);
      double ux0 = 0.0, uy0 = 0.0, uz0 = 0.0, ux1 = 0.0, uy1 = 0.0, uz1 = 0.0;
      if (!ctr0) {
        const double inv = 1.0 / d0;
        ux0 = dx * inv;
        uy0 = dy * inv;
        uz0 = dz0 * inv;
      }
      if (!ctr1) {
        const double inv = 1.0 / d1;
        ux1 = dx * inv;
        uy1 = dy * inv;
        uz1 = dz1 * inv;
      }
      if (ic0 == ic1) {
        const double *cf = coef + ((size_t)(A.cell0 + ic0 - 1) * N) * 8;
        unit_harmonics_fixed<LS>(Pair(ux0, ux1), Pair(uy0, uy1), Pair(uz0, uz1),
                                 [&](int lm, Pair Y) {
          if (lm < lm0 || lm >= N) return;
          const Pair h = horner7_pair(cf + (size_t)lm * 8, t0, t1);
          if (!(ctr0 && lm > 0)) acc.a += h.a * Y.a;
          if (!(ctr1 && lm > 0)) acc.b += h.b * Y.b;
        });
      } else {
        auto one = [&](int ic, double t, double ux, double uy, double uz, bool ctr, double &w) {
          const double *cf = coef + ((size_t)(A.cell0 + ic - 1) * N) * 8;
          unit_harmonics_fixed<LS>(ux, uy, uz, [&](int lm, double Y) {
            if (lm < lm0 || lm >= N) return;
            if (ctr && lm > 0) return;
            w += horner7(cf + (size_t)lm * 8, t) * Y;
          });
        };
        if (ic0) one(ic0, t0, ux0, uy0, uz0, ctr0, acc.a);
        if (ic1) one(ic1, t1, ux1, uy1, uz1, ctr1, acc.b);
      }
    }
    const long long i0 = ix + (long long)nx * (iy + (long long)ny * iz0);
    cube[i0] += factor * acc.a;
    if (has1) {
      const long long i1 = ix + (long long)nx * (iy + (long long)ny * iz1);
      cube[i1] += factor * acc.b;
    }
  }
}

// The cube part of a function product in one pass (Function3D_multiply,
// function3d.F90:1097-1409; the reference GPU path injects each bubble set
// in its own launches per atom, multiplies the cubes, then de-injects,
// bubbles_cuda.cu:3533-3690):
//   out = (c1 + B1)(c2 + B2) - Br
// The three bubble sets share atoms and radial grids, so every atom's
// distance, radial cell, cell coordinate and harmonics are computed once per
// point for all three; Ni = 0 marks an absent set.
// LS >= 0: every set has lmax <= LS and 7-point cells (harmonics unrolled,
// 16-byte coefficient loads); LS = -1: any lmax and cell size.
template <int LS>
__global__ void __launch_bounds__(256)
    function_product_kernel(const AtomTab *__restrict__ atoms, int natom,
                            const double *__restrict__ celld, const double *__restrict__ hcell,
                            const double *__restrict__ coef1, int N1,
                            const double *__restrict__ coef2, int N2,
                            const double *__restrict__ coefr, int Nr, int lmax, int nlip,
                            double first, const double *__restrict__ xs, int nx,
                            const double *__restrict__ ys, int ny, const double *__restrict__ zs,
                            int nz, const double *c1, const double *c2, double *out) {
  __shared__ AtomTab sa[kMaxAtomsSmem];
  for (int a = threadIdx.x; a < natom && a < kMaxAtomsSmem; a += blockDim.x) sa[a] = atoms[a];
  __syncthreads();
  const BrickGrid B(nx, ny, nz);
  for (long long bk = blockIdx.x; bk < B.count; bk += gridDim.x) {
    int ix, iy, iz;
    if (!B.point(bk, ix, iy, iz)) continue;
    const long long i = ix + (long long)nx * (iy + (long long)ny * iz);
    const double px = xs[ix], py = ys[iy], pz = zs[iz];
    double v1 = 0.0, v2 = 0.0, vr = 0.0;
    for (int a = 0; a < natom; ++a) {
      const AtomTab A = a < kMaxAtomsSmem ? sa[a] : atoms[a];
      const double dx = px - A.cx, dy = py - A.cy, dz = pz - A.cz;
      const double d = sqrt(dx * dx + dy * dy + dz * dz);
      if (d > A.rmax) continue;
      const double *cd = celld + A.cell0;
      const int ic = radial_cell(cd, A.ncell, d);
      if (!ic) continue;
      const double t = (d - cd[ic - 1]) / hcell[A.cell0 + ic - 1] + first;
      const size_t cell = (size_t)(A.cell0 + ic - 1);
      double ux = 0.0, uy = 0.0, uz = 0.0;
      const bool at_centre = !(d > 0.0);
      if (!at_centre) {
        const double inv = 1.0 / d;
        ux = dx * inv;
        uy = dy * inv;
        uz = dz * inv;
      }
      if constexpr (LS >= 0) {
        unit_harmonics_fixed<LS>(ux, uy, uz, [&](int lm, double Y) {
          if (at_centre && lm > 0) return;
          if (lm < N1) v1 += horner7(coef1 + (cell * N1 + lm) * 8, t) * Y;
          if (lm < N2) v2 += horner7(coef2 + (cell * N2 + lm) * 8, t) * Y;
          if (lm < Nr) vr += horner7(coefr + (cell * Nr + lm) * 8, t) * Y;
        });
      } else {
        auto horner = [&](const double *c) {
          double v = c[0];
          for (int kk = 1; kk < nlip; ++kk) v = v * t + c[kk];
          return v;
        };
        unit_harmonics(lmax, ux, uy, uz, [&](int lm, double Y) {
          if (at_centre && lm > 0) return;
          if (lm < N1) v1 += horner(coef1 + (cell * N1 + lm) * 8) * Y;
          if (lm < N2) v2 += horner(coef2 + (cell * N2 + lm) * 8) * Y;
          if (lm < Nr) vr += horner(coefr + (cell * Nr + lm) * 8) * Y;
        });
      }
    }
    out[i] = (c1[i] + v1) * (c2[i] + v2) - vr;
  }
}


// function_product_kernel with two points per thread, z and z + 4 of an
// 8 x 8 x 8 brick.  The kernel is bound by the L1 traffic of the radial
// coefficients (4 16-byte loads per polynomial, 43 polynomials per atom at
// lmax 2 x 2 -> 4); when an atom puts both points in the same radial cell
// -- nearly always, the points are 0.4 bohr apart -- each polynomial's
// coefficients are read once for both.  The two factors' sets (lmax <= LSB)
// and the result set (lmax <= LSR) run in two harmonics passes, so that few
// sums are live at once; the recursion visits the harmonics below any l in
// the same order whatever its top l, so every point keeps the single-point
// kernel's arithmetic and summation order.  7-point cells.
template <int LSB, int LSR>
__global__ void __launch_bounds__(256)
    function_product_pair_kernel(const AtomTab *__restrict__ atoms, int natom,
                                 const double *__restrict__ celld,
                                 const double *__restrict__ hcell,
                                 const double *__restrict__ coef1, int N1,
                                 const double *__restrict__ coef2, int N2,
                                 const double *__restrict__ coefr, int Nr, double first,
                                 const double *__restrict__ xs, int nx,
                                 const double *__restrict__ ys, int ny,
                                 const double *__restrict__ zs, int nz, const double *c1,
                                 const double *c2, double *out) {
  __shared__ AtomTab sa[kMaxAtomsSmem];
  for (int a = threadIdx.x; a < natom && a < kMaxAtomsSmem; a += blockDim.x) sa[a] = atoms[a];
  __syncthreads();
  const BrickGrid2 B(nx, ny, nz);
  for (long long bk = blockIdx.x; bk < B.count; bk += gridDim.x) {
    int ix, iy, iz0;
    B.point(bk, ix, iy, iz0);
    const int iz1 = iz0 + 4;
    if (ix >= nx || iy >= ny || iz0 >= nz) continue;
    const bool has1 = iz1 < nz;
    const double px = xs[ix], py = ys[iy], pz0 = zs[iz0], pz1 = has1 ? zs[iz1] : pz0;
    Pair v1(0.0), v2(0.0), vr(0.0);
    for (int a = 0; a < natom; ++a) {
      const AtomTab A = a < kMaxAtomsSmem ? sa[a] : atoms[a];
      const double dx = px - A.cx, dy = py - A.cy, dz0 = pz0 - A.cz, dz1 = pz1 - A.cz;
      const double d0 = sqrt(dx * dx + dy * dy + dz0 * dz0);
      const double d1 = sqrt(dx * dx + dy * dy + dz1 * dz1);
      const bool in0 = d0 <= A.rmax, in1 = has1 && d1 <= A.rmax;
      if (!in0 && !in1) continue;
      const double *cd = celld + A.cell0;
      const int ic0 = in0 ? radial_cell(cd, A.ncell, d0) : 0;
      const int ic1 = in1 ? radial_cell(cd, A.ncell, d1) : 0;
      if (!ic0 && !ic1) continue;
      const double t0 = ic0 ? (d0 - cd[ic0 - 1]) / hcell[A.cell0 + ic0 - 1] + first : 0.0;
      const double t1 = ic1 ? (d1 - cd[ic1 - 1]) / hcell[A.cell0 + ic1 - 1] + first : 0.0;
      const bool ctr0 = !(d0 > 0.0), ctr1 = !(d1 > 0.0);
      double ux0 = 0.0, uy0 = 0.0, uz0 = 0.0, ux1 = 0.0, uy1 = 0.0, uz1 = 0.0;
      if (!ctr0) {
        const double inv = 1.0 / d0;
        ux0 = dx * inv;
        uy0 = dy * inv;
        uz0 = dz0 * inv;
      }
      if (!ctr1) {
        const double inv = 1.0 / d1;
        ux1 = dx * inv;
        uy1 = dy * inv;
        uz1 = dz1 * inv;
      }
      if (ic0 == ic1) {
        const size_t cell = (size_t)(A.cell0 + ic0 - 1);
        const Pair X(ux0, ux1), Yv(uy0, uy1), Z(uz0, uz1);
        unit_harmonics_fixed<LSB>(X, Yv, Z, [&](int lm, Pair Y) {
          const bool use0 = !(ctr0 && lm > 0), use1 = !(ctr1 && lm > 0);
          if (lm < N1) {
            const Pair h = horner7_pair(coef1 + (cell * N1 + lm) * 8, t0, t1);
            if (use0) v1.a += h.a * Y.a;
            if (use1) v1.b += h.b * Y.b;
          }
          if (lm < N2) {
            const Pair h = horner7_pair(coef2 + (cell * N2 + lm) * 8, t0, t1);
            if (use0) v2.a += h.a * Y.a;
            if (use1) v2.b += h.b * Y.b;
          }
        });
        unit_harmonics_fixed<LSR>(X, Yv, Z, [&](int lm, Pair Y) {
          if (lm >= Nr) return;
          const Pair h = horner7_pair(coefr + (cell * Nr + lm) * 8, t0, t1);
          if (!(ctr0 && lm > 0)) vr.a += h.a * Y.a;
          if (!(ctr1 && lm > 0)) vr.b += h.b * Y.b;
        });
      } else {
        // the points in different cells (or one of them outside): each alone
        auto one = [&](int ic, double t, double ux, double uy, double uz, bool ctr, double &w1,
                       double &w2, double &wr) {
          const size_t cell = (size_t)(A.cell0 + ic - 1);
          unit_harmonics_fixed<LSB>(ux, uy, uz, [&](int lm, double Y) {
            if (ctr && lm > 0) return;
            if (lm < N1) w1 += horner7(coef1 + (cell * N1 + lm) * 8, t) * Y;
            if (lm < N2) w2 += horner7(coef2 + (cell * N2 + lm) * 8, t) * Y;
          });
          unit_harmonics_fixed<LSR>(ux, uy, uz, [&](int lm, double Y) {
            if (ctr && lm > 0) return;
            if (lm < Nr) wr += horner7(coefr + (cell * Nr + lm) * 8, t) * Y;
          });
        };
        if (ic0) one(ic0, t0, ux0, uy0, uz0, ctr0, v1.a, v2.a, vr.a);
        if (ic1) one(ic1, t1, ux1, uy1, uz1, ctr1, v1.b, v2.b, vr.b);
      }
    }
    const long long i0 = ix + (long long)nx * (iy + (long long)ny * iz0);
    out[i0] = (c1[i0] + v1.a) * (c2[i0] + v2.a) - vr.a;
    if (has1) {
      const long long i1 = ix + (long long)nx * (iy + (long long)ny * iz1);
      out[i1] = (c1[i1] + v1.b) * (c2[i1] + v2.b) - vr.b;
    }
  }
}


// Radial product of two bubble sets on the same atoms and radial points
// (Bubble_product_kernel, bubbles_multiplier.cu:65-106): one thread per
// (atom, radial point); for every term of the product table
//   out_LM += C * (f1_a f2_b + f1_b f2_a [a != b]),   a <= b.
// The values are the raw radial functions (without r^k).
__global__ void bubbles_product_kernel(const double *__restrict__ f1, int N1,
                                       const double *__restrict__ f2, int N2,
                                       const int *__restrict__ np, const int *__restrict__ poff,
                                       int natom, const ProdTerm *__restrict__ terms, int nterms,
                                       int Nr, double *out) {
  const int total = poff[natom];
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  int a = 0;
  while (poff[a + 1] <= idx) ++a;
  const int j = idx - poff[a], npts = np[a];
  // (lm, point) rows of this atom in each set: atoms are stored one after
  // the other, N rows of npts points each
  const double *g1 = f1 + (size_t)N1 * poff[a] + j;
  const double *g2 = f2 + (size_t)N2 * poff[a] + j;
  double *o = out + (size_t)Nr * poff[a] + j;
  for (int t = 0; t < nterms; ++t) {
    const ProdTerm T = terms[t];
    double s = 0.0;
    if (T.a < N1 && T.b < N2) s += g1[(size_t)T.a * npts] * g2[(size_t)T.b * npts];
    if (T.a != T.b && T.b < N1 && T.a < N2) s += g1[(size_t)T.b * npts] * g2[(size_t)T.a * npts];
    o[(size_t)T.lm * npts] += T.c * s;
  }
}

// Integral of a bubble set over all space (Bubbles_integrate_pick /
// Bubbles_integrate_all, bubbles.F90:3146-3240): only the s functions
// survive, 4 pi sum_A int r^(2+k) f_A,00(r) dr with the radial grids' LIP
// weights.  One block: each atom's points are summed by the block in a
// fixed order, the atoms one after the other.
__global__ void bubbles_integrate_kernel(const double *__restrict__ f,
                                         const double *__restrict__ rpts,
                                         const double *__restrict__ w, const int *__restrict__ np,
                                         const int *__restrict__ foff, int natom, int k,
                                         double *out) {
  __shared__ double red[256];
  double total = 0.0;
  int p0 = 0;
  for (int a = 0; a < natom; ++a) {
    double s = 0.0;
    for (int j = threadIdx.x; j < np[a]; j += blockDim.x) {
      const double r = rpts[p0 + j];
      double rp = 1.0;
      for (int e = 0; e < 2 + k; ++e) rp *= r;
      s += w[p0 + j] * (f[foff[a] + j] * rp);
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
      if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
      __syncthreads();
    }
    if (threadIdx.x == 0) total += 4.0 * M_PI * red[0];
    __syncthreads();
    p0 += np[a];
  }
  if (threadIdx.x == 0) *out = total;
}

}  // namespace
}  // namespace dage

using namespace dage;


namespace dage {
namespace {
void inject_dispatch(const dage_bubbles *b, int blocks, cudaStream_t s, int lmin, const double *xs,
                     int nx, const double *ys, int ny, const double *zs, int nz, double factor,
                     double *d_cube) {
  auto go = [&](auto kernel) {
    kernel<<<blocks, 256, 0, s>>>(b->atoms.as<AtomTab>(), b->natom, b->celld.as<double>(),
                                  b->hcell.as<double>(), b->coef.as<double>(), b->N, b->lmax, lmin,
                                  b->nlip, b->first, xs, nx, ys, ny, zs, nz, factor, d_cube);
  };
  const size_t bricks = (size_t)((nx + 7) / 8) * ((ny + 7) / 8) * ((nz + 7) / 8);
  const int blocks2 = (int)std::min<size_t>(bricks, (size_t)sm_count() * 16);
  auto go2 = [&](auto kernel) {
    kernel<<<blocks2, 256, 0, s>>>(b->atoms.as<AtomTab>(), b->natom, b->celld.as<double>(),
                                   b->hcell.as<double>(), b->coef.as<double>(), b->N, lmin, b->first,
                                   xs, nx, ys, ny, zs, nz, factor, d_cube);
  };
  if (b->nlip != 7 || b->lmax > 6) go(inject_kernel<-1>);
  else if (b->lmax <= 2) go2(inject_pair_kernel<2>);
  else if (b->lmax <= 4) go2(inject_pair_kernel<4>);
  else go2(inject_pair_kernel<6>);
}
}  // namespace
}  // namespace dage

extern "C" {

int dage_bubbles_create(int natom, const double *centers, const dage_grid1d *radial, int lmax,
                        int k, const double *f, dage_bubbles **out) {
  clear_error();
  if (!out || !centers || !radial || !f) return fail(DAGE_E_INVALID, "null argument");
  *out = nullptr;
  if (natom < 1 || lmax < 0 || lmax > 12 || k < 0)
    return fail(DAGE_E_INVALID, "need natom >= 1, 0 <= lmax <= 12, k >= 0");
  auto *b = new dage_bubbles();
  auto cleanup = [&](int rc) {
    for (DevBuf *x : {&b->atoms, &b->celld, &b->hcell, &b->coef, &b->xs, &b->ys, &b->zs,
                      &b->fraw, &b->rpts, &b->np, &b->foff})
      x->release();
    delete b;
    return rc;
  };
  b->natom = natom;
  b->lmax = lmax;
  b->k = k;
  b->N = (lmax + 1) * (lmax + 1);
  cudaGetDevice(&b->device);
  const int nlip = radial[0].nlip;
  b->nlip = nlip;
  LipBasis L;
  int rc = make_lip_basis(nlip, 1, L);
  if (rc) return cleanup(rc);
  b->first = L.first;
  std::vector<AtomTab> tab(natom);
  std::vector<double> celld, hcell, rf, rpts;
  b->centers.assign(centers, centers + 3 * natom);
  b->radial.assign(radial, radial + natom);
  b->scales.resize(natom);
  std::vector<int> np(natom), foff(natom), cell0(natom + 1, 0);
  for (int a = 0; a < natom; ++a) {
    if (radial[a].nlip != nlip || radial[a].grid_type != 1)
      return cleanup(fail(DAGE_E_UNSUPPORTED, "radial grids: equidistant-point cells, one nlip"));
    Axis ax;
    rc = make_axis(radial[a], ax);
    if (rc) return cleanup(rc);
    tab[a].cx = centers[3 * a];
    tab[a].cy = centers[3 * a + 1];
    tab[a].cz = centers[3 * a + 2];
    tab[a].rmax = ax.points.back();
    tab[a].cell0 = (int)celld.size();
    tab[a].ncell = ax.ncell;
    celld.insert(celld.end(), ax.celld.begin(), ax.celld.end());
    hcell.insert(hcell.end(), ax.h.begin(), ax.h.end());
    cell0[a + 1] = cell0[a] + ax.ncell;
    np[a] = ax.n();
    foff[a] = (int)rf.size();
    rpts.insert(rpts.end(), ax.points.begin(), ax.points.end());
    b->scales[a].assign(radial[a].cell_scales, radial[a].cell_scales + ax.ncell);
    b->radial[a].cell_scales = b->scales[a].data();
    for (int lm = 0; lm < b->N; ++lm)
      for (int j = 0; j < np[a]; ++j) {
        double rp = 1.0;
        for (int e = 0; e < k; ++e) rp *= ax.points[j];
        rf.push_back(rp * f[foff[a] + (size_t)lm * np[a] + j]);
      }
    if (ax.points.front() != 0.0) return cleanup(fail(DAGE_E_INVALID, "radial grids start at r = 0"));
  }
  // upload, then LIP values -> monomial coefficients on the GPU
  TmpBuf d_rf, d_np, d_foff, d_cell0, d_lipc;
  if ((rc = b->atoms.alloc(sizeof(AtomTab) * natom)) || (rc = b->celld.alloc(sizeof(double) * celld.size())) ||
      (rc = b->hcell.alloc(sizeof(double) * hcell.size())) ||
      (rc = b->coef.alloc(sizeof(double) * 8 * (size_t)cell0[natom] * b->N)) ||
      (rc = d_rf.alloc(sizeof(double) * rf.size())) || (rc = d_np.alloc(sizeof(int) * natom)) ||
      (rc = d_foff.alloc(sizeof(int) * natom)) || (rc = d_cell0.alloc(sizeof(int) * (natom + 1))) ||
      (rc = d_lipc.alloc(sizeof(double) * L.coeff.size())))
    return cleanup(rc);
  cudaMemcpy(b->atoms.ptr, tab.data(), sizeof(AtomTab) * natom, cudaMemcpyHostToDevice);
  cudaMemcpy(b->celld.ptr, celld.data(), sizeof(double) * celld.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(b->hcell.ptr, hcell.data(), sizeof(double) * hcell.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(d_rf.ptr, rf.data(), sizeof(double) * rf.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(d_np.ptr, np.data(), sizeof(int) * natom, cudaMemcpyHostToDevice);
  cudaMemcpy(d_foff.ptr, foff.data(), sizeof(int) * natom, cudaMemcpyHostToDevice);
  cudaMemcpy(d_cell0.ptr, cell0.data(), sizeof(int) * (natom + 1), cudaMemcpyHostToDevice);
  cudaMemcpy(d_lipc.ptr, L.coeff.data(), sizeof(double) * L.coeff.size(), cudaMemcpyHostToDevice);
  // raw values and radial points for the radial potential
  b->nvals = rf.size();
  if ((rc = b->fraw.alloc(sizeof(double) * rf.size())) || (rc = b->rpts.alloc(sizeof(double) * rpts.size())) ||
      (rc = b->np.alloc(sizeof(int) * natom)) || (rc = b->foff.alloc(sizeof(int) * natom)))
    return cleanup(rc);
  {
    std::vector<double> raw(rf.size());
    std::vector<int> poff(natom);
    for (int a = 0, po = 0; a < natom; ++a) {
      for (size_t e = 0; e < (size_t)b->N * np[a]; ++e) raw[foff[a] + e] = f[foff[a] + e];
      poff[a] = po;
      po += np[a];
    }
    cudaMemcpy(b->fraw.ptr, raw.data(), sizeof(double) * raw.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(b->rpts.ptr, rpts.data(), sizeof(double) * rpts.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(b->np.ptr, np.data(), sizeof(int) * natom, cudaMemcpyHostToDevice);
    cudaMemcpy(b->foff.ptr, foff.data(), sizeof(int) * natom, cudaMemcpyHostToDevice);
  }
  const int total = cell0[natom] * b->N;
  bubble_coeffs_kernel<<<(total + 127) / 128, 128>>>(d_rf.as<double>(), d_np.as<int>(),
                                                     d_foff.as<int>(), d_cell0.as<int>(), natom,
                                                     b->N, d_lipc.as<double>(), nlip,
                                                     b->coef.as<double>());
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cleanup(fail(DAGE_E_CUDA, "bubble setup: %s", cudaGetErrorString(e)));
  *out = b;
  return 0;
}

int dage_bubbles_inject(dage_bubbles *b, const dage_grid1d grid[3], int lmin, double factor,
                        double *cube, unsigned flags);

}  // extern "C"

namespace dage {
// Stream-ordered injection into a device cube whose point coordinates are
// already on the device (allocates nothing: usable inside a stream capture).
int bubbles_inject_launch(const dage_bubbles *b, const double *xs, int nx, const double *ys,
                          int ny, const double *zs, int nz, int lmin, double factor,
                          double *d_cube, cudaStream_t s) {
  if (!b || lmin < 0 || lmin > b->lmax) return fail(DAGE_E_INVALID, "bubbles or lmin");
  const size_t n = (size_t)nx * ny * nz;
  const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)sm_count() * 16);
  inject_dispatch(b, blocks, s, lmin, xs, nx, ys, ny, zs, nz, factor, d_cube);
  DAGE_CUDA_TRY(cudaGetLastError());
  return 0;
}

namespace {
// Radial Coulomb potential of every (atom, lm) function
// (Coulomb3D_evaluate_bubbles_potential, coulomb.F90:222-336):
//   V_lm(r) = 4 pi/(2l+1) [ r^-(l+1) int_0^r f s^(l+2+k) ds + r^l int_r^inf f s^(1-l+k) ds ]
// with the cumulative LIP integrals of InOutIntegrator1D (evaluators.F90:
// 1263-1318): per cell, the values at its points from the cell's LIP
// partial integrals (outward: from its first point, inward: to its last)
// times the cell step, plus the running value at the cell boundary.
// Negative powers are 0 at r = 0 (Bubbles_rpow).  Block = atom, thread = lm;
// the outward integral is kept in V until the inward pass completes it.
template <bool HELM>
__global__ void bubbles_potential_kernel(const AtomTab *__restrict__ atoms,
                                         const double *__restrict__ hcell,
                                         const double *__restrict__ f,
                                         const double *__restrict__ rpts,
                                         const int *__restrict__ np, const int *__restrict__ foff,
                                         int lmax, int k, int nlip,
                                         const double *__restrict__ ints_out,
                                         const double *__restrict__ ints_in,
                                         const double *__restrict__ besi,
                                         const double *__restrict__ besk, int total,
                                         double kappa, double *V) {
  const int a = blockIdx.x, N = (lmax + 1) * (lmax + 1);
  const AtomTab A = atoms[a];
  int poff = 0;  // offset of this atom's points in rpts
  for (int b = 0; b < a; ++b) poff += np[b];
  const double *r = rpts + poff;
  const int n = nlip - 1, npts = np[a];
  for (int lm = threadIdx.x; lm < N; lm += blockDim.x) {
    int l = 0;
    while ((l + 1) * (l + 1) <= lm) ++l;
    const double *fl = f + foff[a] + (size_t)lm * npts;
    double *Vl = V + foff[a] + (size_t)lm * npts;
    const double *Il = besi + (size_t)l * total + poff, *Kl = besk + (size_t)l * total + poff;
    auto rpow = [&](int p, int e) {
      if (e >= 0) {
        double v = 1.0;
        for (int i = 0; i < e; ++i) v *= r[p];
        return v;
      }
      if (p == 0) return 0.0;
      double v = 1.0;
      for (int i = 0; i < -e; ++i) v *= r[p];
      return 1.0 / v;
    };
    // integrands of the outward and inward integrals at point p
    auto g_out = [&](int p) {
      return HELM ? rpow(p, 2 + k) * Il[p] * fl[p] : fl[p] * rpow(p, l + 2 + k);
    };
    auto g_in_raw = [&](int p) {
      return HELM ? rpow(p, 2 + k) * Kl[p] * fl[p] : fl[p] * rpow(p, 1 - l + k);
    };
    auto g_in = [&](int p) {
      if (HELM && p == 0)  // extrapolate_first_nlip7: order 3 for l = 0, else 0
        return l == 0 ? 3.0 * g_in_raw(1) - 3.0 * g_in_raw(2) + g_in_raw(3) : 0.0;
      return g_in_raw(p);
    };
    // outward pass: int_0^{r_p} g_out
    Vl[0] = 0.0;
    for (int c = 0; c < A.ncell; ++c) {
      const int s0 = c * n;
      const double h = hcell[A.cell0 + c], base = Vl[s0];
      for (int j = 1; j <= n; ++j) {
        double acc = 0.0;
        for (int i = 0; i <= n; ++i) acc += g_out(s0 + i) * ints_out[i * n + j - 1];
        Vl[s0 + j] = acc * h + base;
      }
    }
    // inward pass: int_{r_p}^inf g_in, combined point by point
    const double pref = HELM ? 8.0 * kappa : 4.0 * 3.141592653589793238 / (2 * l + 1);
    auto combine = [&](int p, double outv, double inv) {
      return HELM ? pref * (Kl[p] * outv + Il[p] * inv)
                  : pref * (rpow(p, -(l + 1)) * outv + rpow(p, l) * inv);
    };
    double end = 0.0;  // the inward integral at the current cell's last point
    Vl[npts - 1] = combine(npts - 1, Vl[npts - 1], 0.0);
    for (int c = A.ncell - 1; c >= 0; --c) {
      const int s0 = c * n;
      const double h = hcell[A.cell0 + c];
      double vals[8];
      for (int j = 0; j < n; ++j) {
        double acc = 0.0;
        for (int i = 0; i <= n; ++i) acc += g_in(s0 + i) * ints_in[i * n + j];
        vals[j] = acc * h + end;
      }
      for (int j = 0; j < n; ++j) Vl[s0 + j] = combine(s0 + j, Vl[s0 + j], vals[j]);
      end = vals[0];
    }
  }
}

// i_l(kappa r), k_l(kappa r) for l <= lmax at every radial point (thread =
// point): i_l by its power series for l = lmax, lmax - 1 and downward
// recursion, k_l from k_0 = pi/2 e^-x/x, k_1 = pi/2 e^-x (x+1)/x^2 and upward
// recursion (FirstModSphBesselCollection / SecondModSphBesselCollection,
// helmholtz3d.F90:851-1060, there in 128-bit arithmetic); both 0 except
// i_0 = 1 at x = 0.  Output rows [l][point].
__device__ double besseli_series(double x, int n) {
  double pref = 1.0;
  for (int j = 1; j <= n; ++j) pref *= x / (2 * j + 1);
  const double a = 0.5 * x * x;
  double term = 1.0, sum = 1.0;
  for (int i = 1; i < 300; ++i) {
    term *= a / (i * (2.0 * n + 2 * i + 1));
    sum += term;
    if (term <= 1e-17 * sum) break;
  }
  return pref * sum;
}

__global__ void bessel_tables_kernel(const double *__restrict__ rpts, int total, int lmax,
                                     double kappa, double *besi, double *besk) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= total) return;
  const double x = kappa * rpts[p];
  if (!(x > 2.220446049250313e-16)) {
    for (int l = 0; l <= lmax; ++l) {
      besi[(size_t)l * total + p] = l == 0 ? 1.0 : 0.0;
      besk[(size_t)l * total + p] = 0.0;
    }
    return;
  }
  if (lmax == 0) {
    besi[p] = besseli_series(x, 0);
  } else {
    double up = besseli_series(x, lmax), cur = besseli_series(x, lmax - 1);
    besi[(size_t)lmax * total + p] = up;
    besi[(size_t)(lmax - 1) * total + p] = cur;
    for (int l = lmax - 2; l >= 0; --l) {
      const double v = (2 * l + 3) * cur / x + up;
      besi[(size_t)l * total + p] = v;
      up = cur;
      cur = v;
    }
  }
  const double hp = 1.5707963267948966;
  double k0 = hp * exp(-x) / x;
  besk[p] = k0;
  if (lmax >= 1) {
    double k1 = hp * exp(-x) * (x + 1.0) / (x * x);
    besk[(size_t)total + p] = k1;
    for (int l = 2; l <= lmax; ++l) {
      const double v = (2 * l - 1) * k1 / x + k0;
      besk[(size_t)l * total + p] = v;
      k0 = k1;
      k1 = v;
    }
  }
}

// Gauss-Legendre nodes and weights on [-1, 1]: Newton's method on P_n from
// the three-term recurrence, started at cos(pi (i - 1/4) / (n + 1/2)).
void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 1.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; ++k) {
        const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (z * p1 - p0) / (z * z - 1.0);
      const double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; ++k) {
        const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (z * p1 - p0) / (z * z - 1.0);
    }
    x[i] = -z;
    x[n - 1 - i] = z;
    w[i] = w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
}

}  // namespace

// Expansion of products of real harmonics, Y_a Y_b = sum C_ab^LM Y_LM
// (the table of YProduct_init, harmonic.F90:884-951), for a <= b < (lmax+1)^2
// and L <= result_lmax.  Each coefficient is the projection
//   C = (2L+1)/(4 pi) * int Y_a Y_b Y_LM dOmega
// (the Racah-normalised Y_LM have norm 4 pi/(2L+1)), by a Gauss-Legendre x
// trapezoid product rule exact for the polynomial degrees involved.  Only
// the (L, M) that the parity and m selection rules allow are projected.
// Unless `complete`, the reference's term set is kept: its enumeration
// (harmonic.F90:914-926) leaves out every term with L < |m1 - m2|, whose
// content then stays in the cube part of a product.
std::vector<ProdTerm> product_table(int lmax, int result_lmax, bool complete) {
  const int deg = 2 * lmax + result_lmax;
  const int nz = deg / 2 + 2, nphi = deg + 2;
  std::vector<double> zx, zw;
  gauss_legendre(nz, zx, zw);
  const int L = std::max(lmax, result_lmax), NY = (L + 1) * (L + 1);
  std::vector<double> Y((size_t)nz * nphi * NY), W((size_t)nz * nphi);
  for (int i = 0; i < nz; ++i)
    for (int j = 0; j < nphi; ++j) {
      const double st = std::sqrt(1.0 - zx[i] * zx[i]), ph = 2.0 * M_PI * j / nphi;
      double *y = &Y[((size_t)i * nphi + j) * NY];
      unit_harmonics(L, st * std::cos(ph), st * std::sin(ph), zx[i],
                     [&](int lm, double v) { y[lm] = v; });
      W[(size_t)i * nphi + j] = zw[i] * 2.0 * M_PI / nphi;
    }
  const size_t nodes = (size_t)nz * nphi;
  std::vector<double> P(nodes);
  std::vector<ProdTerm> out;
  const int N = (lmax + 1) * (lmax + 1);
  for (int a = 0; a < N; ++a) {
    const int l1 = (int)std::sqrt((double)a), m1 = a - l1 * (l1 + 1);
    for (int b = a; b < N; ++b) {
      const int l2 = (int)std::sqrt((double)b), m2 = b - l2 * (l2 + 1);
      for (size_t q = 0; q < nodes; ++q) P[q] = Y[q * NY + a] * Y[q * NY + b] * W[q];
      const int ms[4] = {std::abs(m1 - m2), -std::abs(m1 - m2), std::abs(m1 + m2),
                         -std::abs(m1 + m2)};
      for (int l = std::abs(l1 - l2); l <= std::min(l1 + l2, result_lmax); l += 2) {
        if (!complete && l < std::abs(m1 - m2)) continue;
        for (int e = 0; e < 4; ++e) {
          const int m = ms[e];
          bool dup = std::abs(m) > l;
          for (int f = 0; f < e; ++f) dup = dup || ms[f] == m;
          if (dup) continue;
          double c = 0.0;
          for (size_t q = 0; q < nodes; ++q) c += P[q] * Y[q * NY + l * (l + 1) + m];
          c *= (2.0 * l + 1.0) / (4.0 * M_PI);
          if (std::fabs(c) > 1e-13) out.push_back({a, b, l * (l + 1) + m, 0, c});
        }
      }
    }
  }
  return out;
}

// Same atoms (centres) and the same radial grids: the product routines share
// every atom's radial cell between the sets.
bool same_layout(const dage_bubbles *x, const dage_bubbles *y) {
  if (x->natom != y->natom || x->nlip != y->nlip || x->centers != y->centers) return false;
  for (int a = 0; a < x->natom; ++a)
    if (x->radial[a].ncell != y->radial[a].ncell || x->scales[a] != y->scales[a]) return false;
  return true;
}

}  // namespace dage

extern "C" {

int dage_bubbles_inject(dage_bubbles *b, const dage_grid1d grid[3], int lmin, double factor,
                        double *cube, unsigned flags) {
  clear_error();
  if (!b || !grid || !cube) return fail(DAGE_E_INVALID, "null argument");
  if (lmin < 0 || lmin > b->lmax) return fail(DAGE_E_INVALID, "lmin out of range");
  DAGE_CUDA_TRY(cudaSetDevice(b->device));
  Axis ax[3];
  for (int d = 0; d < 3; ++d) DAGE_TRY(make_axis(grid[d], ax[d]));
  DevBuf *bufs[3] = {&b->xs, &b->ys, &b->zs};
  for (int d = 0; d < 3; ++d) {
    DAGE_TRY(bufs[d]->alloc(sizeof(double) * ax[d].n()));
    DAGE_CUDA_TRY(cudaMemcpy(bufs[d]->ptr, ax[d].points.data(), sizeof(double) * ax[d].n(),
                             cudaMemcpyHostToDevice));
  }
  const size_t n = (size_t)ax[0].n() * ax[1].n() * ax[2].n();
  TmpBuf staging;
  double *d_cube = cube;
  if (!(flags & DAGE_DEVICE_PTRS)) {
    DAGE_TRY(staging.alloc(sizeof(double) * n));
    DAGE_CUDA_TRY(cudaMemcpy(staging.ptr, cube, sizeof(double) * n, cudaMemcpyHostToDevice));
    d_cube = staging.as<double>();
  }
  const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)sm_count() * 16);
  inject_dispatch(b, blocks, 0, lmin, b->xs.as<double>(), ax[0].n(), b->ys.as<double>(),
                  ax[1].n(), b->zs.as<double>(), ax[2].n(), factor, d_cube);
  DAGE_CUDA_TRY(cudaGetLastError());
  if (!(flags & DAGE_DEVICE_PTRS))
    DAGE_CUDA_TRY(cudaMemcpy(cube, d_cube, sizeof(double) * n, cudaMemcpyDeviceToHost));
  DAGE_CUDA_TRY(cudaDeviceSynchronize());
  return 0;
}

}  // extern "C"

namespace dage {
namespace {
// Radial Coulomb (helm = false) or Helmholtz (kernel e^-kappa r / r) potential
// of every (atom, lm) function, as a new bubble set with k = 0.
int bubbles_radial_potential(const dage_bubbles *in, bool helm, double kappa, dage_bubbles **out) {
  DAGE_CUDA_TRY(cudaSetDevice(in->device));
  // LIP partial integrals on the local nodes (LIPBasis_outward/inward_integrals,
  // lip.F90:414-480): antiderivative of each basis polynomial by Horner
  LipBasis L;
  DAGE_TRY(make_lip_basis(in->nlip, 1, L));
  const int nl = in->nlip, n = nl - 1;
  std::vector<double> outi((size_t)nl * n), ini((size_t)nl * n);
  auto anti = [&](int i, double x) {
    double v = 0.0;
    for (int kk = 0; kk < nl; ++kk) v = (v + L.coeff[(size_t)kk * nl + i] / (double)(nl - kk)) * x;
    return v;
  };
  for (int i = 0; i < nl; ++i)
    for (int j = 0; j < n; ++j) {
      outi[(size_t)i * n + j] = anti(i, L.first + j + 1) - anti(i, L.first);
      ini[(size_t)i * n + j] = anti(i, L.last) - anti(i, L.first + j);
    }
  TmpBuf d_out, d_in, d_V;
  DAGE_TRY(d_out.alloc(sizeof(double) * outi.size()));
  DAGE_TRY(d_in.alloc(sizeof(double) * ini.size()));
  DAGE_TRY(d_V.alloc(sizeof(double) * in->nvals));
  DAGE_CUDA_TRY(cudaMemcpy(d_out.ptr, outi.data(), sizeof(double) * outi.size(), cudaMemcpyHostToDevice));
  DAGE_CUDA_TRY(cudaMemcpy(d_in.ptr, ini.data(), sizeof(double) * ini.size(), cudaMemcpyHostToDevice));
  const int total = (int)(in->nvals / in->N);
  TmpBuf d_I, d_K;
  if (helm) {
    DAGE_TRY(d_I.alloc(sizeof(double) * (size_t)(in->lmax + 1) * total));
    DAGE_TRY(d_K.alloc(sizeof(double) * (size_t)(in->lmax + 1) * total));
    bessel_tables_kernel<<<(total + 127) / 128, 128>>>(in->rpts.as<double>(), total, in->lmax, kappa,
                                                       d_I.as<double>(), d_K.as<double>());
  }
  auto go = [&](auto kernel) {
    kernel<<<in->natom, std::min(256, ((in->N + 31) / 32) * 32)>>>(
        in->atoms.as<AtomTab>(), in->hcell.as<double>(), in->fraw.as<double>(),
        in->rpts.as<double>(), in->np.as<int>(), in->foff.as<int>(), in->lmax, in->k, in->nlip,
        d_out.as<double>(), d_in.as<double>(), d_I.as<double>(), d_K.as<double>(), total, kappa,
        d_V.as<double>());
  };
  if (helm) go(bubbles_potential_kernel<true>);
  else go(bubbles_potential_kernel<false>);
  DAGE_CUDA_TRY(cudaGetLastError());
  std::vector<double> V(in->nvals);
  DAGE_CUDA_TRY(cudaMemcpy(V.data(), d_V.ptr, sizeof(double) * V.size(), cudaMemcpyDeviceToHost));
  // the potential is a bubble set of its own (k = 0) on the same centres and grids
  return dage_bubbles_create(in->natom, in->centers.data(), in->radial.data(), in->lmax, 0,
                             V.data(), out);
}
}  // namespace
}  // namespace dage

extern "C" {

int dage_bubbles_coulomb_potential(const dage_bubbles *in, dage_bubbles **out) {
  clear_error();
  if (!in || !out) return fail(DAGE_E_INVALID, "null argument");
  *out = nullptr;
  return bubbles_radial_potential(in, false, 0.0, out);
}

int dage_bubbles_helmholtz_potential(const dage_bubbles *in, double energy, dage_bubbles **out) {
  clear_error();
  if (!in || !out) return fail(DAGE_E_INVALID, "null argument");
  *out = nullptr;
  if (!(energy < 0.0)) return fail(DAGE_E_INVALID, "Helmholtz bubbles: need energy < 0");
  // the r = 0 extrapolation reads the first four radial points of every atom
  for (int a = 0; a < in->natom; ++a)
    if (in->radial[a].ncell * (in->nlip - 1) + 1 < 4)
      return fail(DAGE_E_UNSUPPORTED, "Helmholtz bubbles: every radial grid needs >= 4 points");
  return bubbles_radial_potential(in, true, std::sqrt(-2.0 * energy), out);
}

int dage_bubbles_multiply(const dage_bubbles *x, const dage_bubbles *y, unsigned flags,
                          dage_bubbles **out) {
  clear_error();
  if (!x || !y || !out) return fail(DAGE_E_INVALID, "null argument");
  *out = nullptr;
  if (!same_layout(x, y))
    return fail(DAGE_E_UNSUPPORTED, "bubble product: the sets need the same atoms and radial grids");
  const int lr = x->lmax + y->lmax;
  if (lr > 12) return fail(DAGE_E_INVALID, "bubble product: lmax1 + lmax2 > 12");
  DAGE_CUDA_TRY(cudaSetDevice(x->device));
  const std::vector<ProdTerm> terms =
      product_table(std::max(x->lmax, y->lmax), lr, (flags & DAGE_PRODUCT_COMPLETE) != 0);
  const int Nr = (lr + 1) * (lr + 1);
  std::vector<int> poff(x->natom + 1, 0), np(x->natom);
  for (int a = 0; a < x->natom; ++a) {
    np[a] = x->radial[a].ncell * (x->nlip - 1) + 1;
    poff[a + 1] = poff[a] + np[a];
  }
  const size_t nout = (size_t)Nr * poff[x->natom];
  TmpBuf d_terms, d_np, d_poff, d_out;
  DAGE_TRY(d_terms.alloc(sizeof(ProdTerm) * std::max<size_t>(terms.size(), 1)));
  DAGE_TRY(d_np.alloc(sizeof(int) * np.size()));
  DAGE_TRY(d_poff.alloc(sizeof(int) * poff.size()));
  DAGE_TRY(d_out.alloc(sizeof(double) * nout));
  DAGE_CUDA_TRY(cudaMemcpy(d_terms.ptr, terms.data(), sizeof(ProdTerm) * terms.size(),
                           cudaMemcpyHostToDevice));
  DAGE_CUDA_TRY(cudaMemcpy(d_np.ptr, np.data(), sizeof(int) * np.size(), cudaMemcpyHostToDevice));
  DAGE_CUDA_TRY(cudaMemcpy(d_poff.ptr, poff.data(), sizeof(int) * poff.size(), cudaMemcpyHostToDevice));
  DAGE_CUDA_TRY(cudaMemset(d_out.ptr, 0, sizeof(double) * nout));
  const int total = poff[x->natom];
  bubbles_product_kernel<<<(total + 127) / 128, 128>>>(
      x->fraw.as<double>(), x->N, y->fraw.as<double>(), y->N, d_np.as<int>(), d_poff.as<int>(),
      x->natom, d_terms.as<ProdTerm>(), (int)terms.size(), Nr, d_out.as<double>());
  DAGE_CUDA_TRY(cudaGetLastError());
  std::vector<double> prod(nout);
  DAGE_CUDA_TRY(cudaMemcpy(prod.data(), d_out.ptr, sizeof(double) * nout, cudaMemcpyDeviceToHost));
  return dage_bubbles_create(x->natom, x->centers.data(), x->radial.data(), lr, x->k + y->k,
                             prod.data(), out);
}

int dage_product_table(int lmax, int result_lmax, unsigned flags, int cap, int *a, int *b, int *lm,
                       double *c, int *nterms) {
  clear_error();
  if (!nterms || lmax < 0 || lmax > 12 || result_lmax < 0 || result_lmax > 24)
    return fail(DAGE_E_INVALID, "need 0 <= lmax <= 12, 0 <= result_lmax <= 24");
  const std::vector<ProdTerm> t = product_table(lmax, result_lmax, (flags & DAGE_PRODUCT_COMPLETE) != 0);
  *nterms = (int)t.size();
  if (cap < (int)t.size() || !a || !b || !lm || !c) return 0;
  for (size_t i = 0; i < t.size(); ++i) {
    a[i] = t[i].a;
    b[i] = t[i].b;
    lm[i] = t[i].lm;
    c[i] = t[i].c;
  }
  return 0;
}

int dage_function3d_multiply(const dage_grid1d grid[3], const double *cube1, const dage_bubbles *b1,
                             const double *cube2, const dage_bubbles *b2, const dage_bubbles *br,
                             double *out, unsigned flags) {
  clear_error();
  if (!grid || !cube1 || !cube2 || !out) return fail(DAGE_E_INVALID, "null argument");
  const dage_bubbles *sets[3] = {b1, b2, br};
  const dage_bubbles *ref = nullptr;
  for (const dage_bubbles *s : sets)
    if (s) {
      if (ref && !same_layout(ref, s))
        return fail(DAGE_E_UNSUPPORTED,
                    "function product: the bubble sets need the same atoms and radial grids");
      if (!ref) ref = s;
    }
  Axis ax[3];
  for (int d = 0; d < 3; ++d) DAGE_TRY(make_axis(grid[d], ax[d]));
  const size_t n = (size_t)ax[0].n() * ax[1].n() * ax[2].n();
  TmpBuf pts[3], s1, s2, so;
  for (int d = 0; d < 3; ++d) {
    DAGE_TRY(pts[d].alloc(sizeof(double) * ax[d].n()));
    DAGE_CUDA_TRY(cudaMemcpy(pts[d].ptr, ax[d].points.data(), sizeof(double) * ax[d].n(),
                             cudaMemcpyHostToDevice));
  }
  const double *d1 = cube1, *d2 = cube2;
  double *dout = out;
  if (!(flags & DAGE_DEVICE_PTRS)) {
    DAGE_TRY(s1.alloc(sizeof(double) * n));
    DAGE_TRY(s2.alloc(sizeof(double) * n));
    DAGE_TRY(so.alloc(sizeof(double) * n));
    DAGE_CUDA_TRY(cudaMemcpy(s1.ptr, cube1, sizeof(double) * n, cudaMemcpyHostToDevice));
    DAGE_CUDA_TRY(cudaMemcpy(s2.ptr, cube2, sizeof(double) * n, cudaMemcpyHostToDevice));
    d1 = s1.as<double>();
    d2 = s2.as<double>();
    dout = so.as<double>();
  }
  int lmax = 0;
  for (const dage_bubbles *s : sets)
    if (s) lmax = std::max(lmax, s->lmax);
  auto coef = [&](const dage_bubbles *s) { return s ? s->coef.as<double>() : nullptr; };
  auto rows = [&](const dage_bubbles *s) { return s ? s->N : 0; };
  const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)sm_count() * 16);
  const int nlip = ref ? ref->nlip : 7;
  auto go = [&](auto kernel) {
    kernel<<<blocks, 256>>>(
        ref ? ref->atoms.as<AtomTab>() : nullptr, ref ? ref->natom : 0,
        ref ? ref->celld.as<double>() : nullptr, ref ? ref->hcell.as<double>() : nullptr,
        coef(b1), rows(b1), coef(b2), rows(b2), coef(br), rows(br), lmax, nlip,
        ref ? ref->first : 0.0, pts[0].as<double>(), ax[0].n(), pts[1].as<double>(), ax[1].n(),
        pts[2].as<double>(), ax[2].n(), d1, d2, dout);
  };
  auto go2 = [&](auto kernel) {
    const size_t bricks = (size_t)((ax[0].n() + 7) / 8) * ((ax[1].n() + 7) / 8) * ((ax[2].n() + 7) / 8);
    const int blocks2 = (int)std::min<size_t>(bricks, (size_t)sm_count() * 16);
    kernel<<<blocks2, 256>>>(
        ref ? ref->atoms.as<AtomTab>() : nullptr, ref ? ref->natom : 0,
        ref ? ref->celld.as<double>() : nullptr, ref ? ref->hcell.as<double>() : nullptr,
        coef(b1), rows(b1), coef(b2), rows(b2), coef(br), rows(br), ref ? ref->first : 0.0,
        pts[0].as<double>(), ax[0].n(), pts[1].as<double>(), ax[1].n(), pts[2].as<double>(),
        ax[2].n(), d1, d2, dout);
  };
  // harmonics passes: the factors' sets up to lb, the result set up to lr
  int lb = 0, lr = 0;
  for (const dage_bubbles *x : {b1, b2})
    if (x) lb = std::max(lb, x->lmax);
  if (br) lr = br->lmax;
  auto up = [](int l) { return l <= 2 ? 2 : l <= 4 ? 4 : 6; };
  const int kb = up(lb), kr = std::max(up(lr), kb);
  if (nlip != 7 || lmax > 6) go(function_product_kernel<-1>);
  else if (kb == 2 && kr == 2) go2(function_product_pair_kernel<2, 2>);
  else if (kb == 2 && kr == 4) go2(function_product_pair_kernel<2, 4>);
  else if (kb == 2) go2(function_product_pair_kernel<2, 6>);
  else if (kb == 4 && kr == 4) go2(function_product_pair_kernel<4, 4>);
  else if (kb == 4) go2(function_product_pair_kernel<4, 6>);
  else go2(function_product_pair_kernel<6, 6>);
  DAGE_CUDA_TRY(cudaGetLastError());
  if (!(flags & DAGE_DEVICE_PTRS))
    DAGE_CUDA_TRY(cudaMemcpy(out, dout, sizeof(double) * n, cudaMemcpyDeviceToHost));
  DAGE_CUDA_TRY(cudaDeviceSynchronize());
  return 0;
}

int dage_bubbles_integrate(const dage_bubbles *b, double *out) {
  clear_error();
  if (!b || !out) return fail(DAGE_E_INVALID, "null argument");
  DAGE_CUDA_TRY(cudaSetDevice(b->device));
  // LIP integration weights of every atom's radial points, in the layout of
  // the radial points (atoms one after the other)
  std::vector<double> w;
  std::vector<int> np(b->natom), foff(b->natom);
  for (int a = 0; a < b->natom; ++a) {
    Axis ax;
    DAGE_TRY(make_axis(b->radial[a], ax));
    np[a] = ax.n();
    foff[a] = (int)((size_t)b->N * w.size());
    w.insert(w.end(), ax.weights.begin(), ax.weights.end());
  }
  TmpBuf d_w, d_i, d_out;
  DAGE_TRY(d_w.alloc(sizeof(double) * w.size()));
  DAGE_TRY(d_i.alloc(sizeof(int) * 2 * b->natom));
  DAGE_TRY(d_out.alloc(sizeof(double)));
  DAGE_CUDA_TRY(cudaMemcpy(d_w.ptr, w.data(), sizeof(double) * w.size(), cudaMemcpyHostToDevice));
  DAGE_CUDA_TRY(cudaMemcpy(d_i.ptr, np.data(), sizeof(int) * b->natom, cudaMemcpyHostToDevice));
  DAGE_CUDA_TRY(cudaMemcpy(d_i.as<int>() + b->natom, foff.data(), sizeof(int) * b->natom,
                           cudaMemcpyHostToDevice));
  bubbles_integrate_kernel<<<1, 256>>>(b->fraw.as<double>(), b->rpts.as<double>(), d_w.as<double>(),
                                       d_i.as<int>(), d_i.as<int>() + b->natom, b->natom, b->k,
                                       d_out.as<double>());
  DAGE_CUDA_TRY(cudaGetLastError());
  DAGE_CUDA_TRY(cudaMemcpy(out, d_out.ptr, sizeof(double), cudaMemcpyDeviceToHost));
  return 0;
}

int dage_bubbles_get_f(const dage_bubbles *b, double *f) {
  clear_error();
  if (!b || !f) return fail(DAGE_E_INVALID, "null argument");
  DAGE_CUDA_TRY(cudaSetDevice(b->device));
  DAGE_CUDA_TRY(cudaMemcpy(f, b->fraw.ptr, sizeof(double) * b->nvals, cudaMemcpyDeviceToHost));
  return 0;
}

int dage_bubbles_destroy(dage_bubbles *b) {
  if (!b) return 0;
  for (DevBuf *x : {&b->atoms, &b->celld, &b->hcell, &b->coef, &b->xs, &b->ys, &b->zs, &b->fraw,
                    &b->rpts, &b->np, &b->foff})
    x->release();
  delete b;
  return 0;
}

}  // extern "C"
