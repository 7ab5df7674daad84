// bubbles.cuh -- internal state of a bubble set and the pieces the bubble
// kernels share: the atom table, the Racah-normalised real spherical
// harmonics of a unit vector, the radial cell search and the real-harmonic
// product table.
#pragma once

#include <vector>

#include "common.cuh"
#include "grid_host.h"

namespace dage {

struct AtomTab {
  double cx, cy, cz, rmax;
  int cell0, ncell;
};

struct ProdTerm {
  int a, b, lm, pad;
  double c;
};

// Racah-normalised real spherical harmonics of a unit vector: the regular
// solid-harmonic recursion with r^2 = 1, visiting each (l, m) once.
template <class F>
__host__ __device__ __forceinline__ void unit_harmonics(int lmax, double x, double y, double z, F &&f) {
  f(0, 1.0);
  if (lmax == 0) return;
  {
    double p2 = 1.0, p1 = z;
    f(2, z);
    for (int l = 2; l <= lmax; ++l) {
      double cur = (2.0 * l - 1.0) * (z * p1) - sqrt((double)((l - 1) * (l - 1))) * p2;
      cur = cur * (1.0 / sqrt((double)(l * l)));
      f(l * (l + 1), cur);
      p2 = p1;
      p1 = cur;
    }
  }
  double top = x, bot = y;
  for (int mm = 1; mm <= lmax; ++mm) {
    if (mm >= 2) {
      const double c = sqrt(1.0 - 0.5 / mm);
      const double nb = c * (top * y + bot * x);
      const double nt = c * (top * x - bot * y);
      top = nt;
      bot = nb;
    }
    f(mm * (mm + 1) + mm, top);
    f(mm * (mm + 1) - mm, bot);
#pragma unroll 1
    for (int sg = 0; sg < 2; ++sg) {
      const int m = sg ? -mm : mm;
      double p2 = 0.0, p1 = sg ? bot : top;
      for (int l = mm + 1; l <= lmax; ++l) {
        double cur = (2.0 * l - 1.0) * (p1 * z);
        if (l - mm > 1) cur = cur - sqrt((l + m - 1.0) * (l - m - 1.0)) * p2;
        cur = (1.0 / sqrt(1.0 * (l - m) * (l + m))) * cur;
        f(l * (l + 1) + m, cur);
        p2 = p1;
        p1 = cur;
      }
    }
  }
}

// Radial cell of distance d (1-based, Grid1D_get_icell, grid.F90:1212-1245)
// for 0 <= d <= rmax; callers test d against rmax first.
__device__ __forceinline__ int radial_cell(const double *cd, int ncell, double d) {
  if (cd[ncell - 1] <= d) return ncell;
  int icell = ncell / 2, maxi = ncell - 1, mini = 1;
  for (int it = 0; it < 64; ++it) {
    if (d >= cd[icell]) {
      if (d < cd[icell + 1]) return icell + 1;
      mini = icell + 2;
    } else {
      if (d >= cd[icell - 1]) return icell;
      maxi = icell - 1;
    }
    icell = (mini + maxi) / 2;
  }
  return 0;
}

}  // namespace dage

struct dage_bubbles {
  using DevBuf = dage::DevBuf;
  int device = 0, natom = 0, lmax = 0, k = 0, nlip = 7, N = 1;
  double first = -3.0;
  DevBuf atoms, celld, hcell, coef, xs, ys, zs;
  int gshape[3] = {0, 0, 0};
  // the radial values as given (without r^k), the radial points, per-atom
  // point counts and offsets; host copies of the centres and radial grids
  DevBuf fraw, rpts, np, foff;
  std::vector<double> centers;
  std::vector<dage_grid1d> radial;
  std::vector<std::vector<double>> scales;
  size_t nvals = 0;
};

namespace dage {

// Expansion of products of real harmonics, Y_a Y_b = sum C_ab^LM Y_LM, for
// a <= b < (lmax+1)^2 and L <= result_lmax (bubbles.cu).
std::vector<ProdTerm> product_table(int lmax, int result_lmax, bool complete);

// Same atoms (centres) and the same radial grids.
bool same_layout(const dage_bubbles *x, const dage_bubbles *y);

}  // namespace dage
