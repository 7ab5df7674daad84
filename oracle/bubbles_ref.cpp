// bubbles_ref.cpp -- CPU FP64 oracle for the bubbles -> cube injection.
//
// TEST INFRASTRUCTURE ONLY (see dage_oracle.h).  Restates Bubbles_eval_pick
// for k >= 0 (src/bubbles/bubbles.F90:1904-1975): for every cube point and
// atom A, the radial function r^k f_lm is interpolated with the 7-point LIP
// basis of A's radial grid at |r - R_A| (Interpolator1D_eval_array,
// src/bubbles/evaluators.F90:631-690, cell search Grid1D_get_icell,
// grid.F90:1212-1245) and multiplied by Y_lm(r - R_A), the Racah-normalised
// real solid harmonic of the unit vector (YBundle, harmonic.F90:612-660).
#include <cmath>
#include <vector>

#include "dage_oracle.h"

namespace {

int get_icell(const std::vector<double> &celld, double qmin, double qmax, double x) {
  const int ncell = (int)celld.size();
  if (x > qmax || x < qmin) return 0;
  if (celld[ncell - 1] <= x) return ncell;
  int icell = ncell / 2, maxi = ncell - 1, mini = 1;
  while (true) {  // 1-based cells, celld[c-1] is the start of cell c
    if (x >= celld[icell]) {
      if (x < celld[icell + 1]) return icell + 1;
      mini = icell + 2;
      icell = (mini + maxi) / 2;
    } else {
      if (x >= celld[icell - 1]) return icell;
      maxi = icell - 1;
      icell = (mini + maxi) / 2;
    }
  }
}

}  // namespace

extern "C" int orc_bubbles_inject(int natom, const double *centers, const int *ncell,
                                  const double *cell_scales, int nlip, int lmax, int lmin, int k,
                                  const double *f, int nx, const double *x, int ny,
                                  const double *y, int nz, const double *z, double factor,
                                  double *cube) {
  double lipc[64], first, last;
  if (orc_lip_coeffs(nlip, 1, lipc, &first, &last)) return -1;
  const int N = (lmax + 1) * (lmax + 1);
  // per-atom radial grids (qmin = 0) and r^k f
  std::vector<std::vector<double>> celld(natom), pts(natom), rf(natom);
  std::vector<std::vector<double>> hs(natom);
  size_t off_h = 0, off_f = 0;
  for (int a = 0; a < natom; ++a) {
    const int nc = ncell[a], np = nc * (nlip - 1) + 1;
    hs[a].assign(cell_scales + off_h, cell_scales + off_h + nc);
    off_h += nc;
    pts[a].resize(np);
    celld[a].resize(nc);
    orc_grid1d_points(0.0, nc, nlip, 1, hs[a].data(), pts[a].data(), celld[a].data());
    rf[a].resize((size_t)N * np);
    for (int lm = 0; lm < N; ++lm)
      for (int j = 0; j < np; ++j) {
        double rp = 1.0;
        for (int e = 0; e < k; ++e) rp *= pts[a][j];
        rf[a][(size_t)lm * np + j] = rp * f[off_f + (size_t)lm * np + j];
      }
    off_f += (size_t)N * np;
  }
  std::vector<double> S(N), polys(nlip);
#pragma omp parallel for schedule(static) firstprivate(S, polys)
  for (int kz = 0; kz < nz; ++kz)
    for (int jy = 0; jy < ny; ++jy)
      for (int ix = 0; ix < nx; ++ix) {
        double acc = 0.0;
        for (int a = 0; a < natom; ++a) {
          const double dx = x[ix] - centers[3 * a], dy = y[jy] - centers[3 * a + 1],
                       dz = z[kz] - centers[3 * a + 2];
          const double d = std::sqrt(dx * dx + dy * dy + dz * dz);
          const int ic = get_icell(celld[a], pts[a].front(), pts[a].back(), d);
          if (ic == 0) continue;
          const double t = (d - celld[a][ic - 1]) / hs[a][ic - 1] + first;
          for (int j = 0; j < nlip; ++j) {  // eval_polys (lip.F90:541-554)
            double v = lipc[j];
            for (int kk = 1; kk < nlip; ++kk) v = v * t + lipc[(size_t)kk * nlip + j];
            polys[j] = v;
          }
          if (d > 0.0) {
            orc_solid_harmonics(lmax, dx / d, dy / d, dz / d, S.data());
          } else {
            for (int s = 0; s < N; ++s) S[s] = s == 0 ? 1.0 : 0.0;
          }
          const int start = (ic - 1) * (nlip - 1);
          const int np = (int)pts[a].size();
          for (int lm = lmin * lmin; lm < N; ++lm) {
            double v = 0.0;
            for (int j = 0; j < nlip; ++j) v += rf[a][(size_t)lm * np + start + j] * polys[j];
            acc += v * S[lm];
          }
        }
        double &c = cube[(size_t)nx * ny * kz + (size_t)nx * jy + ix];
        c = c + factor * acc;
      }
  return 0;
}
