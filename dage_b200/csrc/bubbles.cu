// bubbles.cu -- bubbles -> cube injection on one B200.
//
//   cube(r) += factor * sum_atoms sum_{l >= lmin} sum_m [r^k f_lm](|r - R|) Y_lm(r - R)
//
// The radial functions live on per-atom LIP grids (7-point cells starting at
// r = 0).  At creation each cell's LIP values are turned into monomial
// coefficients in the cell coordinate (the reference's calc_cf,
// src/bubbles/bubbles_cuda.cu:197-300), on the GPU, once per bubble set.  The
// injection is ONE kernel over all atoms: every thread owns cube points,
// loops over the atoms (centres, radial cell starts and steps staged in
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

#include "common.cuh"
#include "grid_host.h"

struct dage_bubbles;

namespace dage {
namespace {

constexpr int kMaxAtomsSmem = 256;

// Racah-normalised real spherical harmonics of a unit vector: the regular
// solid-harmonic recursion with r^2 = 1, visiting each (l, m) once.
template <class F>
__device__ __forceinline__ void unit_harmonics(int lmax, double x, double y, double z, F &&f) {
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

struct AtomTab {
  double cx, cy, cz, rmax;
  int cell0, ncell;
};

__global__ void __launch_bounds__(256)
    inject_kernel(const AtomTab *__restrict__ atoms, int natom, const double *__restrict__ celld,
                  const double *__restrict__ hcell, const double *__restrict__ coef, int N,
                  int lmax, int lmin, int nlip, double first, const double *__restrict__ xs,
                  int nx, const double *__restrict__ ys, int ny, const double *__restrict__ zs,
                  int nz, double factor, double *cube) {
  __shared__ AtomTab sa[kMaxAtomsSmem];
  for (int a = threadIdx.x; a < natom && a < kMaxAtomsSmem; a += blockDim.x) sa[a] = atoms[a];
  __syncthreads();
  const long long n = (long long)nx * ny * nz;
  const int lm0 = lmin * lmin;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(i % nx);
    const long long r = i / nx;
    const int iy = (int)(r % ny), iz = (int)(r / ny);
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
      unit_harmonics(lmax, ux, uy, uz, [&](int lm, double Y) {
        if (lm < lm0) return;
        if (at_centre && lm > 0) return;
        const double *c = cf + (size_t)lm * 8;
        double v = c[0];
        for (int kk = 1; kk < nlip; ++kk) v = v * t + c[kk];
        acc += v * Y;
      });
    }
    cube[i] += factor * acc;
  }
}

}  // namespace
}  // namespace dage

using namespace dage;

struct dage_bubbles {
  int device = 0, natom = 0, lmax = 0, k = 0, nlip = 7, N = 1;
  double first = -3.0;
  DevBuf atoms, celld, hcell, coef, xs, ys, zs;
  int gshape[3] = {0, 0, 0};
};

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
    for (DevBuf *x : {&b->atoms, &b->celld, &b->hcell, &b->coef, &b->xs, &b->ys, &b->zs}) x->release();
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
  std::vector<double> celld, hcell, rf;
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
    for (int lm = 0; lm < b->N; ++lm)
      for (int j = 0; j < np[a]; ++j) {
        double rp = 1.0;
        for (int e = 0; e < k; ++e) rp *= ax.points[j];
        rf.push_back(rp * f[foff[a] + (size_t)lm * np[a] + j]);
      }
    if (ax.points.front() != 0.0) return cleanup(fail(DAGE_E_INVALID, "radial grids start at r = 0"));
  }
  // upload, then LIP values -> monomial coefficients on the GPU
  DevBuf d_rf, d_np, d_foff, d_cell0, d_lipc;
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
  inject_kernel<<<blocks, 256, 0, s>>>(b->atoms.as<AtomTab>(), b->natom, b->celld.as<double>(),
                                       b->hcell.as<double>(), b->coef.as<double>(), b->N, b->lmax,
                                       lmin, b->nlip, b->first, xs, nx, ys, ny, zs, nz, factor,
                                       d_cube);
  DAGE_CUDA_TRY(cudaGetLastError());
  return 0;
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
  DevBuf staging;
  double *d_cube = cube;
  if (!(flags & DAGE_DEVICE_PTRS)) {
    DAGE_TRY(staging.alloc(sizeof(double) * n));
    DAGE_CUDA_TRY(cudaMemcpy(staging.ptr, cube, sizeof(double) * n, cudaMemcpyHostToDevice));
    d_cube = staging.as<double>();
  }
  const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)sm_count() * 16);
  inject_kernel<<<blocks, 256>>>(b->atoms.as<AtomTab>(), b->natom, b->celld.as<double>(),
                                 b->hcell.as<double>(), b->coef.as<double>(), b->N, b->lmax, lmin,
                                 b->nlip, b->first, b->xs.as<double>(), ax[0].n(),
                                 b->ys.as<double>(), ax[1].n(), b->zs.as<double>(), ax[2].n(),
                                 factor, d_cube);
  DAGE_CUDA_TRY(cudaGetLastError());
  if (!(flags & DAGE_DEVICE_PTRS))
    DAGE_CUDA_TRY(cudaMemcpy(cube, d_cube, sizeof(double) * n, cudaMemcpyDeviceToHost));
  DAGE_CUDA_TRY(cudaDeviceSynchronize());
  return 0;
}

int dage_bubbles_destroy(dage_bubbles *b) {
  if (!b) return 0;
  for (DevBuf *x : {&b->atoms, &b->celld, &b->hcell, &b->coef, &b->xs, &b->ys, &b->zs}) x->release();
  delete b;
  return 0;
}

}  // extern "C"
