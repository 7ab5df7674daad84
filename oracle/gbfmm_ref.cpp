// gbfmm_ref.cpp -- CPU FP64 oracle for the GBFMM pieces of the path: real
// regular solid harmonics, the M2L interaction matrix, the M2M/L2L
// translation matrix, the octree box geometry, box multipole moments and
// local-expansion evaluation.
//
// TEST INFRASTRUCTURE ONLY (see dage_oracle.h).  Each routine restates the
// reference routine cited beside it.
#include <cmath>
#include <cstring>
#include <vector>

#include "dage_oracle.h"

namespace {

// lm index of (l, m): l(l+1)+m, 0-based (harmonics.F90:1649-1654 is the
// 1-based l(l+1)+m+1).
inline int lm_map(int l, int m) { return l * (l + 1) + m; }
inline void lm_of(int s, int &l, int &m) {  // inverse, 0-based s
  l = (int)std::floor(std::sqrt((double)s) + 1e-12);
  while ((l + 1) * (l + 1) <= s) ++l;
  while (l * l > s) --l;
  m = s - l * l - l;
}
inline double sgn(int k) { return (k & 1) ? -1.0 : 1.0; }  // (-1)**k
inline int delta(int i, int j) { return i == j ? 1 : 0; }

double fact_prod(int n) {  // product([(1.0d0*i, i=1,n)])
  double p = 1.0;
  for (int i = 1; i <= n; ++i) p = p * (1.0 * i);
  return p;
}

// multipole.F90:485-560 Cc, Cs, Cst, Cct, D
double Cc(int l, int m) {
  if (m == 0) return 1.0 / fact_prod(l);
  if (m > 0) return sgn(m) / std::sqrt(2.0 * fact_prod(l - m) * fact_prod(l + m));
  return sgn(m) * Cc(l, -m);
}
double Cs(int l, int m) {
  if (m == 0) return 0.0;
  if (m > 0) return sgn(m) / std::sqrt(2.0 * fact_prod(l - m) * fact_prod(l + m));
  return -sgn(m) * Cs(l, -m);
}
double Cst(int l, int m) { return fact_prod(l - m) * fact_prod(l + m) * Cs(l, m); }
double Cct(int l, int m) { return fact_prod(l - m) * fact_prod(l + m) * Cc(l, m); }
double Dlm(int l, int m) {
  double d = fact_prod(l + m) * fact_prod(l - m) * (2.0 - delta(m, 0));
  return std::sqrt(d);
}

struct Coeffs {
  int lmax = -1;
  std::vector<int> larr1, marr1, larr2, marr2;
  std::vector<double> c1, c2;
};

// InteractionMatrix_compute_coeffs (multipole.F90:106-187)
void interaction_coeffs(int lmax, Coeffs &C) {
  const int N = (lmax + 1) * (lmax + 1);
  const int M = N * (N + 1) / 2;
  C.lmax = lmax;
  C.larr1.assign(M, -1);
  C.larr2.assign(M, -1);
  C.marr1.assign(M, 0);
  C.marr2.assign(M, 0);
  C.c1.assign(M, 0.0);
  C.c2.assign(M, 0.0);
  const double ij[3] = {1.0, 0.5, 0.25};
  for (int s = 1; s <= N; ++s) {
    int j, k, l, m;
    lm_of(s - 1, j, k);
    for (int i = s; i <= N; ++i) {
      lm_of(i - 1, l, m);
      const double c = 2 * sgn(j) * ij[delta(m, 0) + delta(k, 0)];
      const int r = i + (2 * N - s) * (s - 1) / 2 - 1;
      double a = 0, b = 0;
      if (m >= 0 && k >= 0) {
        C.larr1[r] = l + j; C.marr1[r] = std::abs(m + k); a = Cct(l + j, m + k);
        C.larr2[r] = l + j; C.marr2[r] = std::abs(m - k); b = sgn(k) * Cct(l + j, m - k);
      } else if (m >= 0 && k < 0) {
        C.larr1[r] = l + j; C.marr1[r] = -std::abs(m + k); a = Cst(l + j, m + k);
        C.larr2[r] = l + j; C.marr2[r] = -std::abs(m - k); b = -sgn(k) * Cst(l + j, m - k);
        a = -a * sgn(k); b = -b * sgn(k);
      } else if (m < 0 && k >= 0) {
        C.larr1[r] = l + j; C.marr1[r] = -std::abs(m + k); a = Cst(l + j, m + k);
        C.larr2[r] = l + j; C.marr2[r] = -std::abs(m - k); b = sgn(k) * Cst(l + j, m - k);
        a = -a * sgn(m); b = -b * sgn(m);
      } else {
        C.larr1[r] = l + j; C.marr1[r] = std::abs(m + k); a = -Cct(l + j, m + k);
        C.larr2[r] = l + j; C.marr2[r] = std::abs(m - k); b = sgn(k) * Cct(l + j, m - k);
        a = a * sgn(m + k); b = b * sgn(m + k);
      }
      a = a * c; b = b * c;
      a = sgn(m) * a / Dlm(l, m); b = sgn(m) * b / Dlm(l, m);
      a = sgn(k) * a / Dlm(j, k); b = sgn(k) * b / Dlm(j, k);
      C.c1[r] = a;
      C.c2[r] = b;
    }
  }
}

// TranslationMatrix_compute_coeffs (multipole.F90:372-440)
void translation_coeffs(int lmax, Coeffs &C) {
  const int N = (lmax + 1) * (lmax + 1);
  const int M = N * (N + 1) / 2;
  C.lmax = lmax;
  C.larr1.assign(M, -1);
  C.larr2.assign(M, -1);
  C.marr1.assign(M, 0);
  C.marr2.assign(M, 0);
  C.c1.assign(M, 0.0);
  C.c2.assign(M, 0.0);
  const double ij[2] = {1.0, 0.5};
  for (int s = 1; s <= N; ++s) {
    int j, k, l, m;
    lm_of(s - 1, j, k);
    for (int i = s; i <= N; ++i) {
      lm_of(i - 1, l, m);
      const int r = i + (2 * N - s) * (s - 1) / 2 - 1;
      const int L = l - j;
      auto in = [&](int v) { return -L <= v && v <= L; };
      if (m >= 0 && k >= 0) {
        if (in(std::abs(m - k))) { C.larr1[r] = L; C.marr1[r] = std::abs(m - k); C.c1[r] = Cc(L, m - k) * ij[delta(0, k)]; }
        if (in(std::abs(m + k))) { C.larr2[r] = L; C.marr2[r] = std::abs(m + k); C.c2[r] = sgn(k) * Cc(L, m + k) * ij[delta(0, k)]; }
      } else if (m >= 0 && k < 0) {
        if (in(-std::abs(m - k))) { C.larr1[r] = L; C.marr1[r] = -std::abs(m - k); C.c1[r] = Cs(L, m - k) * sgn(k); }
        if (in(-std::abs(m + k))) { C.larr2[r] = L; C.marr2[r] = -std::abs(m + k); C.c2[r] = -Cs(L, m + k); }
      } else if (m < 0 && k >= 0) {
        if (in(-std::abs(m - k))) { C.larr1[r] = L; C.marr1[r] = -std::abs(m - k); C.c1[r] = -Cs(L, m - k) * sgn(m) * ij[delta(0, k)]; }
        if (in(-std::abs(m + k))) { C.larr2[r] = L; C.marr2[r] = -std::abs(m + k); C.c2[r] = -Cs(L, m + k) * ij[delta(0, k)] * sgn(m + k); }
      } else {
        if (in(std::abs(m - k))) { C.larr1[r] = L; C.marr1[r] = std::abs(m - k); C.c1[r] = Cc(L, m - k) * sgn(m - k); }
        if (in(std::abs(m + k))) { C.larr2[r] = L; C.marr2[r] = std::abs(m + k); C.c2[r] = -Cc(L, m + k) * sgn(m); }
      }
      const double f = Dlm(l, m) * sgn(m - k) / Dlm(j, k);
      C.c1[r] = C.c1[r] * f;
      C.c2[r] = C.c2[r] * f;
    }
  }
}

}  // namespace

extern "C" {

void orc_solid_harmonics(int lmax, double x, double y, double z, double *S) {
  // Racah-normalised real regular solid harmonics by the recursion of
  // harmonics.F90:586-658 (Helgaker, Jorgensen & Olsen).
  const double r2 = x * x + y * y + z * z;
  S[0] = 1.0;
  if (lmax < 1) return;
  S[lm_map(1, -1)] = y;
  S[lm_map(1, 0)] = z;
  S[lm_map(1, 1)] = x;
  for (int l = 2; l <= lmax; ++l) {
    const double top = S[lm_map(l - 1, l - 1)], bot = S[lm_map(l - 1, -(l - 1))];
    const double f = std::sqrt((2 * l - 1.0) / (2.0 * l));
    S[lm_map(l, -l)] = f * (y * top + x * bot);
    for (int m = -(l - 1); m <= l - 1; ++m) {
      double v = (2 * l - 1.0) / std::sqrt(1.0 * (l + m) * (l - m)) * (z * S[lm_map(l - 1, m)]);
      if (l - std::abs(m) > 1)
        v = v - std::sqrt((l + m - 1.0) * (l - m - 1.0) / ((l + m) * (l - m))) * (r2 * S[lm_map(l - 2, m)]);
      S[lm_map(l, m)] = v;
    }
    S[lm_map(l, l)] = f * (x * top - y * bot);
  }
}

int orc_interaction_matrix(int lmax, const double *d, double *T) {
  // InteractionMatrix_eval_pick (multipole.F90:265-303): T(N x N),
  // column-major; far_pot(:, i) += T(c_j - c_i) q(:, j).
  static thread_local Coeffs C;
  if (C.lmax != lmax) interaction_coeffs(lmax, C);
  const int N = (lmax + 1) * (lmax + 1);
  const int L2 = 2 * lmax;
  std::vector<double> I((L2 + 1) * (L2 + 1));
  orc_solid_harmonics(L2, d[0], d[1], d[2], I.data());
  const double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  if (r == 0.0) return -1;
  for (int l = 0; l <= L2; ++l) {
    double rp = 1.0;
    for (int e = 0; e < 2 * l + 1; ++e) rp *= r;
    for (int m = -l; m <= l; ++m) I[lm_map(l, m)] = I[lm_map(l, m)] / rp;
  }
  for (int s = 1; s <= N; ++s) {
    int j, k;
    lm_of(s - 1, j, k);
    for (int i = s; i <= N; ++i) {
      int l, m;
      lm_of(i - 1, l, m);
      const int r0 = i + (2 * N - s) * (s - 1) / 2 - 1;
      double w = C.c1[r0] * I[lm_map(C.larr1[r0], C.marr1[r0])];
      w = w + C.c2[r0] * I[lm_map(C.larr2[r0], C.marr2[r0])];
      T[(size_t)(s - 1) * N + (i - 1)] = w;
      T[(size_t)(i - 1) * N + (s - 1)] = sgn(l - j) * w;
    }
  }
  return 0;
}

int orc_translation_matrix(int lmax, const double *d, double *W) {
  // TranslationMatrix_eval (multipole.F90:443-476): packed lower triangle.
  static thread_local Coeffs C;
  if (C.lmax != lmax) translation_coeffs(lmax, C);
  const int N = (lmax + 1) * (lmax + 1);
  const int M = N * (N + 1) / 2;
  std::vector<double> S(N);
  orc_solid_harmonics(lmax, d[0], d[1], d[2], S.data());
  for (int r = 0; r < M; ++r) {
    double w = 0.0;
    if (C.larr1[r] != -1) w = C.c1[r] * S[lm_map(C.larr1[r], C.marr1[r])];
    if (C.larr2[r] != -1) w = w + C.c2[r] * S[lm_map(C.larr2[r], C.marr2[r])];
    W[r] = w;
  }
  return 0;
}

void orc_dtpmv_lower_unit(int n, const double *A, double *x) {
  // x := A x, A lower triangular (packed by columns) with unit diagonal
  // (BLAS dtpmv('L', 'N', 'U'), as TranslationMatrix_apply uses it).
  for (int j = n - 1; j >= 0; --j) {
    const double t = x[j];
    const size_t col = (size_t)j * n - (size_t)j * (j - 1) / 2;  // start of column j
    for (int i = j + 1; i < n; ++i) x[i] += t * A[col + (i - j)];
  }
}

void orc_box_vector(int ibox, int level, int *v) {
  // GBFMMParallelInfo_get_box_vector (gbfmm_parallel_info.F90:1128-1165):
  // recursive row-major index within each parent (2x2x2 splits).
  int vv[3] = {0, 0, 0};
  int rem;
  if (level > 1) {
    const int parent = (ibox - 1) / 8 + 1;
    orc_box_vector(parent, level - 1, vv);
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

int orc_box_index(const int *v, int level) {
  // GBFMMParallelInfo_get_box_index (gbfmm_parallel_info.F90:1168-1194)
  int idx, rem[3];
  if (level > 1) {
    int pv[3] = {v[0] / 2, v[1] / 2, v[2] / 2};
    idx = (orc_box_index(pv, level - 1) - 1) * 8 + 1;
    for (int d = 0; d < 3; ++d) rem[d] = v[d] - pv[d] * 2;
  } else {
    idx = 1;
    for (int d = 0; d < 3; ++d) rem[d] = v[d];
  }
  return idx + rem[0] + rem[1] * 2 + rem[2] * 4;
}

int orc_nearest_neighbors(int ibox, int level, int *out) {
  // gbfmm_parallel_info.F90:983-1017: the up-to-26 boxes sharing a face,
  // edge or corner, z outermost, x innermost.
  const int lim = 1 << level;
  int v[3];
  orc_box_vector(ibox, level, v);
  int n = 0;
  for (int iz = -1; iz <= 1; ++iz)
    for (int iy = -1; iy <= 1; ++iy)
      for (int ix = -1; ix <= 1; ++ix) {
        if (!ix && !iy && !iz) continue;
        const int w[3] = {v[0] + ix, v[1] + iy, v[2] + iz};
        if (w[0] < 0 || w[1] < 0 || w[2] < 0 || w[0] >= lim || w[1] >= lim || w[2] >= lim) continue;
        out[n++] = orc_box_index(w, level);
      }
  return n;
}

int orc_local_farfield(int ibox, int level, int *out) {
  // gbfmm_parallel_info.F90:827-981, evaluation type 0: the children of
  // the parent's nearest neighbours that are not nearest neighbours of ibox.
  int pnn[26], nn[26];
  const int parent = (ibox - 1) / 8 + 1;
  const int np = level > 1 ? orc_nearest_neighbors(parent, level - 1, pnn) : 0;
  const int nnn = orc_nearest_neighbors(ibox, level, nn);
  int n = 0;
  for (int a = 0; a < np; ++a)
    for (int c = 1; c <= 8; ++c) {
      const int child = (pnn[a] - 1) * 8 + c;
      bool near = false;
      for (int b = 0; b < nnn; ++b) near = near || nn[b] == child;
      if (!near) out[n++] = child;
    }
  return n;
}

int orc_box_multipoles(int lmax, int nx, const double *px, const double *wx, int ny,
                       const double *py, const double *wy, int nz, const double *pz,
                       const double *wz, const double *cube, const double *center, double *q) {
  // q_lm = sum_points cube * wx * wy * wz * S_lm(r - center): the moments
  // the reference's GPU evaluator accumulates (integrator.cu:1112-1160).
  const int N = (lmax + 1) * (lmax + 1);
  std::vector<double> acc(N, 0.0), S(N);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const double v = cube[(size_t)nx * ny * k + (size_t)nx * j + i] * wx[i] * wy[j] * wz[k];
        orc_solid_harmonics(lmax, px[i] - center[0], py[j] - center[1], pz[k] - center[2], S.data());
        for (int s = 0; s < N; ++s) acc[s] += v * S[s];
      }
  std::memcpy(q, acc.data(), sizeof(double) * N);
  return 0;
}

int orc_l2p(int lmax, const double *L, const double *center, int nx, const double *px, int ny,
            const double *py, int nz, const double *pz, double *out) {
  // out(x,y,z) += sum_lm L_lm S_lm(r - center) (gbfmm_coulomb3d.F90:1701-1744)
  const int N = (lmax + 1) * (lmax + 1);
  std::vector<double> S(N);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        orc_solid_harmonics(lmax, px[i] - center[0], py[j] - center[1], pz[k] - center[2], S.data());
        double v = 0.0;
        for (int s = 0; s < N; ++s) v += L[s] * S[s];
        out[(size_t)nx * ny * k + (size_t)nx * j + i] += v;
      }
  return 0;
}

}  // extern "C"
