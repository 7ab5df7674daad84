// helmholtz_ref.cpp -- CPU oracle for the GBFMM Helmholtz (Yukawa) far field:
// modified spherical Bessel functions, Helmholtz box multipoles, the
// multipole-to-local conversion (rotation to the translation axis, coaxial
// translation, rotation back) and local-expansion evaluation.
//
// TEST INFRASTRUCTURE ONLY (see dage_oracle.h).  Each routine restates the
// reference routine cited beside it.  The one deliberate difference: the
// rotation of real spherical-harmonic expansions is computed from its
// defining property (the rotated expansion represents the same function in
// a frame whose z axis is the translation direction) by least squares on the
// solid harmonics, where the reference uses the recursions of Blanco, Florez
// & Bermejo (J. Mol. Struct. Theochem 419 (1997) 19) in
// helmholtz_multipole_tools.F90:919-1200; both are the exact rotation.
#include <cmath>
#include <cstring>
#include <vector>

#include "dage_oracle.h"

namespace {

inline int lm_map(int l, int m) { return l * (l + 1) + m; }
typedef long double ext;  // the reference evaluates the Bessel functions in REAL128

// helmholtz3d.F90:935-971 FirstModSphBesselCollection_evaluate_small:
// i_n(z) = z^n / (2n+1)!! * sum_k (z^2/2)^k / (k! (2n+3)(2n+5)...(2n+2k+1))
ext bessel_i_series(ext z, int n) {
  ext prefactor = std::pow(z, (ext)n);
  ext divider = 1.0L;
  for (int i = 1; i <= 2 * n + 1; i += 2) divider *= i;
  prefactor /= divider;
  ext addition = 1.0L, reslt = 1.0L, b = 1.0L, fact = 1.0L;
  ext div = 1.0L;
  const ext a = 0.5L * z * z;
  for (int i = 1; addition > 1e-15L * reslt && i < 300; ++i) {
    b *= a;
    fact *= i;
    div *= (2 * n + 2 * i + 1);
    addition = b / (fact * div);
    reslt += addition;
  }
  return prefactor * reslt;
}

}  // namespace

extern "C" {

// helmholtz3d.F90:879-933 FirstModSphBesselCollection_evaluate: series for
// lmax and lmax-1, downward recursion i_l = (2l+3)/x i_{l+1} + i_{l+2}.
void orc_bessel_i(double x, int lmax, double *out) {
  std::vector<ext> r(lmax + 3, 0.0L);
  const ext X = x;
  if (std::fabs(x) < 2.220446049250313e-16) {
    for (int l = 0; l <= lmax; ++l) out[l] = l == 0 ? 1.0 : 0.0;
    return;
  }
  r[lmax] = bessel_i_series(X, lmax);
  if (lmax >= 1) r[lmax - 1] = bessel_i_series(X, lmax - 1);
  for (int l = lmax - 2; l >= 0; --l) r[l] = (2 * l + 3) * r[l + 1] / X + r[l + 2];
  for (int l = 0; l <= lmax; ++l) out[l] = (double)r[l];
}

// helmholtz3d.F90:1133-1174 SecondModSphBesselCollection_evaluate:
// k_0 = (pi/2) e^-x / x, k_1 = (pi/2) e^-x (x+1) / x^2, upward recursion
// k_l = (2l-1)/x k_{l-1} + k_{l-2}.
void orc_bessel_k(double x, int lmax, double *out) {
  const ext X = x, pi = 3.14159265358979323846264338327950288L;
  std::vector<ext> r(lmax + 2, 0.0L);
  r[0] = std::exp(-X) / X * pi / 2;
  if (lmax >= 1) r[1] = std::exp(-X) * (X + 1) / (X * X) * pi / 2;
  for (int l = 2; l <= lmax; ++l) r[l] = (2 * l - 1) * r[l - 1] / X + r[l - 2];
  for (int l = 0; l <= lmax; ++l) out[l] = (double)r[l];
}

// helmholtz_multipole_tools.F90:428-511 get_all_aligned_ml_translation_
// coefficients (coaxial multipole-to-local translation along +z, conventional
// normalisation), bessel values k_0 .. k_{lin+1}(kappa d).  out[(l * (lin+1)
// + n) * (lmax+1) + m] = C(l, n, m), l, m <= lmax, n <= lin.  As in the
// reference, the recurrence only has entries up to l = lin + 1 (entries it
// never fills stay zero).
void orc_aligned_ml(const double *bessel, int lmax, int lin, double *out) {
  const int E = lin + 1;  // indices -1 .. lin+1 -> offset 1
  const int D = E + 2;
  std::vector<double> C((size_t)D * D * D, 0.0);
  auto c = [&](int l, int n, int m) -> double & {
    return C[((size_t)(l + 1) * D + (n + 1)) * D + (m + 1)];
  };
  // a_coefficient / b_coefficient (:591-607); the reference tabulates them
  // from n = 0, so n = -1 reads zero
  auto A = [](int n, int m) {
    if (n < 0) return 0.0;
    const int am = std::abs(m);
    return std::sqrt((double)((n + 1 + am) * (n + 1 - am)) / ((2 * n + 1) * (2 * n + 3)));
  };
  auto B = [](int n, int m) {
    if (n < 0) return 0.0;
    double b = std::sqrt((double)((n - m - 1) * (n - m)) / ((2 * n - 1) * (2 * n + 1)));
    if (std::abs(m) > n) return 0.0;
    if (m < 0) b = -b;
    return b;
  };
  c(0, 0, 0) = bessel[0];
  for (int n = 1; n <= lin + 1; ++n) {
    c(n, 0, 0) = ((n & 1) ? -1.0 : 1.0) * std::sqrt(2.0 * n + 1) * bessel[n];
    c(0, n, 0) = std::sqrt(2.0 * n + 1) * bessel[n];
  }
  for (int n = 1; n <= lin; ++n) {
    c(1, n, 0) = (-A(n, 0) * c(0, n + 1, 0) - A(n - 1, 0) * c(0, n - 1, 0)) / A(0, 0);
    c(n, 1, 0) = (((1 + n) & 1) ? -1.0 : 1.0) * c(1, n, 0);
  }
  for (int m = 0; m <= lin; ++m) {
    for (int n = m; n <= lin; ++n)
      for (int l = m; l <= lin; ++l)
        c(l, n + 1, m) = (-A(l, m) * c(l + 1, n, m) - A(l - 1, m) * c(l - 1, n, m) -
                          A(n - 1, m) * c(l, n - 1, m)) /
                         A(n, m);
    for (int l = m; l <= lin; ++l)
      c(l, m + 1, m + 1) = (-B(l, -m - 1) * c(l - 1, m, m) - B(l + 1, m) * c(l + 1, m, m)) /
                           B(m + 1, -m - 1);
  }
  for (int l = 0; l <= lmax; ++l)
    for (int n = 0; n <= lin; ++n)
      for (int m = 0; m <= lmax; ++m) {
        const bool in = l <= lin + 1 && m <= lin + 1;
        out[((size_t)l * (lin + 1) + n) * (lmax + 1) + m] = in ? c(l, n, m) : 0.0;
      }
}

// Rotation of real spherical-harmonic expansions (Racah or orthonormal: the
// same per-l matrices) to the frame whose z axis is dhat: R_l[m' + l][m + l]
// with f'_(l m') = sum_m R_l[m'][m] f_(l m).  Built from its defining
// property S_lm(Q^T r') = sum_m' R_l[m'][m] S_lm'(r') by least squares over
// 4(2l+1) points; out holds the blocks l = 0..lmax one after the other.
void orc_rotation(const double *dhat, int lmax, double *out) {
  // Q: rows are the new axes (x', y', z' = dhat) in old coordinates
  double z[3] = {dhat[0], dhat[1], dhat[2]};
  const double nz = std::sqrt(z[0] * z[0] + z[1] * z[1] + z[2] * z[2]);
  for (double &v : z) v /= nz;
  double t[3] = {1.0, 0.0, 0.0};
  if (std::fabs(z[0]) > 0.9) t[0] = 0.0, t[1] = 1.0;
  double x[3] = {t[1] * z[2] - t[2] * z[1], t[2] * z[0] - t[0] * z[2], t[0] * z[1] - t[1] * z[0]};
  const double nx = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  for (double &v : x) v /= nx;
  const double y[3] = {z[1] * x[2] - z[2] * x[1], z[2] * x[0] - z[0] * x[2], z[0] * x[1] - z[1] * x[0]};
  const int N = (lmax + 1) * (lmax + 1);
  size_t off = 0;
  for (int l = 0; l <= lmax; ++l) {
    const int w = 2 * l + 1, npt = 4 * w;
    std::vector<double> Bm((size_t)npt * w), Gm((size_t)npt * w), S(N);
    for (int k = 0; k < npt; ++k) {
      // deterministic points spread over the sphere (golden spiral)
      const double u = 1.0 - 2.0 * (k + 0.5) / npt, ph = 2.399963229728653 * k;
      const double s = std::sqrt(1.0 - u * u);
      const double rp[3] = {s * std::cos(ph), s * std::sin(ph), u};  // new frame
      orc_solid_harmonics(l, rp[0], rp[1], rp[2], S.data());
      for (int mp = -l; mp <= l; ++mp) Bm[(size_t)k * w + mp + l] = S[lm_map(l, mp)];
      // the same point in old coordinates: Q^T r'
      const double ro[3] = {x[0] * rp[0] + y[0] * rp[1] + z[0] * rp[2],
                            x[1] * rp[0] + y[1] * rp[1] + z[1] * rp[2],
                            x[2] * rp[0] + y[2] * rp[1] + z[2] * rp[2]};
      orc_solid_harmonics(l, ro[0], ro[1], ro[2], S.data());
      for (int m = -l; m <= l; ++m) Gm[(size_t)k * w + m + l] = S[lm_map(l, m)];
    }
    // normal equations (B^T B) R = B^T G, Gauss-Jordan with partial pivoting
    std::vector<double> M((size_t)w * (2 * w), 0.0);
    for (int i = 0; i < w; ++i)
      for (int j = 0; j < w; ++j) {
        double a = 0.0, g = 0.0;
        for (int k = 0; k < npt; ++k) {
          a += Bm[(size_t)k * w + i] * Bm[(size_t)k * w + j];
          g += Bm[(size_t)k * w + i] * Gm[(size_t)k * w + j];
        }
        M[(size_t)i * 2 * w + j] = a;
        M[(size_t)i * 2 * w + w + j] = g;
      }
    for (int c = 0; c < w; ++c) {
      int p = c;
      for (int r = c + 1; r < w; ++r)
        if (std::fabs(M[(size_t)r * 2 * w + c]) > std::fabs(M[(size_t)p * 2 * w + c])) p = r;
      for (int j = 0; j < 2 * w; ++j) std::swap(M[(size_t)c * 2 * w + j], M[(size_t)p * 2 * w + j]);
      const double d = M[(size_t)c * 2 * w + c];
      for (int j = 0; j < 2 * w; ++j) M[(size_t)c * 2 * w + j] /= d;
      for (int r = 0; r < w; ++r)
        if (r != c) {
          const double f = M[(size_t)r * 2 * w + c];
          for (int j = 0; j < 2 * w; ++j) M[(size_t)r * 2 * w + j] -= f * M[(size_t)c * 2 * w + j];
        }
    }
    for (int i = 0; i < w; ++i)
      for (int j = 0; j < w; ++j) out[off + (size_t)i * w + j] = M[(size_t)i * 2 * w + w + j];
    off += (size_t)w * w;
  }
}

// helmholtz_multipole_tools.F90:172-278 HelmholtzExpansionTranslator_
// translate_real with the HelmholtzMultipoleConverter (:385-426): Racah ->
// orthonormal scaling, rotation to the axis destination - source, coaxial
// translation (real basis: C(l, n, |m|) acting on (n, m) for both signs of m,
// :280-331 with :760-800), rotation back, orthonormal -> Racah scaling.
int orc_helm_m2l(int lmax, int lin, double kappa, const double *M, const double *src,
                 const double *dst, double *L) {
  const double pi = 3.14159265358979323846;
  const double d[3] = {dst[0] - src[0], dst[1] - src[1], dst[2] - src[2]};
  const double dist = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  if (dist == 0.0) return -1;
  const int Lr = lmax > lin ? lmax : lin;
  const int Nin = (lin + 1) * (lin + 1), Nout = (lmax + 1) * (lmax + 1);
  std::vector<double> R(0);
  {
    size_t tot = 0;
    for (int l = 0; l <= Lr; ++l) tot += (size_t)(2 * l + 1) * (2 * l + 1);
    R.resize(tot);
  }
  orc_rotation(d, Lr, R.data());
  std::vector<size_t> roff(Lr + 2, 0);
  for (int l = 0; l <= Lr; ++l) roff[l + 1] = roff[l] + (size_t)(2 * l + 1) * (2 * l + 1);
  // scale and rotate the input
  std::vector<double> a(Nin, 0.0);
  for (int l = 0; l <= lin; ++l) {
    const int w = 2 * l + 1;
    const double sc = std::sqrt((2 * l + 1) / (4 * pi));
    for (int mp = -l; mp <= l; ++mp) {
      double s = 0.0;
      for (int m = -l; m <= l; ++m) s += R[roff[l] + (size_t)(mp + l) * w + (m + l)] * M[lm_map(l, m)];
      a[lm_map(l, mp)] = sc * s;
    }
  }
  // coaxial translation
  std::vector<double> bess(lin + 2);
  orc_bessel_k(kappa * dist, lin + 1, bess.data());
  std::vector<double> C((size_t)(lmax + 1) * (lin + 1) * (lmax + 1));
  orc_aligned_ml(bess.data(), lmax, lin, C.data());
  std::vector<double> b(Nout, 0.0);
  for (int l = 0; l <= lmax; ++l)
    for (int m = -l; m <= l; ++m) {
      const int am = std::abs(m);
      double s = 0.0;
      for (int n = am; n <= lin; ++n)
        s += C[((size_t)l * (lin + 1) + n) * (lmax + 1) + am] * a[lm_map(n, m)];
      b[lm_map(l, m)] = s;
    }
  // rotate back (R is orthogonal) and rescale
  for (int l = 0; l <= lmax; ++l) {
    const int w = 2 * l + 1;
    const double sc = std::sqrt(4 * pi / (2 * l + 1));
    for (int m = -l; m <= l; ++m) {
      double s = 0.0;
      for (int mp = -l; mp <= l; ++mp) s += R[roff[l] + (size_t)(mp + l) * w + (m + l)] * b[lm_map(l, mp)];
      L[lm_map(l, m)] = sc * s;
    }
  }
  return 0;
}

// gbfmm_helmholtz3d.F90:1491-1577: q_lm(box) = sum rho w i_l(kappa r) Y_lm(rhat)
// (Racah Y_lm = S_lm / r^l) over the box's points, centre c.
int orc_helm_box_multipoles(int lmax, double kappa, int nx, const double *px, const double *wx,
                            int ny, const double *py, const double *wy, int nz, const double *pz,
                            const double *wz, const double *rho, const double *center, double *q) {
  const int N = (lmax + 1) * (lmax + 1);
  std::vector<double> acc(N, 0.0), S(N), bi(lmax + 1);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const double x = px[i] - center[0], y = py[j] - center[1], z = pz[k] - center[2];
        const double r = std::sqrt(x * x + y * y + z * z);
        const double v = rho[i + (size_t)nx * (j + (size_t)ny * k)] * wx[i] * wy[j] * wz[k];
        orc_bessel_i(kappa * r, lmax, bi.data());
        orc_solid_harmonics(lmax, x, y, z, S.data());
        for (int l = 0; l <= lmax; ++l) {
          const double rl = r > 0.0 ? std::pow(r, l) : (l == 0 ? 1.0 : 0.0);
          for (int m = -l; m <= l; ++m) {
            const double Y = l == 0 ? 1.0 : (r > 0.0 ? S[lm_map(l, m)] / rl : 0.0);
            acc[lm_map(l, m)] += v * bi[l] * Y;
          }
        }
      }
  std::memcpy(q, acc.data(), sizeof(double) * N);
  return 0;
}

// gbfmm_helmholtz3d.F90:1019-1105: V(r) += 8 kappa sum_lm (2l+1)/(4 pi)
// i_l(kappa |r - c|) Y_lm L_lm over a box's points.
int orc_helm_l2p(int lmax, double kappa, const double *L, const double *center, int nx,
                 const double *px, int ny, const double *py, int nz, const double *pz, double *V) {
  const double pi = 3.14159265358979323846;
  const int N = (lmax + 1) * (lmax + 1);
  std::vector<double> S(N), bi(lmax + 1);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const double x = px[i] - center[0], y = py[j] - center[1], z = pz[k] - center[2];
        const double r = std::sqrt(x * x + y * y + z * z);
        orc_bessel_i(kappa * r, lmax, bi.data());
        orc_solid_harmonics(lmax, x, y, z, S.data());
        double v = 0.0;
        for (int l = 0; l <= lmax; ++l) {
          const double rl = r > 0.0 ? std::pow(r, l) : (l == 0 ? 1.0 : 0.0);
          double s = 0.0;
          for (int m = -l; m <= l; ++m) {
            const double Y = l == 0 ? 1.0 : (r > 0.0 ? S[lm_map(l, m)] / rl : 0.0);
            s += Y * L[lm_map(l, m)];
          }
          v += (2 * l + 1) / (4 * pi) * bi[l] * s;
        }
        V[i + (size_t)nx * (j + (size_t)ny * k)] += 8.0 * kappa * v;
      }
  return 0;
}

}  // extern "C"
