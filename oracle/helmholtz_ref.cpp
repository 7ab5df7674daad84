// helmholtz_ref.cpp -- CPU oracle for the GBFMM Helmholtz (Yukawa) far field:
// modified spherical Bessel functions, Helmholtz box multipoles, the
// multipole-to-local conversion (rotation to the translation axis, coaxial
// translation, rotation back) and local-expansion evaluation.
//
// TEST INFRASTRUCTURE ONLY (see dage_oracle.h).  Each routine restates the
// reference routine cited beside it.  The rotation of real
// spherical-harmonic expansions follows the reference's recursions of
// Blanco, Florez & Bermejo (J. Mol. Struct. Theochem 419 (1997) 19),
// helmholtz_multipole_tools.F90:911-1200, with the reference's Euler angles
// (:695-701) and its forward/backward rotation (:240-256).  orc_rotation, a
// rotation computed instead from its defining property by least squares on
// the solid harmonics, is kept as an independent check of that restatement.
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

// helmholtz_multipole_tools.F90:1003-1200 get_rotation_coefficient_matrices:
// the small-d matrices d^l_{m' m}(beta) by the recursions of Blanco, Florez &
// Bermejo, stored as the reference's array reslt(-lmax:lmax, 0:lmax, 0:lmax)
// indexed (m', m, l), m >= 0.
struct DMat {
  int L;
  std::vector<double> v;
  explicit DMat(int lmax) : L(lmax), v((size_t)(2 * lmax + 1) * (lmax + 1) * (lmax + 1), 0.0) {}
  double &operator()(int mp, int m, int l) {
    return v[((size_t)l * (L + 1) + m) * (2 * L + 1) + (mp + L)];
  }
};

double fact_int(int x) {  // the reference's factorial: integer(16) product
  unsigned __int128 r = 1;
  for (int i = 1; i <= x; ++i) r *= (unsigned __int128)i;
  return (double)r;
}

double ipow(double b, int e) {  // Fortran x**n for integer n
  double r = 1.0;
  for (int i = 0; i < e; ++i) r *= b;
  return r;
}

// Explicit Wigner sum for one small-d entry in the reference's convention
// R(m', m, l), in extended precision (used by the repaired recursion only).
double wigner_d(int l, int m, int mp, double beta) {
  // R(m', m, l) = d^l_{m m'}(beta) with d^j_{a b} = sum_s (-1)^(a - b + s)
  //   sqrt((j+a)!(j-a)!(j+b)!(j-b)!) / ((j+b-s)! s! (a-b+s)! (j-a-s)!)
  //   cos(beta/2)^(2j+b-a-2s) sin(beta/2)^(a-b+2s)
  const int a = m, b = mp;
  const long double c = cosl(0.5L * beta), s = sinl(0.5L * beta);
  auto f = [](int n) {
    long double r = 1.0L;
    for (int i = 2; i <= n; ++i) r *= i;
    return r;
  };
  long double sum = 0.0L;
  for (int k = 0; k <= 2 * l; ++k) {
    if (l + b - k < 0 || a - b + k < 0 || l - a - k < 0) continue;
    const long double den = f(l + b - k) * f(k) * f(a - b + k) * f(l - a - k);
    const long double term = powl(c, 2 * l + b - a - 2 * k) * powl(s, a - b + 2 * k) / den;
    sum += ((a - b + k) % 2 ? -1.0L : 1.0L) * term;
  }
  return (double)(sqrtl(f(l + a) * f(l - a) * f(l + b) * f(l - b)) * sum);
}

// repaired = false: the reference as written.  repaired = true: its two
// defects corrected -- the single-precision literal sqrt(2.0) (:1018; every
// rotation then carries ~3e-8 relative error) becomes a double, and the rows
// m = l - 1 of eq. 68 (:1119-1131), whose step divides by l cos(beta) - m'
// and hits 0/0 where l cos(beta) is an integer (e.g. the lattice direction
// (2, 1, 2) at l = 3, 6, 9, ...; the reference's epsilon guard then zeroes the
// rest of the row), are taken from the explicit Wigner sum (wigner_d).
void ref_rotation_dmatrices(double beta, int lmax, DMat &R, bool repaired) {
  const double pi = 3.14159265358979323846;
  // sqrt(2.0): a default-real (single-precision) literal in the reference
  const double sqrt_2 = repaired ? std::sqrt(2.0) : (double)std::sqrt(2.0f);
  const double cos_beta = std::cos(beta), sin_beta = std::sin(beta);
  const double cos_beta_p2 = std::cos(0.5 * beta), sin_beta_p2 = std::sin(0.5 * beta);
  const double tan_beta_p2 = std::tan(0.5 * beta);
  R(0, 0, 0) = 1.0;
  if (lmax < 1) return;
  R(0, 0, 1) = cos_beta;
  R(-1, 1, 1) = std::pow(sin_beta_p2, 2.0);
  R(0, 1, 1) = -1.0 / sqrt_2 * sin_beta;
  R(-1, 0, 1) = R(0, 1, 1);
  R(1, 0, 1) = -1.0 * R(0, 1, 1);
  R(1, 1, 1) = cos_beta_p2 * cos_beta_p2;
  auto general = [&](int l) {
    for (int m = 0; m <= l - 2; ++m) {
      for (int mp = -m; mp <= 0; ++mp) {
        R(mp, m, l) = l * (2 * l - 1) / std::sqrt((double)((l * l - m * m) * (l * l - mp * mp))) *
                      ((R(0, 0, 1) - m * mp / (double)(l * (l - 1))) * R(mp, m, l - 1) -
                       std::sqrt((double)(((l - 1) * (l - 1) - m * m) * ((l - 1) * (l - 1) - mp * mp))) *
                           R(mp, m, l - 2) / ((l - 1) * (2 * l - 1)));
        R(-m, -mp, l) = R(mp, m, l);
      }
      R(m, 0, l) = ipow(-1.0, m) * R(0, m, l);
      for (int mp = 1; mp <= m; ++mp) {
        R(mp, m, l) = l * (2 * l - 1) / std::sqrt((double)((l * l - m * m) * (l * l - mp * mp))) *
                      ((R(0, 0, 1) - m * mp / (double)(l * (l - 1))) * R(mp, m, l - 1) -
                       std::sqrt((double)(((l - 1) * (l - 1) - m * m) * ((l - 1) * (l - 1) - mp * mp))) *
                           R(mp, m, l - 2) / ((l - 1) * (2 * l - 1)));
        R(m, mp, l) = ipow(-1.0, mp + m) * R(mp, m, l);
      }
    }
    R(l, l, l) = R(1, 1, 1) * R(l - 1, l - 1, l - 1);
    R(l - 1, l - 1, l) = (l * R(0, 0, 1) - l + 1) * R(l - 1, l - 1, l - 1);
  };
  auto eq67 = [&](int l) {
    for (int mp = -1; mp >= -l + 1; --mp) {
      R(mp, l - 1, l) = (l * cos_beta - mp) *
                        std::sqrt(fact_int(2 * l - 1) / (fact_int(l + mp) * fact_int(l - mp))) *
                        ipow(cos_beta_p2, l + mp - 1) * ipow(-sin_beta_p2, l - mp - 1);
      R(-(l - 1), -mp, l) = R(mp, l - 1, l);
    }
  };
  if ((pi - std::fabs(beta)) > 1e-5) {
    for (int l = 2; l <= lmax; ++l) {
      general(l);
      for (int mp = l; mp >= 1; --mp) {
        R(mp - 1, l, l) = -1.0 * std::sqrt((double)(l + mp) / (double)(l - mp + 1)) * tan_beta_p2 *
                          R(mp, l, l);
        R(l, mp - 1, l) = ipow(-1.0, l + mp - 1) * R(mp - 1, l, l);
      }
      R(-l, 0, l) = R(0, l, l);
      R(l, 0, l) = ipow(-1.0, l) * R(0, l, l);
      for (int mp = 0; mp >= -l + 1; --mp) {
        R(mp - 1, l, l) = -1.0 * std::sqrt((double)(l + mp) / (double)(l - mp + 1)) * tan_beta_p2 *
                          R(mp, l, l);
        R(-l, -(mp - 1), l) = R(mp - 1, l, l);
      }
      R(-l + 1, l, l) = std::sqrt(fact_int(2 * l) / (fact_int(1) * fact_int(2 * l - 1))) *
                        ipow(cos_beta_p2, 1) * ipow(-sin_beta_p2, 2 * l - 1);
      for (int mp = l - 1; mp >= 1 && repaired; --mp) {
        R(mp - 1, l - 1, l) = wigner_d(l, l - 1, mp - 1, beta);
        R(l - 1, mp - 1, l) = ipow(-1.0, l - 1 + mp - 1) * R(mp - 1, l - 1, l);
      }
      for (int mp = l - 1; mp >= 1 && !repaired; --mp) {
        if (std::fabs(R(mp, l - 1, l)) > 2.220446049250313e-16)
          R(mp - 1, l - 1, l) = -1.0 * (l * cos_beta - mp + 1) / (l * cos_beta - mp) *
                                std::sqrt((double)(l + mp) / (double)(l - mp + 1)) * tan_beta_p2 *
                                R(mp, l - 1, l);
        else
          R(mp - 1, l - 1, l) = 0.0;
        R(l - 1, mp - 1, l) = ipow(-1.0, l - 1 + mp - 1) * R(mp - 1, l - 1, l);
      }
      R(-(l - 1), 0, l) = R(0, l - 1, l);
      R((l - 1), 0, l) = ipow(-1.0, l - 1) * R(0, l - 1, l);
      eq67(l);
    }
  } else {
    for (int l = 2; l <= lmax; ++l) {
      general(l);
      for (int mp = -lmax; mp <= lmax; ++mp) R(mp, l, l) = 0.0;
      for (int m = 0; m <= lmax; ++m) R(-l, m, l) = 0.0;
      for (int mp = -lmax; mp <= lmax; ++mp) R(mp, l - 1, l) = 0.0;
      for (int m = 0; m <= lmax; ++m) R(-(l - 1), m, l) = 0.0;
      R(-l, l, l) = 1.0;
      R(1 - l, l - 1, l) = -1.0;
      R(-(l - 1), -(1 - l), l) = -1.0;
      eq67(l);
    }
  }
}

// helmholtz_multipole_tools.F90:911-1001 get_real_spherical_harmonic_
// rotation_coefficients: out[l][(m'+l)(2l+1) + (m+l)] = reslt(m', m, l) for
// Euler angles (alpha, beta, gamma), m the original order, m' the new.
void ref_real_rotation(double alpha, double beta, double gamma, int lmax,
                       std::vector<std::vector<double>> &out, bool repaired) {
  const double sqrt_2 = std::sqrt(2.0);
  std::vector<double> cma(lmax + 1), sma(lmax + 1), cmg(lmax + 1), smg(lmax + 1);
  for (int m = 0; m <= lmax; ++m) {
    cma[m] = std::cos(m * alpha);
    sma[m] = std::sin(m * alpha);
    cmg[m] = std::cos(m * gamma);
    smg[m] = std::sin(m * gamma);
  }
  DMat D(lmax);
  ref_rotation_dmatrices(beta, lmax, D, repaired);
  out.assign(lmax + 1, {});
  for (int l = 0; l <= lmax; ++l) {
    const int w = 2 * l + 1;
    std::vector<double> &r = out[l];
    r.assign((size_t)w * w, 0.0);
    auto at = [&](int mp, int m) -> double & { return r[(size_t)(mp + l) * w + (m + l)]; };
    for (int m = -l; m <= -1; ++m) {
      const double sg = ipow(-1.0, -m);
      for (int mp = -l; mp <= -1; ++mp)
        at(mp, m) = -2.0 * sma[-m] * smg[-mp] * (D(-m, -mp, l) + sg * D(mp, -m, l)) / 2.0 +
                    2.0 * cma[-m] * cmg[-mp] * (D(-m, -mp, l) - sg * D(mp, -m, l)) / 2.0;
      at(0, m) = sqrt_2 * sma[-m] * (D(-m, 0, l) + sg * D(0, -m, l)) / 2.0 +
                 sqrt_2 * cma[-m] * (D(-m, 0, l) - sg * D(0, -m, l)) / 2.0;
      for (int mp = 1; mp <= l; ++mp)
        at(mp, m) = +2.0 * sma[-m] * cmg[mp] * (D(-m, mp, l) + sg * D(-mp, -m, l)) / 2.0 +
                    2.0 * cma[-m] * smg[mp] * (D(-m, mp, l) - sg * D(-mp, -m, l)) / 2.0;
    }
    for (int mp = -l; mp <= -1; ++mp)
      at(mp, 0) = -sqrt_2 * smg[-mp] * (D(0, -mp, l) + D(mp, 0, l)) / 2.0 -
                  sqrt_2 * cmg[-mp] * (D(0, -mp, l) - D(mp, 0, l)) / 2.0;
    at(0, 0) = 1.0 * (D(0, 0, l) + D(0, 0, l)) / 2.0;
    for (int mp = 1; mp <= l; ++mp)
      at(mp, 0) = sqrt_2 * cmg[mp] * (D(0, mp, l) + D(-mp, 0, l)) / 2.0 -
                  sqrt_2 * smg[mp] * (D(0, mp, l) - D(-mp, 0, l)) / 2.0;
    for (int m = 1; m <= l; ++m) {
      const double sg = ipow(-1.0, m);
      for (int mp = -l; mp <= -1; ++mp)
        at(mp, m) = -2.0 * cma[m] * smg[-mp] * (D(m, -mp, l) + sg * D(mp, m, l)) / 2.0 -
                    2.0 * sma[m] * cmg[-mp] * (D(m, -mp, l) - sg * D(mp, m, l)) / 2.0;
      at(0, m) = sqrt_2 * cma[m] * (D(m, 0, l) + sg * D(0, m, l)) / 2.0 -
                 sqrt_2 * sma[m] * (D(m, 0, l) - sg * D(0, m, l)) / 2.0;
      for (int mp = 1; mp <= l; ++mp)
        at(mp, m) = 2.0 * cma[m] * cmg[mp] * (D(m, mp, l) + sg * D(-mp, m, l)) / 2.0 -
                    2.0 * sma[m] * smg[mp] * (D(m, mp, l) - sg * D(-mp, m, l)) / 2.0;
    }
  }
}

// helmholtz_multipole_tools.F90:737-758 rotate_real_spherical_harmonic_
// expansion: reslt(l, m) = sum_m2 coefficients(m, m2, l) values(l, m2).
void ref_rotate_real(const double *in, int lmax, double alpha, double beta, double gamma,
                     double *out, bool repaired) {
  std::vector<std::vector<double>> C;
  ref_real_rotation(alpha, beta, gamma, lmax, C, repaired);
  for (int l = 0; l <= lmax; ++l) {
    const int w = 2 * l + 1;
    for (int m = -l; m <= l; ++m) {
      double s = 0.0;
      for (int m2 = -l; m2 <= l; ++m2) s += C[l][(size_t)(m + l) * w + (m2 + l)] * in[lm_map(l, m2)];
      out[lm_map(l, m)] = s;
    }
  }
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

// helmholtz_multipole_tools.F90:513-588 get_all_aligned_translation_
// coefficients (coaxial multipole-to-multipole translation along +z,
// conventional normalisation), bessel values i_0 .. i_{lin+1}(kappa d); the
// layout of orc_aligned_ml.
void orc_aligned_mm(const double *bessel, int lmax, int lin, double *out) {
  const int E = lin + 1;
  const int D = E + 2;
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
    if (n < 0) return 0.0;
    double b = std::sqrt((double)((n - m - 1) * (n - m)) / ((2 * n - 1) * (2 * n + 1)));
    if (std::abs(m) > n) return 0.0;
    if (m < 0) b = -b;
    return b;
  };
  // (:534-537) seeds (n, 0, 0) and (0, n, 0) for n = 0 .. lin + 1
  for (int n = 0; n <= lin + 1; ++n) {
    c(n, 0, 0) = ((n & 1) ? -1.0 : 1.0) * std::sqrt(2.0 * n + 1) * bessel[n];
    c(0, n, 0) = ((n & 1) ? -1.0 : 1.0) * c(n, 0, 0);
  }
  for (int n = 1; n <= lin; ++n) {  // (:543-551)
    c(1, n, 0) = (A(n, 0) * c(0, n + 1, 0) + A(n - 1, 0) * c(0, n - 1, 0)) / A(0, 0);
    c(n, 1, 0) = (((1 + n) & 1) ? -1.0 : 1.0) * c(1, n, 0);
  }
  for (int m = 0; m <= lin; ++m) {  // (:563-585)
    for (int n = m; n <= lin; ++n)
      for (int l = m; l <= lin; ++l)
        c(l, n + 1, m) = (A(l, m) * c(l + 1, n, m) + A(l - 1, m) * c(l - 1, n, m) -
                          A(n - 1, m) * c(l, n - 1, m)) /
                         A(n, m);
    for (int l = m; l <= lin; ++l)
      c(l, m + 1, m + 1) = (B(l, -m - 1) * c(l - 1, m, m) + B(l + 1, m) * c(l + 1, m, m)) /
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

// Exposed for the oracle's own tests: the reference's real rotation
// coefficients, blocks l = 0..lmax of (2l+1)^2 values, [m'][m].
void orc_ref_real_rotation(double alpha, double beta, double gamma, int lmax, int repaired,
                           double *out) {
  std::vector<std::vector<double>> C;
  ref_real_rotation(alpha, beta, gamma, lmax, C, repaired != 0);
  size_t off = 0;
  for (int l = 0; l <= lmax; ++l) {
    std::memcpy(out + off, C[l].data(), sizeof(double) * C[l].size());
    off += C[l].size();
  }
}

// Multipole-to-local conversion: Racah -> orthonormal scaling, rotation to
// the axis destination - source, coaxial translation (real basis:
// C(l, n, |m|) acting on (n, m) for both signs of m, :280-331 with
// :760-800), rotation back, orthonormal -> Racah scaling.
// kind 0: the multipole-to-local converter (k_l, orc_aligned_ml); kind 1:
// the multipole translator (i_l, orc_aligned_mm, :338-378).
static int helm_m2l_impl(int lmax, int lin, double kappa, const double *M, const double *src,
                         const double *dst, double *L, bool lsq, int kind = 0) {
  const double pi = 3.14159265358979323846;
  const double d[3] = {dst[0] - src[0], dst[1] - src[1], dst[2] - src[2]};
  const double dist = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  if (dist == 0.0) return -1;
  const int Nin = (lin + 1) * (lin + 1), Nout = (lmax + 1) * (lmax + 1);
  // Racah -> orthonormal scaling of the input (:209-214)
  std::vector<double> a(Nin, 0.0), t(Nin, 0.0);
  for (int l = 0; l <= lin; ++l)
    for (int m = -l; m <= l; ++m) t[lm_map(l, m)] = std::sqrt((2 * l + 1) / (4 * pi)) * M[lm_map(l, m)];
  // rotation to the frame whose z axis is (destination - source) / distance
  const double zv[3] = {d[0] / dist, d[1] / dist, d[2] / dist};
  const double beta = std::acos(zv[2]), alpha = std::atan2(zv[1], zv[0]), gamma = 0.0;  // :695-701
  const int Lr = lmax > lin ? lmax : lin;
  std::vector<double> R;
  std::vector<size_t> roff(Lr + 2, 0);
  if (lsq) {
    for (int l = 0; l <= Lr; ++l) roff[l + 1] = roff[l] + (size_t)(2 * l + 1) * (2 * l + 1);
    R.resize(roff[Lr + 1]);
    orc_rotation(d, Lr, R.data());
    for (int l = 0; l <= lin; ++l) {
      const int w = 2 * l + 1;
      for (int mp = -l; mp <= l; ++mp) {
        double s = 0.0;
        for (int m = -l; m <= l; ++m) s += R[roff[l] + (size_t)(mp + l) * w + (m + l)] * t[lm_map(l, m)];
        a[lm_map(l, mp)] = s;
      }
    }
  } else {
    ref_rotate_real(t.data(), lin, alpha, beta, gamma, a.data(), true);  // :240-241
  }
  // coaxial translation (:245-246)
  std::vector<double> bess(lin + 2);
  std::vector<double> C((size_t)(lmax + 1) * (lin + 1) * (lmax + 1));
  if (kind == 0) {
    orc_bessel_k(kappa * dist, lin + 1, bess.data());
    orc_aligned_ml(bess.data(), lmax, lin, C.data());
  } else {
    orc_bessel_i(kappa * dist, lin + 1, bess.data());
    orc_aligned_mm(bess.data(), lmax, lin, C.data());
  }
  std::vector<double> b(Nout, 0.0), c(Nout, 0.0);
  for (int l = 0; l <= lmax; ++l)
    for (int m = -l; m <= l; ++m) {
      const int am = std::abs(m);
      double s = 0.0;
      for (int n = am; n <= lin; ++n)
        s += C[((size_t)l * (lin + 1) + n) * (lmax + 1) + am] * a[lm_map(n, m)];
      b[lm_map(l, m)] = s;
    }
  // rotation back (:252-253) and orthonormal -> Racah scaling (:256-261)
  if (lsq) {
    for (int l = 0; l <= lmax; ++l) {
      const int w = 2 * l + 1;
      for (int m = -l; m <= l; ++m) {
        double s = 0.0;
        for (int mp = -l; mp <= l; ++mp) s += R[roff[l] + (size_t)(mp + l) * w + (m + l)] * b[lm_map(l, mp)];
        c[lm_map(l, m)] = s;
      }
    }
  } else {
    ref_rotate_real(b.data(), lmax, -gamma, -beta, -alpha, c.data(), true);
  }
  for (int l = 0; l <= lmax; ++l)
    for (int m = -l; m <= l; ++m) L[lm_map(l, m)] = std::sqrt(4 * pi / (2 * l + 1)) * c[lm_map(l, m)];
  return 0;
}

// helmholtz_multipole_tools.F90:172-278 HelmholtzExpansionTranslator_
// translate_real with the HelmholtzMultipoleConverter (:385-426), the
// rotations by the reference's recursions (ref_rotate_real).
int orc_helm_m2l(int lmax, int lin, double kappa, const double *M, const double *src,
                 const double *dst, double *L) {
  return helm_m2l_impl(lmax, lin, kappa, M, src, dst, L, false);
}

// The same conversion with the least-squares rotation (orc_rotation): an
// independent check of the recursion restatement.
int orc_helm_m2l_lsq(int lmax, int lin, double kappa, const double *M, const double *src,
                     const double *dst, double *L) {
  return helm_m2l_impl(lmax, lin, kappa, M, src, dst, L, true);
}

// helmholtz_multipole_tools.F90:172-278 translate_real with the
// HelmholtzMultipoleTranslator (:338-378): multipoles M about src moved to
// dst (GBFMMHelmholtz3D_translate_multipoles, gbfmm_helmholtz3d.F90:1223-1278).
int orc_helm_m2m(int lmax, int lin, double kappa, const double *M, const double *src,
                 const double *dst, double *out) {
  return helm_m2l_impl(lmax, lin, kappa, M, src, dst, out, false, 1);
}

// The whole (lmax+1)^2 x (lin+1)^2 matrix of the converter (kind 0) or the
// translator (kind 1) for src -> dst, column k = the image of unit input k;
// out[k * Nout + i].
int orc_helm_matrix(int kind, int lmax, int lin, double kappa, const double *src,
                    const double *dst, double *out) {
  const int Nin = (lin + 1) * (lin + 1), Nout = (lmax + 1) * (lmax + 1);
  std::vector<double> e(Nin, 0.0);
  for (int k = 0; k < Nin; ++k) {
    e[k] = 1.0;
    const int rc = helm_m2l_impl(lmax, lin, kappa, e.data(), src, dst, out + (size_t)k * Nout,
                                 false, kind);
    e[k] = 0.0;
    if (rc) return rc;
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
