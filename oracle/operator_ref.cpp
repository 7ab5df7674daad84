// operator_ref.cpp -- CPU FP64 oracle: quadrature, LIP basis, grids, Coulomb
// operator matrices, operator application, integration and Gaussian test
// densities.
//
// TEST INFRASTRUCTURE ONLY (see dage_oracle.h).  Each function restates the
// algorithm of the reference Fortran routine cited beside it, in the same
// arithmetic order where that order matters for bitwise-close results.
#include "dage_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

// erf and exp as the reference's Fortran runtime calls them (derf, dexp ->
// the C library).  Built with -DORACLE_LIBM_1ULP, every result is moved by
// -1, 0 or +1 ulp (a deterministic hash of the argument picks which): a
// second oracle that measures how far the reference algorithm's results move
// when the math library differs in the last bit, which bounds the agreement
// any other FP64 implementation (the GPU's) can show.
#ifdef ORACLE_LIBM_1ULP
inline double libm_bump(double v, double x) {
  uint64_t b;
  std::memcpy(&b, &x, 8);
  b ^= b >> 29;
  b *= 0x9E3779B97F4A7C15ull;
  int d = (int)(b >> 62) - 1;
  if (d > 1) d = 0;
  return d ? std::nextafter(v, d > 0 ? INFINITY : -INFINITY) : v;
}
inline double m_erf(double x) { return libm_bump(std::erf(x), x); }
inline double m_exp(double x) { return libm_bump(std::exp(x), x + 0.5); }
#else
inline double m_erf(double x) { return std::erf(x); }
inline double m_exp(double x) { return std::exp(x); }
#endif

const double PI = std::acos(-1.0);          // globals.F90:54
const double SQRTPI = std::sqrt(PI);        // globals.F90:57
const double TWOOVERSQRTPI = 2.0 / SQRTPI;  // globals.F90:61

// Integer power by repeated squaring (the libgcc __powidf2 scheme used for
// Fortran x**n with an integer exponent).
inline double powi(double x, int n) {
  unsigned m = (unsigned)n;
  double y = (m & 1u) ? x : 1.0;
  while (m >>= 1) {
    x = x * x;
    if (m & 1u) y = y * x;
  }
  return y;
}

// gauss.F90:427-452 gauss_lobatto_grid (only n = 6, 7 are defined there).
bool gauss_lobatto_grid(int n, double left, double right, double *tp) {
  if (n == 6) {
    tp[0] = -1.0;
    tp[1] = -std::sqrt((7.0 + 2 * std::sqrt(7.0)) / 21.0);
    tp[2] = -std::sqrt((7.0 - 2 * std::sqrt(7.0)) / 21.0);
    tp[3] = std::sqrt((7.0 - 2 * std::sqrt(7.0)) / 21.0);
    tp[4] = std::sqrt((7.0 + 2 * std::sqrt(7.0)) / 21.0);
    tp[5] = 1.0;
  } else if (n == 7) {
    tp[0] = -1.0;
    tp[1] = -std::sqrt((15.0 + 2 * std::sqrt(15.0)) / 33.0);
    tp[2] = -std::sqrt((15.0 - 2 * std::sqrt(15.0)) / 33.0);
    tp[3] = 0.0;
    tp[4] = std::sqrt((15.0 - 2 * std::sqrt(15.0)) / 33.0);
    tp[5] = std::sqrt((15.0 + 2 * std::sqrt(15.0)) / 33.0);
    tp[6] = 1.0;
  } else {
    return false;
  }
  for (int i = 0; i < n; ++i) tp[i] = 0.5 * ((right + left) + (right - left) * tp[i]);
  return true;
}

struct Lip {
  int n = 0, type = 0;
  double first = 0, last = 0;
  std::vector<double> c;  // c[(k)*n + j] = p(j+1, k+1), column-major
  double &p(int j, int k) { return c[(size_t)k * n + j]; }
};

// lip.F90:118-141 LIPBasisInit + lip.F90:285-362 LIPBasis_coeffs(0)
bool make_lip(int nlip, int grid_type, Lip &L) {
  L.n = nlip;
  L.type = grid_type;
  if (grid_type != 1 && grid_type != 2) return false;
  L.first = (double)(-((nlip - 1) / 2));
  L.last = (double)(nlip / 2);
  L.c.assign((size_t)nlip * nlip, 0.0);
  const int n = nlip;
  std::vector<double> xs(n);
  if (grid_type == 1) {
    for (int i = 1; i <= n; ++i) xs[i - 1] = (double)(i - (nlip + 1) / 2);
  } else {
    if (!gauss_lobatto_grid(n, L.first, L.last, xs.data())) return false;
  }
  for (int j = 0; j < n; ++j) L.p(j, n - 1) = 1.0;
  std::vector<double> old(n);
  for (int i = 1; i <= n; ++i) {
    const double x_i = xs[i - 1];
    for (int j = 1; j <= n; ++j) {
      if (i == j) continue;
      double dx = (grid_type == 1) ? (double)(j - i) : (xs[j - 1] - xs[i - 1]);
      for (int k = 0; k < n; ++k) old[k] = L.p(j - 1, k);
      for (int k = 0; k < n - 1; ++k) L.p(j - 1, k) = (old[k + 1] - old[k] * x_i) / dx;
      L.p(j - 1, n - 1) = -old[n - 1] * x_i / dx;
    }
  }
  return true;
}

// lip.F90:369-411 integral_coeffs + integrals
void lip_integrals(Lip &L, double *ints) {
  const int n = L.n;
  std::vector<double> ic((size_t)n * (n + 1), 0.0);  // ic[k*n + j]
  for (int i = 0; i <= n - 1; ++i)
    for (int j = 0; j < n; ++j) ic[(size_t)(n - 1 - i) * n + j] = L.p(j, n - 1 - i) / (i + 1);
  for (int j = 0; j < n; ++j) {
    double t1 = 0.0, t2 = 0.0;
    for (int i = 0; i < n; ++i) t1 = (t1 + ic[(size_t)i * n + j]) * L.first;
    for (int i = 0; i < n; ++i) t2 = (t2 + ic[(size_t)i * n + j]) * L.last;
    ints[j] = t2 - t1;
  }
}

struct Grid1 {
  int ncell, nlip, type;
  double first;
  std::vector<double> h, celld, pts;
};

// grid.F90:446-534 Grid1D_init_step
bool make_grid(double qmin, int ncell, int nlip, int grid_type, const double *cs,
               Grid1 &g) {
  g.ncell = ncell;
  g.nlip = nlip;
  g.type = grid_type;
  g.first = (double)(-((nlip - 1) / 2));
  g.h.assign(cs, cs + ncell);
  g.celld.assign(ncell, 0.0);
  g.pts.assign((size_t)ncell * (nlip - 1) + 1, 0.0);
  std::vector<double> tmpl(nlip - 1);
  if (grid_type == 1) {
    for (int k = 1; k <= nlip - 1; ++k) tmpl[k - 1] = (double)k;
  } else if (grid_type == 2) {
    std::vector<double> gl(nlip);
    if (!gauss_lobatto_grid(nlip, 0.0, (double)(nlip - 1), gl.data())) return false;
    for (int k = 1; k <= nlip - 1; ++k) tmpl[k - 1] = gl[k];
  } else {
    return false;
  }
  size_t ip = 0;
  g.pts[0] = qmin;
  for (int ic = 0; ic < ncell; ++ic) {
    g.celld[ic] = g.pts[ip];
    for (int k = 1; k <= nlip - 1; ++k) {
      ++ip;
      g.pts[ip] = g.celld[ic] + tmpl[k - 1] * g.h[ic];
    }
  }
  return true;
}

// ---------------------------------------------------------------------------
// Analytic integrals int_a^b x^n exp(-t^2 (x-p)^2) dx, exponentials.F90:695-1297
// ---------------------------------------------------------------------------
inline double ser(double q) {  // q + q^2/2 + q^3/6 + q^4/24 as written there
  return q + q * q / 2.0 + q * q * q / 6.0 + q * q * q * q / 24.0;
}
inline double ser1(double q) {  // 1 + q + ...
  return 1.0 + q + q * q / 2.0 + q * q * q / 6.0 + q * q * q * q / 24.0;
}

double expo_0(double a, double b, double t, double p) {
  const double thr = 1.0e-06;
  if (t == 0.0 || t < thr) return b - a;
  return SQRTPI * (m_erf(b * t - t * p) - m_erf(a * t - t * p)) / t / 2.0;
}

double expo_1(double a, double b, double t, double p) {
  const double thr = 1.0e-06;
  if (t == 0.0 || t < thr) return (b * b - a * a) / 2.0;
  double v1 = p * SQRTPI * m_erf(t * (b - p));
  double v2;
  if (t > 1.0e-03) {
    v2 = (m_exp(-(t * t) * ((a - p) * (a - p))) - m_exp(-(t * t) * ((b - p) * (b - p)))) / t;
  } else {
    double q = -(t * t) * ((a - p) * (a - p));
    double r = -(t * t) * ((b - p) * (b - p));
    v2 = (q + q * q / 2.0 + q * q * q / 6.0 + q * q * q * q / 24.0 - r - r * r / 2.0 -
          r * r * r / 6.0 - r * r * r * r / 24.0) /
         t;
  }
  double v3 = -p * SQRTPI * m_erf(a * t - t * p);
  return (v1 + v2 + v3) / t / 2.0;
}

double expo_2(double a, double b, double t, double p) {
  const double thr = 0.5e-04;
  if (t == 0.0 || t < thr) return (b * b * b - a * a * a) / 3.0;
  double v1 = p * p * SQRTPI * m_erf(b * t - t * p) / 2.0;
  double v2, v3;
  if (t > 1.0e-03) {
    double ea = m_exp(-(t * t * ((a - p) * (a - p))));
    double eb = m_exp(-(t * t * ((b - p) * (b - p))));
    v2 = (ea * a - eb * b);
    v3 = (ea - eb) * p / t / 2.0;
  } else {
    double q = -(t * t * ((a - p) * (a - p)));
    double r = -(t * t * ((b - p) * (b - p)));
    v2 = ser(q) * a - ser(r) * b;
    v2 = (v2 + a - b);
    v3 = ser(q) - ser(r);
    v3 = v3 * p / t / 2.0;
  }
  double v5 = SQRTPI * (m_erf(t * (b - p)) - m_erf(t * (a - p))) / t / 2.0;
  v2 = (v2 + v5) / t / 2.0;
  v5 = 0.0;
  double v4 = -(p * p) * SQRTPI * m_erf(a * t - t * p) / 2.0;
  return (v1 + v2 + v3 + v4 + v5) / t;
}

double expo_3(double a, double b, double t, double p) {
  const double thr = 1.0e-04;
  if (t == 0.0 || t < thr) return (powi(b, 4) - powi(a, 4)) / 4.0;
  double v1, v2, v3, v5;
  if (t > 1.0e-03) {
    double ea = m_exp(-(t * t) * ((a - p) * (a - p)));
    double eb = m_exp(-(t * t) * ((b - p) * (b - p)));
    double ea2 = m_exp(-(t * t * ((a - p) * (a - p))));
    double eb2 = m_exp(-(t * t * ((b - p) * (b - p))));
    v1 = 2.0 * (ea * (a * a) - eb * (b * b)) / (t * t);
    v2 = 2.0 * p * (a * ea2 - b * eb2) * t;
    v3 = 2.0 * (ea * (p * p) - eb * (p * p)) / (t * t);
    v5 = 2.0 * (ea - eb) / t;
  } else {
    double q = -(t * t * ((a - p) * (a - p)));
    double r = -(t * t * ((b - p) * (b - p)));
    v1 = ser1(q) * a * a - ser1(r) * b * b;
    v1 = 2.0 * v1 / t / t;
    v2 = ser(q) * a - ser(r) * b;
    v2 = v2 + a - b;
    v2 = 2.0 * v2 * p * t;
    v3 = ser(q) - ser(r);
    v3 = 2.0 * v3 * p * p / t / t;
    v5 = ser(q) - ser(r);
    v5 = 2.0 * v5 / t;
  }
  double eb_ = m_erf(b * t - t * p), ea_ = m_erf(a * t - t * p);
  double v4 = 2.0 * powi(p, 3) * SQRTPI * (eb_ - ea_) / t;
  double v6 = 3.0 * p * SQRTPI * (eb_ - ea_);
  v6 = (v6 + v2 + v5) / t / t / t;
  v2 = 0.0;
  v5 = 0.0;
  return 0.25 * (v1 + v2 + v3 + v4 + v5 + v6);
}

double expo_4(double a, double b, double t, double p) {
  const double thr = 1.0e-03;
  if (t == 0.0 || t < thr) return (powi(b, 5) - powi(a, 5)) / 5.0;
  double v1, v2, v3, v4, v7, v8;
  if (t > 1.0e-03) {
    double ea = m_exp(-(t * t) * ((a - p) * (a - p)));
    double eb = m_exp(-(t * t) * ((b - p) * (b - p)));
    v1 = 4.0 * (ea * powi(a, 3) - eb * powi(b, 3));
    v2 = 4.0 * (ea * p * (a * a) - eb * p * (b * b));
    v3 = 4.0 * (ea * (p * p) * a - eb * (p * p) * b);
    v4 = 4.0 * (ea * powi(p, 3) - eb * powi(p, 3));
    v7 = 10.0 * p * (ea - eb) / t / t;
    v8 = 6.0 * (ea * a - eb * b);
  } else {
    double q = -(t * t * ((a - p) * (a - p)));
    double r = -(t * t * ((b - p) * (b - p)));
    v1 = ser1(q) * powi(a, 3) - ser1(r) * powi(b, 3);
    v1 = 4.0 * v1;
    v2 = ser1(q) * p * a * a - ser1(r) * p * b * b;
    v2 = 4.0 * v2;
    v3 = ser1(q) * p * p * a - ser1(r) * p * p * b;
    v3 = 4.0 * v3;
    v4 = ser(q) - ser(r);
    v4 = 4.0 * v4 * powi(p, 3);
    v7 = ser(q) - ser(r);
    v7 = 10.0 * v7 * p / t / t;
    v8 = ser1(q) * a - ser1(r) * b;
    v8 = 6.0 * v8;
  }
  double d = m_erf(a * t - t * p) - m_erf(b * t - t * p);
  double v5 = -(4.0 * t * powi(p, 4) * SQRTPI * d);
  double v6 = -(12.0 / t * (p * p) * SQRTPI * d);
  double v9 = -(3.0 * SQRTPI * d / t);
  v2 = v2 / (t * t);
  v5 = (v4 + v5) / (t * t);
  v7 = (v3 + v6 + v7) / (t * t);
  v8 = ((v8 + v9) / t / t + v1) / (t * t);
  v1 = 0.0;
  v3 = 0.0;
  v4 = 0.0;
  v6 = 0.0;
  v9 = 0.0;
  return 0.125 * (v1 + v2 + v3 + v4 + v5 + v6 + v7 + v8 + v9);
}

double expo_5(double a, double b, double t, double p) {
  const double thr = 2.5e-03;
  if (t == 0.0 || t < thr) return (powi(b, 6) - powi(a, 6)) / 6.0;
  double v1, v2, v3, v4, v5, v8, v9, v11, v12;
  const double t2 = t * t;
  if (t > 1.0e-02) {
    double ea = m_exp(-t2 * ((a - p) * (a - p)));
    double eb = m_exp(-t2 * ((b - p) * (b - p)));
    v1 = 4.0 * (ea * powi(a, 4) - eb * powi(b, 4));
    v2 = 4.0 * (ea * p * powi(a, 3) - eb * p * powi(b, 3));
    v3 = 4.0 * (ea * (p * p) * (a * a) - eb * (p * p) * (b * b));
    v4 = 4.0 * (ea * powi(p, 3) * a - eb * powi(p, 3) * b);
    v5 = 4.0 * (ea * powi(p, 4) - eb * powi(p, 4));
    v8 = 18.0 * (ea - eb) * (p * p) / t2;
    v9 = 14.0 * (ea * p * a - eb * p * b) / t2;
    v11 = 8.0 * (ea * (a * a) - eb * (b * b)) / t2;
    v12 = 8.0 * (ea - eb) / powi(t, 4);
  } else {
    double q = -(t * t * ((a - p) * (a - p)));
    double r = -(t * t * ((b - p) * (b - p)));
    v1 = 4.0 * (ser1(q) * powi(a, 4) - ser1(r) * powi(b, 4));
    v2 = 4.0 * (ser1(q) * p * powi(a, 3) - ser1(r) * p * powi(b, 3));
    v3 = 4.0 * (ser1(q) * (p * p) * (a * a) - ser1(r) * (p * p) * (b * b));
    v4 = 4.0 * (ser1(q) * powi(p, 3) * a - ser1(r) * powi(p, 3) * b);
    v5 = 4.0 * (ser(q) * powi(p, 4) - ser(r) * powi(p, 4));
    v8 = 18.0 * ((ser(q) - ser(r)) * (p * p) / t2);
    v9 = 14.0 * ((ser1(q) * a * p - ser1(r) * b * p) / t2);
    v11 = 8.0 * ((ser1(q) * a * a - ser1(r) * b * b) / t2);
    v12 = 8.0 * ((ser(q) - ser(r)) / powi(t, 4));
  }
  double d = m_erf(a * t - t * p) - m_erf(b * t - t * p);
  double v6 = -(4.0 * t * powi(p, 5) * SQRTPI * d);
  double v7 = -(20.0 / t * powi(p, 3) * SQRTPI * d);
  double v10 = -(15.0 * p * SQRTPI * d / powi(t, 3));
  double value = v1 + v2 + v3 + v4 + v5 + v6;
  value = value + v7 + v8 + v9 + v10 + v11 + v12;
  value = value / t2;
  return 0.125 * value;
}

double expo_6(double a, double b, double t, double p) {
  const double thr = 5.0e-03;
  if (t == 0.0 || t < thr) return (powi(b, 7) - powi(a, 7)) / 7.0;
  const double ea = m_exp(-(t * t) * ((a - p) * (a - p)));
  const double eb = m_exp(-(t * t) * ((b - p) * (b - p)));
  const double d = m_erf(b * t - t * p) - m_erf(a * t - t * p);
  double v1 = 30.0 * (ea * a - eb * b);
  double v2 = 15.0 * SQRTPI * d;
  v1 = (v1 + v2 / t) / t / t / t;
  v2 = 0.0;
  double v3 = 90.0 * (p * p) * SQRTPI * d / t / t;
  double v4 = 56.0 * (ea - eb) * powi(p, 3) / t;
  double v5 = 66.0 * (ea - eb) * p / t / t / t;
  double v6 = 8.0 * (ea - eb) * powi(p, 5) * t;
  double v7 = 20.0 * (ea * powi(a, 3) - eb * powi(b, 3)) / t;
  double v8 = 36.0 * (ea * (a * a) - eb * (b * b)) * p / t;
  double v9 = 48.0 * (ea * a - eb * b) * (p * p) / t;
  double v10 = 8.0 * powi(p, 6) * SQRTPI * d * (t * t);
  double v11 = 8.0 * (ea * powi(a, 4) - eb * powi(b, 4)) * p * t;
  double v12 = 8.0 * (ea * powi(a, 3) - eb * powi(b, 3)) * (p * p) * t;
  double v13 = 8.0 * (ea * powi(a, 5) - eb * powi(b, 5)) * t;
  double v14 = 8.0 * (ea * a - eb * b) * powi(p, 4) * t;
  double v15 = 8.0 * (ea * (a * a) - eb * (b * b)) * powi(p, 3) * t;
  double v16 = 60.0 * powi(p, 4) * SQRTPI * d;
  double value = v1 + v2 + v3 + v4 + v5 + v6 + v7 + v8;
  value = value + v9 + v10 + v11 + v12 + v13 + v14 + v15 + v16;
  value = value / powi(t, 3);
  return 0.0625 * value;
}

// 12-point Gauss-Legendre rule with the 15-digit constants written in
// exponentials.F90:2370-2394 (kept to those digits for parity).
const double GL12_W[12] = {0.047175336386512, 0.106939325995318, 0.160078328543346,
                           0.203167426723066, 0.233492536538355, 0.249147045813403,
                           0.249147045813403, 0.233492536538355, 0.203167426723066,
                           0.160078328543346, 0.106939325995318, 0.047175336386512};
const double GL12_X[12] = {-0.981560634246719, -0.904117256370475, -0.769902674194305,
                           -0.587317954286617, -0.367831498998180, -0.125233408511469,
                           0.125233408511469,  0.367831498998180,  0.587317954286617,
                           0.769902674194305,  0.904117256370475,  0.981560634246719};

// exponentials.F90:2287-2429 gauss_expo_n: 4 equal sub-intervals x 12 points.
double gauss_expo_n(double a, double b, double t, double p, int n) {
  if (t == 0.0) {
    if (n == 0) return b - a;
    return (powi(b, n + 1) - powi(a, n + 1)) / (n + 1);
  }
  const int interval = 4;
  double limit[5];
  for (int i = 1; i <= interval + 1; ++i)
    limit[i - 1] = ((interval + 1 - i) * a + (i - 1) * b) / interval;
  double summa = 0.0;
  for (int i = 1; i <= interval; ++i) {
    double a0 = limit[i - 1], a1 = limit[i];
    double pr = 1.0 - a1 * 2.0 / (a1 - a0);
    double qr = 2.0 / (a1 - a0);
    for (int j = 0; j < 12; ++j) {
      double tp = (GL12_X[j] - pr) / qr;
      double tw = GL12_W[j] / qr;
      double e = m_exp(-(t * t * (tp - p) * (tp - p)));
      if (n > 0)
        summa = summa + powi(tp, n) * e * tw;
      else
        summa = summa + e * tw;
    }
  }
  return summa;
}

double expo_an(double a, double b, double t, double p, int n) {
  switch (n) {
    case 0: return expo_0(a, b, t, p);
    case 1: return expo_1(a, b, t, p);
    case 2: return expo_2(a, b, t, p);
    case 3: return expo_3(a, b, t, p);
    case 4: return expo_4(a, b, t, p);
    case 5: return expo_5(a, b, t, p);
    case 6: return expo_6(a, b, t, p);
  }
  return 0.0;
}

// exponentials.F90:647-666
void integrals(double a, double b, double t, double p, int n, double *values) {
  if (t < 0.1) {
    for (int i = 0; i < n; ++i) values[n - 1 - i] = gauss_expo_n(a, b, t, p, i);
  } else {
    for (int i = 0; i < n; ++i) values[n - 1 - i] = expo_an(a, b, t, p, i);
  }
}

// One (t-point, input cell, output point) element of exponentials():
// temp = (lip_coeffs x integrals) * cell_scale (exponentials.F90:270-330).
inline void cell_row(const Lip &L, double cell_scale, double t, double pst0, double *out) {
  const int n = L.n;
  double vals[16];
  integrals(L.first, L.last, t * cell_scale, pst0, n, vals);
  for (int j = 0; j < n; ++j) {
    double s = 0.0;
    for (int k = 0; k < n; ++k) s += L.c[(size_t)k * n + j] * vals[k];
    out[j] = s * cell_scale;
  }
}

}  // namespace

extern "C" {

void orc_gauleg(int n, double *x, double *w) {
  // gauss.F90:344-383
  const double EPS = 3.0e-15;
  const int m = (n + 1) / 2;
  for (int i = 1; i <= m; ++i) {
    double z = std::cos(PI * (i - 0.25) / (n + 0.5));
    double p1, p2, p3, pp, z1;
    do {
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
    } while (std::fabs(z - z1) > EPS);
    x[i - 1] = -z;
    x[n - i] = z;
    w[i - 1] = 2.0 / ((1.0 - z * z) * pp * pp);
    w[n - i] = w[i - 1];
  }
}

void orc_gauss_quad(int nlin, int nlog, double tstart, double tlin, double tlog,
                    double *tp, double *tw) {
  // gauss.F90:81-122 and gauleg_int (gauss.F90:307-322)
  if (nlin > 0) {
    orc_gauleg(nlin, tp, tw);
    for (int i = 0; i < nlin; ++i) {
      tp[i] = 0.5 * ((tlin + tstart) + (tlin - tstart) * tp[i]);
      tw[i] = 0.5 * (tlin - tstart) * tw[i];
    }
  }
  if (nlog > 0) {
    double *lp = tp + nlin, *lw = tw + nlin;
    orc_gauleg(nlog, lp, lw);
    const double a = tlin, b = tlog;
    for (int i = 0; i < nlog; ++i) lp[i] = a * std::pow(b / a, 0.5 * (lp[i] + 1.0));
    for (int i = 0; i < nlog; ++i) lw[i] = 0.5 * std::log(b / a) * lw[i] * lp[i];
  }
}

int orc_lip_coeffs(int nlip, int grid_type, double *coeffs, double *first, double *last) {
  Lip L;
  if (!make_lip(nlip, grid_type, L)) return -1;
  std::memcpy(coeffs, L.c.data(), sizeof(double) * nlip * nlip);
  *first = L.first;
  *last = L.last;
  return 0;
}

int orc_lip_integrals(int nlip, int grid_type, double *ints) {
  Lip L;
  if (!make_lip(nlip, grid_type, L)) return -1;
  lip_integrals(L, ints);
  return 0;
}

int orc_grid1d_points(double qmin, int ncell, int nlip, int grid_type,
                      const double *cell_scales, double *points, double *celld) {
  Grid1 g;
  if (!make_grid(qmin, ncell, nlip, grid_type, cell_scales, g)) return -1;
  std::memcpy(points, g.pts.data(), sizeof(double) * g.pts.size());
  if (celld) std::memcpy(celld, g.celld.data(), sizeof(double) * ncell);
  return 0;
}

int orc_grid1d_spheres(int n, const double *centers, const double *radii, double step,
                       int nlip, double *qmin, double *cell_scale) {
  // grid.F90:604-640 Grid1D_init_spheres, then grid.F90:539-564
  // Grid1D_init_equidistant.
  double b1 = centers[0] - radii[0], b2 = centers[0] + radii[0];
  for (int i = 1; i < n; ++i) {
    b1 = std::min(b1, centers[i] - radii[i]);
    b2 = std::max(b2, centers[i] + radii[i]);
  }
  double cell_len = step * (nlip - 1);
  int ncell = (int)std::ceil((b2 - b1) / cell_len);
  double dx = ncell * cell_len - (b2 - b1);
  b1 = b1 - 0.5 * dx;
  b2 = b2 + 0.5 * dx;
  int nc = (int)std::ceil((b2 - b1) / (step * (nlip - 1)));
  double s = (b2 - b1) / (double)(nc * (nlip - 1));
  *qmin = b1;
  *cell_scale = s;
  return nc;
}

int orc_grid1d_weights(int ncell, int nlip, int grid_type, const double *cell_scales,
                       double *weights) {
  Lip L;
  if (!make_lip(nlip, grid_type, L)) return -1;
  std::vector<double> bi(nlip);
  lip_integrals(L, bi.data());
  const int n = ncell * (nlip - 1) + 1;
  for (int i = 0; i < n; ++i) weights[i] = 0.0;
  for (int c = 0; c < ncell; ++c)
    for (int i = 0; i < nlip; ++i) weights[c * (nlip - 1) + i] += bi[i] * cell_scales[c];
  return 0;
}

void orc_expo_integrals(double a, double b, double t, double p, int n, double *values) {
  integrals(a, b, t, p, n, values);
}

int orc_coulomb_matrix(double qmin_in, int ncell_in, int nlip, int grid_type,
                       const double *cell_scales_in, int n_out, const double *out_points,
                       int P, const double *tp, double *T) {
  Lip L;
  Grid1 g;
  if (!make_lip(nlip, grid_type, L)) return -1;
  if (!make_grid(qmin_in, ncell_in, nlip, grid_type, cell_scales_in, g)) return -1;
  const int n_in = ncell_in * (nlip - 1) + 1;
  const size_t slab = (size_t)n_out * n_in;
#pragma omp parallel for schedule(dynamic)
  for (int ip = 0; ip < P; ++ip) {
    double *Tp = T + slab * ip;
    std::fill(Tp, Tp + slab, 0.0);
    double row[16];
    for (int ic = 0; ic < ncell_in; ++ic) {
      const double h = g.h[ic];
      const int j0 = ic * (nlip - 1);
      for (int io = 0; io < n_out; ++io) {
        const double pst0 = (out_points[io] - g.celld[ic]) / h + L.first;  // grid.F90:1768-1776
        cell_row(L, h, tp[ip], pst0, row);
        for (int j = 0; j < nlip; ++j) Tp[(size_t)(j0 + j) * n_out + io] += row[j];
      }
    }
  }
  return 0;
}

int orc_coulomb_border_matrix(double qmin_in, int ncell_in, int nlip, int grid_type,
                              const double *cell_scales_in, int n_out,
                              const double *out_points, int P, const double *tp,
                              double *T) {
  // exponentials.F90:348-600: the first and last input cells against every
  // output point, then the interior cells against the first and last output
  // points only.
  Lip L;
  Grid1 g;
  if (!make_lip(nlip, grid_type, L)) return -1;
  if (!make_grid(qmin_in, ncell_in, nlip, grid_type, cell_scales_in, g)) return -1;
  const int n_in = ncell_in * (nlip - 1) + 1;
  const size_t slab = (size_t)n_out * n_in;
#pragma omp parallel for schedule(dynamic)
  for (int ip = 0; ip < P; ++ip) {
    double *Tp = T + slab * ip;
    std::fill(Tp, Tp + slab, 0.0);
    double row[16];
    const int edge_cells[2] = {0, ncell_in - 1};
    for (int e = 0; e < 2; ++e) {
      const int ic = edge_cells[e];
      const double h = g.h[ic];
      const int j0 = ic * (nlip - 1);
      for (int io = 0; io < n_out; ++io) {
        const double pst0 = (out_points[io] - g.celld[ic]) / h + L.first;
        cell_row(L, h, tp[ip], pst0, row);
        for (int j = 0; j < nlip; ++j) Tp[(size_t)(j0 + j) * n_out + io] += row[j];
      }
    }
    const int edge_pts[2] = {0, n_out - 1};
    for (int ic = 1; ic < ncell_in - 1; ++ic) {
      const double h = g.h[ic];
      const int j0 = ic * (nlip - 1);
      for (int e = 0; e < 2; ++e) {
        const int io = edge_pts[e];
        const double pst0 = (out_points[io] - g.celld[ic]) / h + L.first;
        cell_row(L, h, tp[ip], pst0, row);
        for (int j = 0; j < nlip; ++j) Tp[(size_t)(j0 + j) * n_out + io] += row[j];
      }
    }
  }
  return 0;
}

int orc_transform_cube(int nix, int niy, int niz, int nox, int noy, int noz, int P,
                       const double *Tx, const double *Ty, const double *Tz, const double *w,
                       double coda, const double *rho, double *V) {
  // function3d.F90:4296-4332 (CPU branch): per t-point, x and y products per
  // z-slice, then the z product per output y-plane, weighted and accumulated.
  const size_t nout = (size_t)nox * noy * noz;
  std::fill(V, V + nout, 0.0);
  std::vector<double> tmp_u((size_t)nox * noy * niz);
  for (int ip = 0; ip < P; ++ip) {
    const double *tx = Tx + (size_t)nox * nix * ip;
    const double *ty = Ty + (size_t)noy * niy * ip;
    const double *tz = Tz + (size_t)noz * niz * ip;
#pragma omp parallel
    {
      std::vector<double> tmp1((size_t)nox * niy);
#pragma omp for schedule(static)
      for (int iz = 0; iz < niz; ++iz) {
        // tmp1 = fX(:,:,ip) . rho(:,:,iz)          [nox x niy]
        std::fill(tmp1.begin(), tmp1.end(), 0.0);
        const double *r = rho + (size_t)nix * niy * iz;
        for (int b = 0; b < niy; ++b)
          for (int a = 0; a < nix; ++a) {
            const double rv = r[(size_t)b * nix + a];
            const double *col = tx + (size_t)a * nox;
            double *o = tmp1.data() + (size_t)b * nox;
            for (int i = 0; i < nox; ++i) o[i] += col[i] * rv;
          }
        // tmp_u(:,:,iz) = tmp1 . fY(:,:,ip), fY(b, j) = Ty(j, b)   [nox x noy]
        double *u = tmp_u.data() + (size_t)nox * noy * iz;
        std::fill(u, u + (size_t)nox * noy, 0.0);
        for (int j = 0; j < noy; ++j)
          for (int b = 0; b < niy; ++b) {
            const double f = ty[(size_t)b * noy + j];
            const double *src = tmp1.data() + (size_t)b * nox;
            double *o = u + (size_t)j * nox;
            for (int i = 0; i < nox; ++i) o[i] += src[i] * f;
          }
      }
#pragma omp for schedule(static)
      for (int iy = 0; iy < noy; ++iy) {
        // cubeout(:,iy,:) += w(ip) * tmp_u(:,iy,:) . fZ(:,:,ip)
        std::vector<double> acc((size_t)nox * noz, 0.0);
        for (int k = 0; k < noz; ++k)
          for (int c = 0; c < niz; ++c) {
            const double f = tz[(size_t)c * noz + k];
            const double *src = tmp_u.data() + (size_t)nox * noy * c + (size_t)iy * nox;
            double *o = acc.data() + (size_t)k * nox;
            for (int i = 0; i < nox; ++i) o[i] += src[i] * f;
          }
        for (int k = 0; k < noz; ++k) {
          double *dst = V + (size_t)nox * noy * k + (size_t)iy * nox;
          const double *s = acc.data() + (size_t)k * nox;
          for (int i = 0; i < nox; ++i) dst[i] = dst[i] + w[ip] * s[i];
        }
      }
    }
  }
  if (coda != 0.0 && nix == nox && niy == noy && niz == noz) {
    for (size_t i = 0; i < nout; ++i) V[i] = V[i] + coda * rho[i];
  }
  return 0;
}

double orc_integrate_cube(int nlip, int grid_type, int ncx, const double *hx, int ncy,
                          const double *hy, int ncz, const double *hz, const double *f) {
  // evaluators.F90:1064-1098: contract x (per (y,z) line), then y, then z.
  Lip L;
  if (!make_lip(nlip, grid_type, L)) return NAN;
  std::vector<double> bi(nlip);
  lip_integrals(L, bi.data());
  const int nc[3] = {ncx, ncy, ncz};
  const double *h[3] = {hx, hy, hz};
  int shape[3];
  for (int d = 0; d < 3; ++d) shape[d] = nc[d] * (nlip - 1) + 1;
  size_t len = (size_t)shape[0] * shape[1] * shape[2];
  std::vector<double> cur(f, f + len), nxt;
  for (int d = 0; d < 3; ++d) {
    const size_t blk = len / shape[d];
    nxt.assign(blk, 0.0);
    size_t a = 0;
    for (size_t k = 0; k < blk; ++k) {
      for (int ic = 0; ic < nc[d]; ++ic) {
        double s = 0.0;
        for (int i = 0; i < nlip; ++i) s += cur[a + i] * bi[i];
        nxt[k] = nxt[k] + s * h[d][ic];
        a += nlip - 1;
      }
      a += 1;
    }
    cur.swap(nxt);
    len = blk;
  }
  return cur[0];
}

void orc_gauss_cube(int ng, const double *q, const double *alpha, const double *centers,
                    int nx, const double *x, int ny, const double *y, int nz, const double *z,
                    double *cube) {
  // gauss_generator.F90:291-318
  const size_t n = (size_t)nx * ny * nz;
  std::fill(cube, cube + n, 0.0);
  std::vector<double> ex(nx), ey(ny), ez(nz);
  for (int p = 0; p < ng; ++p) {
    const double norm = std::pow(alpha[p] / PI, 1.5);
    for (int i = 0; i < nx; ++i) ex[i] = std::exp(-alpha[p] * ((x[i] - centers[3 * p]) * (x[i] - centers[3 * p])));
    for (int j = 0; j < ny; ++j) ey[j] = std::exp(-alpha[p] * ((y[j] - centers[3 * p + 1]) * (y[j] - centers[3 * p + 1])));
    for (int k = 0; k < nz; ++k) ez[k] = std::exp(-alpha[p] * ((z[k] - centers[3 * p + 2]) * (z[k] - centers[3 * p + 2])));
    const double qn = q[p] * norm;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j) {
        double *row = cube + (size_t)nx * ny * k + (size_t)nx * j;
        for (int i = 0; i < nx; ++i) row[i] = row[i] + qn * ex[i] * ey[j] * ez[k];
      }
  }
}

static double gausspot(double alpha, double r) {
  // gauss_generator.F90:411-428
  const double sa = std::sqrt(alpha);
  const double temp = r * sa;
  if (temp < 0.01)
    return TWOOVERSQRTPI * sa * (1.0 - 0.33333333333333333 * (temp * temp) + 0.1 * powi(temp, 4));
  if (temp < 10.0) return std::erf(r * sa) / r;
  return 1.0 / r;
}

void orc_gauss_pot_cube(int ng, const double *q, const double *alpha, const double *centers,
                        int nx, const double *x, int ny, const double *y, int nz,
                        const double *z, double *cube) {
  const size_t n = (size_t)nx * ny * nz;
  std::fill(cube, cube + n, 0.0);
  for (int p = 0; p < ng; ++p) {
    const double cx = centers[3 * p], cy = centers[3 * p + 1], cz = centers[3 * p + 2];
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const double r = std::sqrt((cx - x[i]) * (cx - x[i]) + (cy - y[j]) * (cy - y[j]) +
                                     (cz - z[k]) * (cz - z[k]));
          double &c = cube[(size_t)nx * ny * k + (size_t)nx * j + i];
          c = c + q[p] * gausspot(alpha[p], r);
        }
  }
}

double orc_gauss_analytical_energy(int ng, const double *q, const double *alpha,
                                   const double *centers) {
  // analytical.F90:308-420 (no PBC)
  double E = 0.0;
  for (int i = 0; i < ng; ++i) {
    E = E + q[i] * q[i] * std::sqrt(2.0 * alpha[i] / PI);
    for (int j = i + 1; j < ng; ++j) {
      double d2 = 0.0;
      for (int c = 0; c < 3; ++c) {
        const double d = centers[3 * i + c] - centers[3 * j + c];
        d2 += d * d;
      }
      const double rij = std::sqrt(d2);
      const double sqrtmu = std::sqrt((alpha[i] * alpha[j]) / (alpha[i] + alpha[j]));
      const double temp = sqrtmu * rij;
      double u;
      if (temp < 0.01)
        u = TWOOVERSQRTPI * sqrtmu * (1.0 - 0.33333333333333333 * (temp * temp) + 0.1 * powi(temp, 4));
      else if (temp < 10.0)
        u = std::erf(temp) / rij;
      else
        u = 1.0 / rij;
      u = q[i] * q[j] * u;
      E = E + 2.0 * u;
    }
  }
  return E;
}

void orc_gauss_extent(int ng, const double *q, const double *alpha, double thres,
                      double *extent) {
  for (int i = 0; i < ng; ++i)
    extent[i] = std::sqrt(std::log(std::fabs(q[i]) * std::pow(alpha[i] / PI, 1.5) / thres) / alpha[i]);
}

}  // extern "C"
