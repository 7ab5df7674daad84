// expo.cuh -- the one-dimensional Gaussian-kernel integrals of the Coulomb
// operator matrices, evaluated in FP64 (host and device).
//
// I_n(a, b, t, p) = int_a^b x^n exp(-t^2 (x-p)^2) dx for n = 0..6, with the
// reference's two regimes (src/bubbles/exponentials.F90:647-666): for
// t < 0.1 a composite 12-point Gauss-Legendre rule on four sub-intervals
// (gauss_expo_n, exponentials.F90:2287-2429); otherwise closed forms in erf
// and exp (expo_0..expo_6, exponentials.F90:695-1297).  The closed forms are
// evaluated term by term in the order the reference writes them, because
// their cancellation pattern decides the last digits of the result.
#pragma once

#include <math.h>

#ifndef DAGE_HD
#define DAGE_HD __host__ __device__ __forceinline__
#endif

namespace dage {
namespace expo {

constexpr double kSqrtPi = 1.7724538509055160273;  // sqrt(acos(-1))

DAGE_HD double ipow(double x, int n) {  // x**n by repeated squaring
  unsigned m = (unsigned)n;
  double y = (m & 1u) ? x : 1.0;
  while (m >>= 1) {
    x = x * x;
    if (m & 1u) y = y * x;
  }
  return y;
}

DAGE_HD double s4(double q) { return q + q * q / 2.0 + q * q * q / 6.0 + q * q * q * q / 24.0; }
DAGE_HD double s4one(double q) {
  return 1.0 + q + q * q / 2.0 + q * q * q / 6.0 + q * q * q * q / 24.0;
}

DAGE_HD double i0(double a, double b, double t, double p) {
  if (t == 0.0 || t < 1.0e-06) return b - a;
  return kSqrtPi * (erf(b * t - t * p) - erf(a * t - t * p)) / t / 2.0;
}

DAGE_HD double i1(double a, double b, double t, double p) {
  if (t == 0.0 || t < 1.0e-06) return (b * b - a * a) / 2.0;
  const double v1 = p * kSqrtPi * erf(t * (b - p));
  double v2;
  if (t > 1.0e-03) {
    v2 = (exp(-(t * t) * ((a - p) * (a - p))) - exp(-(t * t) * ((b - p) * (b - p)))) / t;
  } else {
    const double q = -(t * t) * ((a - p) * (a - p));
    const double r = -(t * t) * ((b - p) * (b - p));
    v2 = (q + q * q / 2.0 + q * q * q / 6.0 + q * q * q * q / 24.0 - r - r * r / 2.0 -
          r * r * r / 6.0 - r * r * r * r / 24.0) /
         t;
  }
  const double v3 = -p * kSqrtPi * erf(a * t - t * p);
  return (v1 + v2 + v3) / t / 2.0;
}

DAGE_HD double i2(double a, double b, double t, double p) {
  if (t == 0.0 || t < 0.5e-04) return (b * b * b - a * a * a) / 3.0;
  const double v1 = p * p * kSqrtPi * erf(b * t - t * p) / 2.0;
  double v2, v3;
  if (t > 1.0e-03) {
    const double ea = exp(-(t * t * ((a - p) * (a - p))));
    const double eb = exp(-(t * t * ((b - p) * (b - p))));
    v2 = ea * a - eb * b;
    v3 = (ea - eb) * p / t / 2.0;
  } else {
    const double q = -(t * t * ((a - p) * (a - p)));
    const double r = -(t * t * ((b - p) * (b - p)));
    v2 = s4(q) * a - s4(r) * b;
    v2 = v2 + a - b;
    v3 = (s4(q) - s4(r)) * p / t / 2.0;
  }
  double v5 = kSqrtPi * (erf(t * (b - p)) - erf(t * (a - p))) / t / 2.0;
  v2 = (v2 + v5) / t / 2.0;
  v5 = 0.0;
  const double v4 = -(p * p) * kSqrtPi * erf(a * t - t * p) / 2.0;
  return (v1 + v2 + v3 + v4 + v5) / t;
}

DAGE_HD double i3(double a, double b, double t, double p) {
  if (t == 0.0 || t < 1.0e-04) return (ipow(b, 4) - ipow(a, 4)) / 4.0;
  double v1, v2, v3, v5;
  if (t > 1.0e-03) {
    const double ea = exp(-(t * t) * ((a - p) * (a - p)));
    const double eb = exp(-(t * t) * ((b - p) * (b - p)));
    v1 = 2.0 * (ea * (a * a) - eb * (b * b)) / (t * t);
    v2 = 2.0 * p * (a * ea - b * eb) * t;
    v3 = 2.0 * (ea * (p * p) - eb * (p * p)) / (t * t);
    v5 = 2.0 * (ea - eb) / t;
  } else {
    const double q = -(t * t * ((a - p) * (a - p)));
    const double r = -(t * t * ((b - p) * (b - p)));
    v1 = 2.0 * (s4one(q) * a * a - s4one(r) * b * b) / t / t;
    v2 = 2.0 * ((s4(q) * a - s4(r) * b) + a - b) * p * t;
    v3 = 2.0 * (s4(q) - s4(r)) * p * p / t / t;
    v5 = 2.0 * (s4(q) - s4(r)) / t;
  }
  const double d = erf(b * t - t * p) - erf(a * t - t * p);
  const double v4 = 2.0 * ipow(p, 3) * kSqrtPi * d / t;
  double v6 = 3.0 * p * kSqrtPi * d;
  v6 = (v6 + v2 + v5) / t / t / t;
  v2 = 0.0;
  v5 = 0.0;
  return 0.25 * (v1 + v2 + v3 + v4 + v5 + v6);
}

DAGE_HD double i4(double a, double b, double t, double p) {
  if (t == 0.0 || t < 1.0e-03) return (ipow(b, 5) - ipow(a, 5)) / 5.0;
  double v1, v2, v3, v4, v7, v8;
  {
    // t >= 1e-3 here, so only the closed-form branch of expo_4 is reachable
    // (its series branch needs t <= 1e-3 < threshold).
    const double ea = exp(-(t * t) * ((a - p) * (a - p)));
    const double eb = exp(-(t * t) * ((b - p) * (b - p)));
    if (t > 1.0e-03) {
      v1 = 4.0 * (ea * ipow(a, 3) - eb * ipow(b, 3));
      v2 = 4.0 * (ea * p * (a * a) - eb * p * (b * b));
      v3 = 4.0 * (ea * (p * p) * a - eb * (p * p) * b);
      v4 = 4.0 * (ea * ipow(p, 3) - eb * ipow(p, 3));
      v7 = 10.0 * p * (ea - eb) / t / t;
      v8 = 6.0 * (ea * a - eb * b);
    } else {
      const double q = -(t * t * ((a - p) * (a - p)));
      const double r = -(t * t * ((b - p) * (b - p)));
      v1 = 4.0 * (s4one(q) * ipow(a, 3) - s4one(r) * ipow(b, 3));
      v2 = 4.0 * (s4one(q) * p * a * a - s4one(r) * p * b * b);
      v3 = 4.0 * (s4one(q) * p * p * a - s4one(r) * p * p * b);
      v4 = 4.0 * (s4(q) - s4(r)) * ipow(p, 3);
      v7 = 10.0 * (s4(q) - s4(r)) * p / t / t;
      v8 = 6.0 * (s4one(q) * a - s4one(r) * b);
    }
  }
  const double d = erf(a * t - t * p) - erf(b * t - t * p);
  double v5 = -(4.0 * t * ipow(p, 4) * kSqrtPi * d);
  double v6 = -(12.0 / t * (p * p) * kSqrtPi * d);
  double v9 = -(3.0 * kSqrtPi * d / t);
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

DAGE_HD double i5(double a, double b, double t, double p) {
  if (t == 0.0 || t < 2.5e-03) return (ipow(b, 6) - ipow(a, 6)) / 6.0;
  const double t2 = t * t;
  double v1, v2, v3, v4, v5, v8, v9, v11, v12;
  if (t > 1.0e-02) {
    const double ea = exp(-t2 * ((a - p) * (a - p)));
    const double eb = exp(-t2 * ((b - p) * (b - p)));
    v1 = 4.0 * (ea * ipow(a, 4) - eb * ipow(b, 4));
    v2 = 4.0 * (ea * p * ipow(a, 3) - eb * p * ipow(b, 3));
    v3 = 4.0 * (ea * (p * p) * (a * a) - eb * (p * p) * (b * b));
    v4 = 4.0 * (ea * ipow(p, 3) * a - eb * ipow(p, 3) * b);
    v5 = 4.0 * (ea * ipow(p, 4) - eb * ipow(p, 4));
    v8 = 18.0 * (ea - eb) * (p * p) / t2;
    v9 = 14.0 * (ea * p * a - eb * p * b) / t2;
    v11 = 8.0 * (ea * (a * a) - eb * (b * b)) / t2;
    v12 = 8.0 * (ea - eb) / ipow(t, 4);
  } else {
    const double q = -(t * t * ((a - p) * (a - p)));
    const double r = -(t * t * ((b - p) * (b - p)));
    v1 = 4.0 * (s4one(q) * ipow(a, 4) - s4one(r) * ipow(b, 4));
    v2 = 4.0 * (s4one(q) * p * ipow(a, 3) - s4one(r) * p * ipow(b, 3));
    v3 = 4.0 * (s4one(q) * (p * p) * (a * a) - s4one(r) * (p * p) * (b * b));
    v4 = 4.0 * (s4one(q) * ipow(p, 3) * a - s4one(r) * ipow(p, 3) * b);
    v5 = 4.0 * (s4(q) * ipow(p, 4) - s4(r) * ipow(p, 4));
    v8 = 18.0 * ((s4(q) - s4(r)) * (p * p) / t2);
    v9 = 14.0 * ((s4one(q) * a * p - s4one(r) * b * p) / t2);
    v11 = 8.0 * ((s4one(q) * a * a - s4one(r) * b * b) / t2);
    v12 = 8.0 * ((s4(q) - s4(r)) / ipow(t, 4));
  }
  const double d = erf(a * t - t * p) - erf(b * t - t * p);
  const double v6 = -(4.0 * t * ipow(p, 5) * kSqrtPi * d);
  const double v7 = -(20.0 / t * ipow(p, 3) * kSqrtPi * d);
  const double v10 = -(15.0 * p * kSqrtPi * d / ipow(t, 3));
  double value = v1 + v2 + v3 + v4 + v5 + v6;
  value = value + v7 + v8 + v9 + v10 + v11 + v12;
  value = value / t2;
  return 0.125 * value;
}

DAGE_HD double i6(double a, double b, double t, double p) {
  if (t == 0.0 || t < 5.0e-03) return (ipow(b, 7) - ipow(a, 7)) / 7.0;
  const double ea = exp(-(t * t) * ((a - p) * (a - p)));
  const double eb = exp(-(t * t) * ((b - p) * (b - p)));
  const double d = erf(b * t - t * p) - erf(a * t - t * p);
  double v1 = 30.0 * (ea * a - eb * b);
  double v2 = 15.0 * kSqrtPi * d;
  v1 = (v1 + v2 / t) / t / t / t;
  v2 = 0.0;
  const double v3 = 90.0 * (p * p) * kSqrtPi * d / t / t;
  const double v4 = 56.0 * (ea - eb) * ipow(p, 3) / t;
  const double v5 = 66.0 * (ea - eb) * p / t / t / t;
  const double v6 = 8.0 * (ea - eb) * ipow(p, 5) * t;
  const double v7 = 20.0 * (ea * ipow(a, 3) - eb * ipow(b, 3)) / t;
  const double v8 = 36.0 * (ea * (a * a) - eb * (b * b)) * p / t;
  const double v9 = 48.0 * (ea * a - eb * b) * (p * p) / t;
  const double v10 = 8.0 * ipow(p, 6) * kSqrtPi * d * (t * t);
  const double v11 = 8.0 * (ea * ipow(a, 4) - eb * ipow(b, 4)) * p * t;
  const double v12 = 8.0 * (ea * ipow(a, 3) - eb * ipow(b, 3)) * (p * p) * t;
  const double v13 = 8.0 * (ea * ipow(a, 5) - eb * ipow(b, 5)) * t;
  const double v14 = 8.0 * (ea * a - eb * b) * ipow(p, 4) * t;
  const double v15 = 8.0 * (ea * (a * a) - eb * (b * b)) * ipow(p, 3) * t;
  const double v16 = 60.0 * ipow(p, 4) * kSqrtPi * d;
  double value = v1 + v2 + v3 + v4 + v5 + v6 + v7 + v8;
  value = value + v9 + v10 + v11 + v12 + v13 + v14 + v15 + v16;
  value = value / ipow(t, 3);
  return 0.0625 * value;
}

// Composite 12-point Gauss-Legendre rule; nodes and weights to the 15
// digits the reference writes (exponentials.F90:2370-2394).
DAGE_HD double gauss_rule(double a, double b, double t, double p, int n) {
  constexpr double W[6] = {0.047175336386512, 0.106939325995318, 0.160078328543346,
                           0.203167426723066, 0.233492536538355, 0.249147045813403};
  constexpr double X[6] = {0.981560634246719, 0.904117256370475, 0.769902674194305,
                           0.587317954286617, 0.367831498998180, 0.125233408511469};
  if (t == 0.0) {
    if (n == 0) return b - a;
    return (ipow(b, n + 1) - ipow(a, n + 1)) / (n + 1);
  }
  double limit[5];
#pragma unroll
  for (int i = 1; i <= 5; ++i) limit[i - 1] = ((5 - i) * a + (i - 1) * b) / 4;
  double summa = 0.0;
  for (int i = 0; i < 4; ++i) {
    const double a0 = limit[i], a1 = limit[i + 1];
    const double pr = 1.0 - a1 * 2.0 / (a1 - a0);
    const double qr = 2.0 / (a1 - a0);
#pragma unroll
    for (int j = 0; j < 12; ++j) {
      const double xk = (j < 6) ? -X[j] : X[11 - j];
      const double wk = (j < 6) ? W[j] : W[11 - j];
      const double tp = (xk - pr) / qr;
      const double tw = wk / qr;
      const double e = exp(-(t * t * (tp - p) * (tp - p)));
      if (n > 0)
        summa = summa + ipow(tp, n) * e * tw;
      else
        summa = summa + e * tw;
    }
  }
  return summa;
}

DAGE_HD double closed_form(double a, double b, double t, double p, int n) {
  switch (n) {
    case 0: return i0(a, b, t, p);
    case 1: return i1(a, b, t, p);
    case 2: return i2(a, b, t, p);
    case 3: return i3(a, b, t, p);
    case 4: return i4(a, b, t, p);
    case 5: return i5(a, b, t, p);
    default: return i6(a, b, t, p);
  }
}

// values[n-1-i] = I_i(a, b, t, p), i = 0..n-1 (highest power first).
DAGE_HD void integrals(double a, double b, double t, double p, int n, double *values) {
  if (t < 0.1) {
    for (int i = 0; i < n; ++i) values[n - 1 - i] = gauss_rule(a, b, t, p, i);
  } else {
    for (int i = 0; i < n; ++i) values[n - 1 - i] = closed_form(a, b, t, p, i);
  }
}

}  // namespace expo
}  // namespace dage
