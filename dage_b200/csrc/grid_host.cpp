// grid_host.cpp -- LIP basis and grid-axis metadata (see grid_host.h).
#include "grid_host.h"

#include <cmath>

#include "common.cuh"

namespace dage {

namespace {

// Gauss-Lobatto nodes on [left, right] for n = 6, 7 -- the only orders the
// reference defines (src/bubbles/gauss.F90:427-452).
bool lobatto(int n, double left, double right, double *x) {
  if (n == 6) {
    const double u = std::sqrt((7.0 + 2 * std::sqrt(7.0)) / 21.0);
    const double v = std::sqrt((7.0 - 2 * std::sqrt(7.0)) / 21.0);
    const double z[6] = {-1.0, -u, -v, v, u, 1.0};
    for (int i = 0; i < 6; ++i) x[i] = z[i];
  } else if (n == 7) {
    const double u = std::sqrt((15.0 + 2 * std::sqrt(15.0)) / 33.0);
    const double v = std::sqrt((15.0 - 2 * std::sqrt(15.0)) / 33.0);
    const double z[7] = {-1.0, -u, -v, 0.0, v, u, 1.0};
    for (int i = 0; i < 7; ++i) x[i] = z[i];
  } else {
    return false;
  }
  for (int i = 0; i < n; ++i) x[i] = 0.5 * ((right + left) + (right - left) * x[i]);
  return true;
}

}  // namespace

int make_lip_basis(int nlip, int grid_type, LipBasis &L) {
  if (nlip < 2 || nlip > 7)
    return fail(DAGE_E_UNSUPPORTED, "nlip=%d: supported LIP orders are 2..7", nlip);
  if (grid_type != 1 && grid_type != 2)
    return fail(DAGE_E_UNSUPPORTED, "grid_type=%d: 1 (equidistant) or 2 (Gauss-Lobatto)",
                grid_type);
  L.nlip = nlip;
  L.grid_type = grid_type;
  L.first = (double)(-((nlip - 1) / 2));
  L.last = (double)(nlip / 2);
  const int n = nlip;
  std::vector<double> nodes(n);
  if (grid_type == 1) {
    for (int i = 0; i < n; ++i) nodes[i] = (double)(i + 1 - (nlip + 1) / 2);
  } else if (!lobatto(n, L.first, L.last, nodes.data())) {
    return fail(DAGE_E_UNSUPPORTED, "Gauss-Lobatto cells exist for nlip 6 and 7 only");
  }
  // Build each basis polynomial as a product of (x - x_i)/(x_j - x_i),
  // coefficients in decreasing powers: c[k][j] multiplies x^(n-1-k).
  std::vector<double> c((size_t)n * n, 0.0), prev(n);
  for (int j = 0; j < n; ++j) c[(size_t)(n - 1) * n + j] = 1.0;
  for (int i = 0; i < n; ++i) {
    const double xi = nodes[i];
    for (int j = 0; j < n; ++j) {
      if (i == j) continue;
      const double dx = (grid_type == 1) ? (double)(j - i) : (nodes[j] - nodes[i]);
      for (int k = 0; k < n; ++k) prev[k] = c[(size_t)k * n + j];
      for (int k = 0; k < n - 1; ++k) c[(size_t)k * n + j] = (prev[k + 1] - prev[k] * xi) / dx;
      c[(size_t)(n - 1) * n + j] = -prev[n - 1] * xi / dx;
    }
  }
  L.coeff = c;
  // Integrals over [first, last] by Horner on the antiderivative.
  L.integrals.assign(n, 0.0);
  for (int j = 0; j < n; ++j) {
    double lo = 0.0, hi = 0.0;
    for (int k = 0; k < n; ++k) {
      const double ic = c[(size_t)k * n + j] / (double)(n - k);
      lo = (lo + ic) * L.first;
      hi = (hi + ic) * L.last;
    }
    L.integrals[j] = hi - lo;
  }
  return 0;
}

int make_axis(const dage_grid1d &g, Axis &ax) {
  if (g.ncell < 1 || !g.cell_scales)
    return fail(DAGE_E_INVALID, "grid axis needs ncell >= 1 and cell_scales");
  LipBasis L;
  DAGE_TRY(make_lip_basis(g.nlip, g.grid_type, L));
  ax.ncell = g.ncell;
  ax.nlip = g.nlip;
  ax.grid_type = g.grid_type;
  ax.qmin = g.qmin;
  ax.h.assign(g.cell_scales, g.cell_scales + g.ncell);
  for (double h : ax.h)
    if (!(h > 0.0)) return fail(DAGE_E_INVALID, "cell_scales must be positive");
  std::vector<double> tmpl(g.nlip - 1);
  if (g.grid_type == 1) {
    for (int k = 1; k < g.nlip; ++k) tmpl[k - 1] = (double)k;
  } else {
    std::vector<double> gl(g.nlip);
    lobatto(g.nlip, 0.0, (double)(g.nlip - 1), gl.data());
    for (int k = 1; k < g.nlip; ++k) tmpl[k - 1] = gl[k];
  }
  ax.points.assign(ax.n(), 0.0);
  ax.celld.assign(g.ncell, 0.0);
  size_t ip = 0;
  ax.points[0] = g.qmin;
  for (int c = 0; c < g.ncell; ++c) {
    ax.celld[c] = ax.points[ip];
    for (int k = 1; k < g.nlip; ++k) {
      ++ip;
      ax.points[ip] = ax.celld[c] + tmpl[k - 1] * ax.h[c];
    }
  }
  ax.weights.assign(ax.n(), 0.0);
  for (int c = 0; c < g.ncell; ++c)
    for (int i = 0; i < g.nlip; ++i)
      ax.weights[(size_t)c * (g.nlip - 1) + i] += L.integrals[i] * ax.h[c];
  return 0;
}

bool same_axis(const Axis &a, const Axis &b) {
  return a.ncell == b.ncell && a.nlip == b.nlip && a.grid_type == b.grid_type &&
         a.points == b.points;
}

}  // namespace dage
