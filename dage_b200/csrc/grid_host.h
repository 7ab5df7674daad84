// grid_host.h -- grid metadata on the host: LIP basis polynomials, grid
// point coordinates and LIP integration weights of one axis.  These are the
// inputs the GPU kernels consume (they describe the grid; no operator work
// happens here).
#pragma once

#include <vector>

#include "../../include/dage_gpu.h"

namespace dage {

struct LipBasis {
  int nlip = 0;
  int grid_type = 0;
  double first = 0.0, last = 0.0;
  // coeff[k * nlip + j]: coefficient of x^(nlip-1-k) of basis polynomial j
  // (src/bubbles/lip.F90:285-362, decreasing powers).
  std::vector<double> coeff;
  std::vector<double> integrals;  // int_first^last of each polynomial
};

struct Axis {
  int ncell = 0, nlip = 0, grid_type = 0;
  double qmin = 0.0;
  std::vector<double> h;       // cell step lengths
  std::vector<double> celld;   // cell start coordinates
  std::vector<double> points;  // ncell*(nlip-1)+1 coordinates
  std::vector<double> weights; // LIP integration weight of every point
  int n() const { return ncell * (nlip - 1) + 1; }
};

// LIPBasisInit + LIPBasis_coeffs + LIPBasis_integrals
// (src/bubbles/lip.F90:118-141, 285-411).  Returns 0 or DAGE_E_*.
int make_lip_basis(int nlip, int grid_type, LipBasis &out);

// Grid1D_init_step (src/bubbles/grid.F90:446-534) plus the per-point
// integration weights used by the reference Integrator
// (src/bubbles/evaluators.F90:1023-1098).
int make_axis(const dage_grid1d &g, Axis &out);

bool same_axis(const Axis &a, const Axis &b);

}  // namespace dage
