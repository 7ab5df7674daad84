// near_mixed.cuh -- the GBFMM near field in the fp16x3 split precision on the
// tensor cores (near_mixed.cu).
//
// The near field of a box is the cube operator restricted to the box's
// near-field input region (the box and its neighbours) and its owned output
// points, three "contract the fastest index and rotate" stages per t-point
// (gbfmm_coulomb3d.F90:933-1098 in the reference, FP64 there).  Here every
// box of every density of a set is one job of a grouped tcgen05 launch per
// (stage, t-point); the operands are FP16 two-part splits with the
// bound-based power-of-two scales of the cube operator's fp16x3 mode.
#pragma once

#include <vector>

#include "common.cuh"

namespace dage {

// Geometry of one GBFMM grid (plan): per axis, per box position, the near
// region (first point, points) and the owned output points, and the FP64
// near-field matrices T[pos][p][own][nq] with their K bands per (t-point,
// 128-row tile).
struct NearGeom {
  int npts[3] = {0, 0, 0};
  int P = 0;
  std::vector<int> q0[3], nq[3], own[3], p0[3];
  std::vector<const double *> T[3];
  std::vector<const int2 *> band[3];
};

// One box of a plan: its position along each axis.
struct NearBox {
  int pos[3];
};

struct NearF16Plan;  // FP16 matrix parts of one plan (built once)
struct NearF16Set;   // intermediates, tensor maps and job tables of n densities of one plan

int near_f16_plan_create(NearF16Plan **out, const NearGeom &geom, cudaStream_t s);
void near_f16_plan_destroy(NearF16Plan *p);

// n densities of one plan; tile width 64 or 128 output columns.  ws: null
// (the set allocates its intermediates) or three zero-initialised device
// buffers of at least near_f16_set_sizes bytes (split input, U, W) that
// sets running one after another on one stream may share.
int near_f16_set_create(NearF16Set **out, const NearF16Plan *plan, const std::vector<NearBox> &boxes,
                        int n, int tile_n, cudaStream_t s, void *const ws[3] = nullptr);
void near_f16_set_destroy(NearF16Set *s);
void near_f16_set_sizes(const NearF16Plan *plan, const std::vector<NearBox> &boxes, int n,
                        size_t bytes[3]);
size_t near_f16_set_bytes(const NearF16Plan *plan, const std::vector<NearBox> &boxes, int n);

// Binds device cubes and per-density t-point weights (device arrays of P
// doubles): uploads the job tables (synchronises the stream).
int near_f16_set_bind(NearF16Set *s, const double *const *rho, double *const *V,
                      const double *const *w, cudaStream_t st);

// Stream work of one near-field pass (no allocation, no host synchronisation;
// capturable): V_i (= on the first t-point group, then +=) near field of rho_i.
int near_f16_set_run(NearF16Set *s, cudaStream_t st);

// After the stream's work: DAGE_E_TIMEOUT if a kernel of the set gave up on
// an mbarrier wait (the flag is cleared), else 0.  Synchronises the stream.
int near_f16_set_check(NearF16Set *s, cudaStream_t st);

// Sets the kernels' shared-memory limits (before graph capture).
int near_f16_prepare();

}  // namespace dage
