// op3d.cuh -- internal state of a tensor-product cube operator handle and
// the kernel launchers shared by its FP64 and mixed-precision paths.
#pragma once

#include <vector>

#include "common.cuh"
#include "grid_host.h"

struct dage_op3d {
  int precision = DAGE_FP64;
  int device = 0;
  dage::Axis in[3], out[3];
  int nin[3] = {0, 0, 0}, nout[3] = {0, 0, 0};
  bool same_grid = false;

  // quadrature
  dage_quad quad{};
  int P = 0;
  std::vector<double> tp, tw, w;  // host copies; w = weights in use
  double coda = 0.0;

  // FP64 matrices, per axis: T[p][i_out][j_in] (row-major in j_in).  Axes
  // with identical input/output grids share one buffer (owner index).
  dage::DevBuf Tbuf[3];
  int Towner[3] = {0, 1, 2};
  // per axis owner: K band (first, last index, inclusive) of each t-point's
  // 128-row tiles, int2[P][ceil(n_out / 128)]
  dage::DevBuf band[3];
  const double *T(int axis) const { return Tbuf[Towner[axis]].as<double>(); }

  // per-point LIP integration weights of the output grid (energy)
  dage::DevBuf wts[3];
  dage::DevBuf d_w;          // weights w_p on the device
  dage::DevBuf d_rho, d_V;   // staging for host pointers
  dage::DevBuf tmp1, tmp2;   // intermediates of the FP64 path
  dage::DevBuf partials;     // energy reduction partial sums

  // FP64 path: contraction tile width (32, 64 or 128 output columns) of each
  // stage, from the autotuner (tune.h)
  int tile_n[3] = {128, 128, 128};
  bool from_cache = false;  // matrices read from an operator cache file

  // mixed-precision state (op3d_mixed.cu)
  void *mixed = nullptr;

  // per-kernel timing (dage_op3d_set_timing)
  static constexpr int kKinds = 3;
  bool timing = false;
  std::vector<cudaEvent_t> tev;          // event pool
  std::vector<std::pair<int, int>> tq;   // (kind, first event index) queued
  long long t_launches[kKinds] = {0, 0, 0};
  double t_ms[kKinds] = {0, 0, 0};
  int tmark_begin(int kind);             // returns slot or -1
  void tmark_end(int slot);
  int tcollect();                        // after stream sync

  // pipelined host-pointer applies (dage_op3d_apply_batched): two staging
  // slots, copy-in and copy-out streams beside the compute stream, per-slot
  // events ordering copy-in -> compute -> copy-out and the slots' reuse
  dage::DevBuf pipe_rho[2], pipe_V[2];
  cudaStream_t pipe_in = nullptr, pipe_out = nullptr;
  cudaEvent_t pipe_h2d[2] = {nullptr, nullptr}, pipe_comp[2] = {nullptr, nullptr},
              pipe_d2h[2] = {nullptr, nullptr};
  bool pipe_open = false;  // applies queued since the last pipeline wait

  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_ms = 0.0f;
};

namespace dage {

// FP64 "contract the fastest index and rotate" stage:
//   out[R + n*M] (= or +=) alpha * sum_K X[R*ldx + K] * T[n*ldt + K]
// krange (optional): per 128-column tile of out, the K band [first, last].
int launch_stage_fp64(const double *X, long long ldx, int M, int N, int K, const double *T,
                      long long ldt, double *out, double alpha, bool accumulate,
                      cudaStream_t s, const int2 *krange = nullptr, int tn = 128);

// K band of every (t-point, 128-row tile) of an axis matrix T[p][n][K]: the
// first and last K index holding an entry above 2^-64 of its row's scale.
int launch_band(const double *T, int K, int N, int P, int2 *range, cudaStream_t s);

// V += coda * rho (when coda != 0) and the LIP-weighted integral of
// f1 * f2 (f2 may be null: integral of f1).  The result lands in *d_result
// (device) after a deterministic two-pass reduction.
int launch_finalize(const double *f1, double *f2_or_V, const double *rho_for_coda,
                    double coda, const double *wx, const double *wy, const double *wz,
                    int nx, int ny, int nz, double *partials, int npartials,
                    double *d_result, cudaStream_t s);

int finalize_partials_count();

// Gauss-Legendre t-points/weights on the GPU (host copies + device tp).
int build_quadrature(const dage_quad &q, std::vector<double> &tp, std::vector<double> &tw,
                     DevBuf &d_tp, cudaStream_t s);
// FP64 operator matrix of one axis, T[p][i_out][j_in], for an input axis and
// arbitrary output coordinates (host array of n_out values).
int build_axis_matrix(const Axis &in, const double *out_points, int n_out, const double *d_tp,
                      int P, double *d_T, cudaStream_t s);

// bubbles -> device cube on a stream (bubbles.cu); coordinates on the device
int bubbles_inject_launch(const dage_bubbles *b, const double *xs, int nx, const double *ys,
                          int ny, const double *zs, int nz, int lmin, double factor,
                          double *d_cube, cudaStream_t s);

// mixed-precision path (op3d_mixed.cu)
int mixed_setup(dage_op3d *op);
int mixed_apply(dage_op3d *op, const double *d_rho, double *d_V, cudaStream_t s);
// the same in two halves: the launches, then (after any further work on s)
// the wait and the check of the kernels' timeout flag
int mixed_enqueue(dage_op3d *op, const double *d_rho, double *d_V, cudaStream_t s);
int mixed_check(dage_op3d *op, cudaStream_t s);
int mixed_set_weights(dage_op3d *op);
int mixed_tune(dage_op3d *op);
int mixed_schedule(const dage_op3d *op, int *ring_stages, int *group);
void mixed_destroy(dage_op3d *op);

}  // namespace dage
