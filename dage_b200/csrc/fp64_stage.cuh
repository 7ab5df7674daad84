// fp64_stage.cuh -- FP64 contraction stage on the FP64 tensor path (DMMA,
// mma.sync m8n8k4 f64), shared by the cube operator and the GBFMM near field.
//
//   out[o(R, n)] (= or +=) alpha * sum_K X[a(R) + K] * T[n * ldt + K]
//   a(R)    = (R % a_d0) a_s1 + (R / a_d0) a_s2
//   o(R, n) = (R % o_d0) o_s1 + (R / o_d0) o_s2 + n o_sn
//
// One descriptor describes one independent contraction (a whole cube stage,
// or one GBFMM box); a launch covers any number of them (grid.z).  Tiles are
// 128 x TN per 256-thread block (TN = 32, 64 or 128), 64 x TN/4 per warp
// (8 x TN/32 MMA tiles of 8 x 8), K in steps of 16 through a 3-deep
// cp.async ring.  Rows of both
// operands are K-contiguous but only 8-byte aligned, so the copies are
// 8 bytes wide; shared rows are padded to 20 doubles, which keeps the
// fragment loads free of bank conflicts.  An optional per-n-tile K range
// (first, last index) limits the K loop to the band of the matrix (entries
// outside it are below 2^-64 of their row's scale).  With accumulation each
// output element gets one correctly rounded FP64 add (an L2 reduction; one
// writer per element per launch).
#pragma once

#include "common.cuh"

namespace dage {

struct StageDesc {
  const double *X;
  long long a_d0, a_s1, a_s2;
  const double *T;
  long long ldt;
  double *out;
  long long o_d0, o_s1, o_s2, o_sn;
  int M, N, K;
  const int2 *krange;  // per 128-column tile: K band [first, last], or null
  long long t_ps;      // batched launches: T of t-point p is T + p * t_ps
  int kr_ps;           // ... and its K bands start at krange + p * kr_ps
  const double *wp;    // batched launches: alpha of t-point p is wp[p] (null: the argument)
};

constexpr int kFp64TileM = 128, kFp64TileN = 128;

// Contiguous cube stage: X[R * ldx + K], out[R + n * M].
inline StageDesc cube_stage(const double *X, long long ldx, int M, int N, int K, const double *T,
                            long long ldt, double *out, const int2 *krange) {
  StageDesc d{};
  d.X = X;
  d.a_d0 = M;
  d.a_s1 = ldx;
  d.a_s2 = 0;
  d.T = T;
  d.ldt = ldt;
  d.out = out;
  d.o_d0 = M;
  d.o_s1 = 1;
  d.o_s2 = 0;
  d.o_sn = M;
  d.M = M;
  d.N = N;
  d.K = K;
  d.krange = krange;
  return d;
}

// One contraction given by value; tn = tile width in n (32, 64 or 128).
int launch_fp64_stage(const StageDesc &d, double alpha, bool accumulate, cudaStream_t s,
                      int tn = kFp64TileN);
// ndesc contractions from a device array, with the matrices of t-point p;
// mtiles bounds the 128-row tile count and ncols the N of every descriptor.
int launch_fp64_stages(const StageDesc *d_descs, int ndesc, int mtiles, int ncols, int p,
                       double alpha, bool accumulate, cudaStream_t s, int tn = kFp64TileN);

// Sets the shared-memory limits of every stage kernel variant (done lazily by
// the launchers; call it before capturing launches into a CUDA graph).
int prepare_fp64_stages();

}  // namespace dage
