/*
 * dage_gpu.h -- C ABI of the B200-native grid-based Coulomb/Helmholtz
 * operator path (libdagegpu.so).
 *
 * Conventions shared by every entry point
 *  - Cubes are Fortran column-major cube(x, y, z), x fastest, FP64, exactly
 *    as the reference's Function3D cubes (src/bubbles/function3d.F90:86-190).
 *  - Pointers are host pointers unless the call takes a flags word with
 *    DAGE_DEVICE_PTRS set, in which case they are device pointers on the
 *    device that was current when the handle was created.
 *  - Every function returns 0 on success and a negative DAGE_E_* code on
 *    failure; dage_last_error() then returns a message for the calling
 *    thread.  No function prints or exits (the reference prints and calls
 *    exit(-1), src/bubbles/cuda_blas.cu:36-47).
 *  - A handle owns its CUDA stream and device buffers.  Calls on distinct
 *    handles may run concurrently from different host threads; calls on one
 *    handle must be serialised by the caller.
 *  - Indices are 0-based.
 */
#ifndef DAGE_GPU_H
#define DAGE_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DAGE_ABI_VERSION 1

/* status codes */
#define DAGE_OK 0
#define DAGE_E_INVALID (-1)   /* bad argument (null pointer, bad shape) */
#define DAGE_E_CUDA (-2)      /* a CUDA runtime/driver call failed */
#define DAGE_E_NOMEM (-3)     /* device allocation failed */
#define DAGE_E_UNSUPPORTED (-4)
#define DAGE_E_TIMEOUT (-5)   /* a bounded device-side wait ran out */

/* flags for apply-style calls */
#define DAGE_DEVICE_PTRS 1u   /* input/output pointers are device pointers */
#define DAGE_ENERGY 2u        /* also return the integral of rho * V */
#define DAGE_NO_CODA 4u       /* skip the coda term for this call */
#define DAGE_ACCUMULATE 8u    /* V += result instead of V = result */
#define DAGE_NO_GRAPH 16u     /* batch apply: launch the pipeline directly, no CUDA graph */
#define DAGE_PRODUCT_COMPLETE 32u /* bubble product: also the terms the reference table omits */
#define DAGE_TAYLOR_EXACT 64u     /* Taylor bubbles: the true series (1/kappa!, exact harmonic
                                     expansion) instead of the reference's */
#define DAGE_TAYLOR_IGNORE_BUBBLES 128u /* Taylor bubbles: leave out the other atoms' bubbles */

/* operator precisions */
#define DAGE_FP64 0            /* FP64 everywhere: the drop-in */
#define DAGE_MIXED_BF16X3 1    /* 2-way BF16 splits, 3 products, FP32 accum */
#define DAGE_MIXED_BF16X6 2    /* 3-way BF16 splits, 6 products, FP32 accum */
#define DAGE_MIXED_FP16X3 3    /* 2-way FP16 splits with power-of-two stage scales,
                                  3 products, FP32 accum with the toward-zero
                                  rounding bias removed */

/* One axis of a Grid3D: ncell LIP cells of nlip points each; the axis holds
 * ncell*(nlip-1)+1 points (src/bubbles/grid.F90:446-534, Grid1D_init_step).
 * grid_type 1 = equidistant points in a cell, 2 = Gauss-Lobatto points. */
typedef struct dage_grid1d {
  int ncell;
  int nlip;
  int grid_type;
  double qmin;
  const double *cell_scales; /* ncell host values (step length per cell) */
} dage_grid1d;

/* GaussQuad parameters (src/bubbles/gauss.F90:55-122): nlin Gauss-Legendre
 * t-points on [tstart, tlin] and nlog log-mapped points on [tlin, tlog]. */
typedef struct dage_quad {
  int nlin;
  int nlog;
  double tstart;
  double tlin;
  double tlog;
} dage_quad;

typedef struct dage_op3d dage_op3d;

/* ---------------------------------------------------------------------------
 * Tensor-product cube operator (Coulomb3D / Helmholtz3D cube part)
 * ------------------------------------------------------------------------ */

/* Builds the operator on the current CUDA device: quadrature, weights
 * w_p = 2/sqrt(pi) tw_p, coda = pi/tlog^2, and the per-axis matrices
 * T_p(i_out, j_in), all in FP64 on the GPU.
 * Replaces Coulomb3D_init_explicit_sub + make_Coulomb3D_matrices
 * (src/bubbles/coulomb.F90:109-176, src/bubbles/exponentials.F90:602-639)
 * and Operator3D_cuda_init (src/bubbles/function3d.F90:4172-4209). */
int dage_op3d_create(const dage_grid1d grid_in[3], const dage_grid1d grid_out[3],
                     const dage_quad *quad, int precision, dage_op3d **op);

/* Applies the operator to one cube: V = sum_p w_p (T^x_p (x) T^y_p (x) T^z_p)
 * rho [+ coda * rho when the input and output grids coincide].  With
 * DAGE_ENERGY, *energy receives the LIP-weighted integral of rho*V over the
 * output grid (FP64).  rho and V may be host or device pointers (flags).
 * Replaces Operator3D_operator_cube's CUDA branch and
 * Operator3D_transform_cuda_cube (src/bubbles/function3d.F90:3795-3882,
 * 4354-4480); the coda follows the CPU branch (function3d.F90:4327-4332). */
int dage_op3d_apply(dage_op3d *op, const double *rho, double *V, unsigned flags,
                    double *energy);

/* n applies queued back to back (each as dage_op3d_apply with the same
 * flags) on their operators' streams, with one wait per distinct operator at
 * the end: applies on distinct operators overlap.  With host pointers each
 * operator pipelines its applies through two device staging slots and
 * copy-in/copy-out streams, so one density's copies overlap the neighbouring
 * densities' compute (asynchronously when the host arrays are pinned); the
 * slots are two input and two output cubes of device memory per operator,
 * allocated on its first host-pointer batch and held until it is destroyed.
 * energies[i] receives apply i's energy with DAGE_ENERGY.  An operator's
 * last_time_ms covers its last apply of the batch (host pointers: the whole
 * pipeline, first copy-in to last copy-out).  Replaces the per-orbital loop
 * of operate calls with Operator3D_transform_cuda_cube
 * (src/bubbles/function3d.F90:4354-4480). */
int dage_op3d_apply_batched(int n, dage_op3d *const *ops, const double *const *rho,
                            double *const *V, unsigned flags, double *energies);

/* Replaces the quadrature weights (length P = nlin+nlog).
 * Operator3D%set_transformation_weights, used by Helmholtz3D_set_energy
 * (src/bubbles/helmholtz3d.F90:411-444). */
int dage_op3d_set_weights(dage_op3d *op, int P, const double *w);

/* Helmholtz weights w_p = 2/sqrt(pi) tw_p exp(2E/(4 t_p^2)) for E < -0.005,
 * else the Coulomb weights (src/bubbles/helmholtz3d.F90:411-444). */
int dage_op3d_set_energy(dage_op3d *op, double energy);

/* Sets the coda coefficient (coulomb.F90:151 sets pi/tlog^2; 0 disables). */
int dage_op3d_set_coda(dage_op3d *op, double coda);

/* Uses the caller's cudaStream_t for all later work of this handle
 * (NULL restores the handle's own stream). */
int dage_op3d_set_stream(dage_op3d *op, void *stream);

/* Number of t-points and the t-points/weights in use (host copies). */
int dage_op3d_get_quadrature(const dage_op3d *op, int *P, double *tp, double *w);

/* Copies the FP64 matrix of one axis (0=x,1=y,2=z), layout T(i_out, j_in, p)
 * column-major, n_out*n_in*P values, to host memory. */
int dage_op3d_get_matrix(const dage_op3d *op, int axis, double *T_host);

/* Milliseconds of device time of the last apply (CUDA events). */
int dage_op3d_last_time_ms(const dage_op3d *op, float *ms);

/* Per-kernel device timing of later applies: with timing enabled, every
 * kernel launch of an apply is bracketed by CUDA events on the handle's
 * stream and its duration is added to a per-kind total.
 * kind: 0 = contraction stage kernel, 1 = precision split of the input,
 * 2 = finalize (coda + energy).  get_timing returns totals since enabling. */
int dage_op3d_set_timing(dage_op3d *op, int enable);
int dage_op3d_get_timing(const dage_op3d *op, int kind, long long *launches, double *ms);

/* As dage_op3d_create, with an on-disk cache of the operator matrices keyed by
 * (input grids, output grids, quadrature): when cache_dir holds a file with
 * this key (op3d_<hash>.bin), the FP64 matrices are read from it instead of
 * being built on the GPU; otherwise they are built and the file is written.
 * *from_cache (may be NULL) tells which happened.  The file layout follows
 * the reference's stream dump of grids (store_Grid1Ds / resume_Grid1Ds,
 * src/bubbles/grid.F90:2024-2068) for its key.  The GPU build takes ~5-60 ms
 * for the largest operators, so the cache serves callers that reuse
 * operators across processes rather than speed. */
int dage_op3d_create_cached(const dage_grid1d grid_in[3], const dage_grid1d grid_out[3],
                            const dage_quad *quad, int precision, const char *cache_dir,
                            int *from_cache, dage_op3d **op);

/* Tile widths (32, 64 or 128 output columns) the autotuner chose for the three
 * FP64 contraction stages (the split-precision stages use 128).  No reference
 * counterpart: the reference's stages are cuBLAS DGEMMs. */
int dage_op3d_tiles(const dage_op3d *op, int tile_n[3]);
/* The schedule of a split-precision operator's tensor-core stages: the
 * TMA/MMA ring stages the autotuner chose (4 or 6) and the t-points summed
 * per pass of the last stage (min(P, 8) unless a tune-cache entry sets it).
 * DAGE_E_INVALID for an FP64 operator.  No reference counterpart. */
int dage_op3d_mixed_schedule(const dage_op3d *op, int *ring_stages, int *tpoint_group);
int dage_op3d_destroy(dage_op3d *op);

/* ---------------------------------------------------------------------------
 * GBFMM Coulomb operator (GBFMMCoulomb3D, FP64)
 * ------------------------------------------------------------------------ */
typedef struct dage_gbfmm dage_gbfmm;

/* Builds the operator for a grid split into 2^maxlevel boxes per axis:
 * near-field sub-operator matrices (quadrature `quad`, the reference's
 * default for the near field is GaussQuad(25, 25)), box geometry, local
 * far-field lists of every level and the M2L matrices of all box
 * displacements, and for maxlevel >= 3 the M2M/L2L translation matrices, on
 * the GPU.  maxlevel 2..5 (the reference default is 2: 4x4x4 boxes, whose
 * local far field needs no M2M/L2L; deeper levels run the upward M2M pass,
 * M2L at every level and the downward L2L pass of gbfmm_coulomb3d.F90:
 * 650-905, 1502-1621); lmax <= 15.  precision: DAGE_FP64 (the drop-in) or
 * DAGE_MIXED_FP16X3: the near field on the tensor cores in the FP16 split
 * precision of the cube operator (one grouped tcgen05 launch over all boxes
 * per contraction stage and t-point), the far field in FP64.  Boxes take
 * ncell/2^maxlevel cells per axis; when that does not divide, the first
 * ncell mod 2^maxlevel boxes along the axis take one cell more, and a box
 * of a coarser level is the union of its children.  The Helmholtz kernel
 * (dage_gbfmm_set_energy with E < 0) runs at every maxlevel and in the
 * adaptive mode: M2M by the reference's Helmholtz multipole translator
 * (gbfmm_helmholtz3d.F90:598-601, 1223-1278), L2L by the transposed relation
 * that M2M implies (the reference has no Helmholtz L2L).
 * Replaces GBFMMCoulomb3D_init + init_nearfield + init_interaction_matrices
 * and gbfmmcoulomb3d_init_cuda (src/gbfmm/gbfmm_coulomb3d.F90:331-508,
 * 1313-1438; src/gbfmm/gbfmm_coulomb3d.cu:583-600). */
int dage_gbfmm_create(const dage_grid1d grid[3], int maxlevel, int lmax, const dage_quad *quad,
                      int precision, dage_gbfmm **g);

/* As dage_gbfmm_create, in the reference's adaptive mode (GBFMMCoulomb3D_init
 * with adaptive_mode, src/gbfmm/gbfmm_coulomb3d.F90:374-384; far-field lists
 * of gbfmm_coulomb3d.F90:1386-1433 with GBFMMParallelInfo evaluation types 1
 * and 2, src/gbfmm/gbfmm_parallel_info.F90:827-983): multipoles are
 * translated up to level 1; a box of level l >= 2 takes M2L from the children
 * of its parent's neighbours that contain one of its nearest neighbours
 * (minus those neighbours) and, as whole boxes of level l - 1, from its
 * parent's other neighbours.  Coulomb and Helmholtz kernels. */
int dage_gbfmm_create_adaptive(const dage_grid1d grid[3], int maxlevel, int lmax,
                               const dage_quad *quad, int precision, dage_gbfmm **g);

/* V = near field + far field (multipoles -> M2L -> L2P), every point taking
 * the contributions of the box that owns it; optional LIP-weighted energy.
 * Replaces GBFMMCoulomb3D_calculate_potential's CUDA path
 * (src/gbfmm/gbfmm_coulomb3d.F90:650-819). */
int dage_gbfmm_apply(dage_gbfmm *g, const double *rho, double *V, unsigned flags,
                     double *energy);

/* Multipole moments of every box, host array (N_lm, nbox) column-major with
 * lm = l(l+1)+m and boxes in the reference's octree order.  Replaces
 * gbfmmcoulomb3d_calculate_multipole_moments_cuda + _download_multipole_
 * moments_cuda (src/gbfmm/gbfmm_coulomb3d.cu:620-640). */
int dage_gbfmm_multipole_moments(dage_gbfmm *g, const double *rho, unsigned flags,
                                 double *moments);

/* Local expansions (N_lm, nbox) of the last apply (the far-field potential
 * coefficients, GBFMMFunction3D%farfield_potential). */
int dage_gbfmm_local_expansions(dage_gbfmm *g, double *L);

/* V += sum_lm L_lm S_lm(r - c_box) over every box's points for host local
 * expansions (N_lm, nbox).  Replaces gbfmmcoulomb3d_evaluate_potential_le_cuda
 * (src/gbfmm/gbfmm_coulomb3d.cu:641-660). */
int dage_gbfmm_evaluate_le(dage_gbfmm *g, const double *local_expansions, double *V,
                           unsigned flags);

int dage_gbfmm_box_count(const dage_gbfmm *g, int *nbox, int *nlm);
/* GBFMMHelmholtz3D_set_energy (src/gbfmm/gbfmm_helmholtz3d.F90:478-516): energy < 0
 * switches the operator to the Helmholtz kernel e^(-kappa r)/r, kappa = sqrt(-2 energy):
 * near-field weights times e^(2E/(4 t_p^2)) (when E < -0.005), multipoles and local
 * expansions with modified spherical Bessel functions, the Helmholtz
 * multipole-to-local converter (src/bubbles/helmholtz_multipole_tools.F90:172-511).
 * energy = 0 returns to the Coulomb kernel. */
int dage_gbfmm_set_energy(dage_gbfmm *g, double energy);
/* Tile widths (32, 64 or 128 columns) the plan's autotuner chose for the
 * three near-field contraction stages (no reference counterpart: the
 * reference issues one cuBLAS call per box). */
int dage_gbfmm_tiles(const dage_gbfmm *g, int tile_n[3]);
int dage_gbfmm_set_stream(dage_gbfmm *g, void *stream);
int dage_gbfmm_last_time_ms(const dage_gbfmm *g, float *ms);
int dage_gbfmm_destroy(dage_gbfmm *g);

/* ---------------------------------------------------------------------------
 * Batched GBFMM: many independent densities of any grid sizes
 * ------------------------------------------------------------------------ */
/* Replaces the reference's per-density loop over GBFMMCoulomb3D_calculate_potential
 * (src/gbfmm/gbfmm_coulomb3d.F90:650-819) when many orbitals/densities are
 * operated on in one SCF step.  Densities on equal grids share one plan
 * (boxes, near-field matrices, M2L matrices); every pipeline stage
 * (moments, M2L, near field per t-point and contraction stage, L2P, energy)
 * is one launch over all densities.  The near field's intermediates are
 * processed in chunks of densities that fit near_budget_bytes (0 = 8 GiB).
 * grids holds 3 axes per density.  precision: DAGE_FP64 or DAGE_MIXED_FP16X3
 * (near field on the tensor cores; the chunks then share one workspace). */
typedef struct dage_gbfmm_batch dage_gbfmm_batch;
typedef struct dage_bubbles dage_bubbles;
int dage_gbfmm_batch_create(int n, const dage_grid1d *grids, int maxlevel, int lmax,
                            const dage_quad *quad, int precision, size_t near_budget_bytes,
                            dage_gbfmm_batch **out);
/* rho[i], V[i]: cube i (host arrays, or device pointers with DAGE_DEVICE_PTRS);
 * energies[n] receives each int rho V with DAGE_ENERGY.  The pipeline is
 * captured into a CUDA graph for the set of device cubes it runs on and
 * replayed while later calls use the same cubes (host-array calls always
 * use the batch's own device cubes); DAGE_NO_GRAPH launches it directly.
 * The near-field tile widths are autotuned on the first call. */
int dage_gbfmm_batch_apply(dage_gbfmm_batch *b, const double *const *rho, double *const *V,
                           unsigned flags, double *energies);
/* Per-density kernel (as dage_gbfmm_set_energy): energies[i] < 0 gives density i
 * the Helmholtz kernel e^(-kappa r)/r, kappa = sqrt(-2 energies[i]); 0 the Coulomb
 * kernel (the default).  Densities with equal grids and energies share matrices. */
int dage_gbfmm_batch_set_energies(dage_gbfmm_batch *b, const double *energies);
/* Optional first stage of the batch pipeline (the SCF step's inject -> near field ->
 * moments -> M2L -> evaluate, all in the one graph): rho_i += factors[i] * bubbles
 * (from lmin) on density i's grid, in place, before the operator runs; factors[i] = 0
 * skips density i; bubbles = NULL removes the stage.  The bubbles object must outlive
 * the batch's use of it. */
int dage_gbfmm_batch_set_bubbles(dage_gbfmm_batch *b, const dage_bubbles *bubbles,
                                 const double *factors, int lmin);
int dage_gbfmm_batch_info(const dage_gbfmm_batch *b, int *nplans, int *nchunks, int tile_n[3],
                          long long *graph_nodes);
int dage_gbfmm_batch_set_stream(dage_gbfmm_batch *b, void *stream);
int dage_gbfmm_batch_last_time_ms(const dage_gbfmm_batch *b, float *ms);
int dage_gbfmm_batch_destroy(dage_gbfmm_batch *b);

/* ---------------------------------------------------------------------------
 * Bubbles -> cube injection
 * ------------------------------------------------------------------------ */

/* Uploads a bubble set: natom centres (3*natom), one radial LIP grid per atom
 * (equidistant-point cells starting at r = 0; any cell steps), lmax <= 12,
 * the r^k exponent k >= 0, and the radial values f: per atom (lmax+1)^2 rows
 * (lm = l(l+1)+m) of that atom's grid points, atoms concatenated.  The LIP
 * values are turned into per-cell monomial coefficients on the GPU.
 * Replaces bubbles_init_cuda / bubble_init_cuda / bubble_upload_all_cuda
 * (src/bubbles/bubbles_cuda.cu:3716-3770). */
int dage_bubbles_create(int natom, const double *centers, const dage_grid1d *radial, int lmax,
                        int k, const double *f, dage_bubbles **b);

/* cube += factor * sum_atoms sum_{l >= lmin} [r^k f_lm](|r-R|) Y_lm(r-R) at
 * every point of `grid` (Y_lm: Racah-normalised real spherical harmonics).
 * Replaces bubbles_inject_cuda / Bubbles::inject
 * (src/bubbles/bubbles_cuda.cu:3090-3350, 3774-3776). */
int dage_bubbles_inject(dage_bubbles *b, const dage_grid1d grid[3], int lmin, double factor,
                        double *cube, unsigned flags);
/* Radial Coulomb potential of a bubble set (Coulomb3D_evaluate_bubbles_potential,
 * src/bubbles/coulomb.F90:222-336): a new bubble set (k = 0, same centres,
 * radial grids and lmax) holding, per atom and (l, m),
 *   V_lm(r) = 4 pi/(2l+1) [ r^-(l+1) int_0^r f s^(l+2+k) ds + r^l int_r^inf f s^(1-l+k) ds ]
 * by the cumulative LIP integrals of InOutIntegrator1D
 * (src/bubbles/evaluators.F90:1263-1318), computed on the GPU.  The result
 * can be injected into a cube like any bubble set. */
int dage_bubbles_coulomb_potential(const dage_bubbles *in, dage_bubbles **out);

/* Radial Helmholtz potential of a bubble set for the kernel e^(-kappa r)/r,
 * kappa = sqrt(-2 energy), energy < 0 (Helmholtz3D_transform_bubbles_sub,
 * src/bubbles/helmholtz3d.F90:519-650): a new bubble set (k = 0) holding
 *   V_lm(r) = 8 kappa [ k_l(kappa r) int_0^r i_l(kappa s) f s^(2+k) ds
 *                       + i_l(kappa r) int_r^inf k_l(kappa s) f s^(2+k) ds ]
 * with the modified spherical Bessel functions i_0 = sinh x/x,
 * k_0 = pi/2 e^-x/x (helmholtz3d.F90:851-1060), computed on the GPU. */
int dage_bubbles_helmholtz_potential(const dage_bubbles *in, double energy, dage_bubbles **out);

/* Integral of a bubble set over all space (Bubbles_integrate_all,
 * src/bubbles/bubbles.F90:3146-3240): 4 pi sum_atoms int r^(2+k) f_00(r) dr
 * with the radial grids' LIP weights, on the GPU.  With dage_integrate of
 * the cube this is Function3D_integrate (function3d.F90:1793-1840). */
int dage_bubbles_integrate(const dage_bubbles *b, double *out);

/* Copies the radial values of a bubble set (as given at creation: per atom,
 * (lmax+1)^2 functions of the atom's radial points) to host memory. */
int dage_bubbles_get_f(const dage_bubbles *b, double *f);

/* Product of two bubble sets on the same atoms and radial grids
 * (BubblesMultiplier_multiply, option (2), src/bubbles/bubbles.F90:3567-3690;
 * Bubble_product_kernel, src/bubbles/bubbles_multiplier.cu:65-106): a new set
 * with lmax = lmax_x + lmax_y (<= 12) and k = k_x + k_y whose radial functions
 * are sum_{a<=b} C_ab^LM (x_a y_b + x_b y_a [a != b]), C the real-harmonic
 * product coefficients of YProduct (src/bubbles/harmonic.F90:884-1089).  By
 * default the reference's term set is kept (it leaves out terms with
 * L < |m1 - m2|); DAGE_PRODUCT_COMPLETE includes them. */
int dage_bubbles_multiply(const dage_bubbles *x, const dage_bubbles *y, unsigned flags,
                          dage_bubbles **out);

/* The real-harmonic product table the bubble product uses (host only, no
 * GPU call): Y_a Y_b = sum c Y_lm for a <= b < (lmax+1)^2, l <= result_lmax
 * (YProduct_init, src/bubbles/harmonic.F90:884-951).  Sets *nterms; fills
 * a, b, lm, c when cap >= *nterms. */
int dage_product_table(int lmax, int result_lmax, unsigned flags, int cap, int *a, int *b, int *lm,
                       double *c, int *nterms);

/* Cube part of a function product (Function3D_multiply,
 * src/bubbles/function3d.F90:1097-1409; Function3DMultiplier::multiply,
 * src/bubbles/bubbles_cuda.cu:3533-3690) in one kernel:
 *   out = (cube1 + b1)(cube2 + b2) - br        at every point of `grid`
 * Any of b1, b2, br may be NULL; those given must share atoms and radial
 * grids.  `out` may alias cube1 or cube2.  DAGE_DEVICE_PTRS: the cubes are
 * device pointers. */
int dage_function3d_multiply(const dage_grid1d grid[3], const double *cube1, const dage_bubbles *b1,
                             const double *cube2, const dage_bubbles *b2, const dage_bubbles *br,
                             double *out, unsigned flags);

int dage_bubbles_destroy(dage_bubbles *b);

/* ---------------------------------------------------------------------------
 * Taylor-series contaminant bubbles
 * ------------------------------------------------------------------------ */

/* Contaminants are the partial derivatives d^kappa = d^(a+b+c)/dx^a dy^b dz^c,
 * |kappa| = a+b+c <= tmax (0 <= tmax <= 3), of the smooth part of a function
 * at each atom centre, stored contams[atom * ncart + i] with
 * ncart = (tmax+1)(tmax+2)(tmax+3)/6 and i the position of kappa in the
 * reference's CartIter order (last index fastest: 000, 001, 002, 010, ...;
 * src/bubbles/cartiter.F90:169-223).  Host arrays. */

/* Bubble contaminants: at each atom B, the derivatives of the sum of the
 * OTHER atoms' bubbles, sum_{A != B} [r^k f_A,lm](r_A) Y_lm (Bubbles_get_contaminants,
 * src/bubbles/bubbles.F90:2844-2910).  Derivatives are exact (Taylor-
 * polynomial arithmetic on the GPU) on the LIP interpolant of each radial
 * function; an atom beyond another's radial grid contributes 0.  Atoms may
 * not share a centre. */
int dage_bubbles_contaminants(const dage_bubbles *b, int tmax, double *contams);

/* Cube contaminants: the derivatives of the cube's 3-D LIP interpolant at
 * natom centres (Function3D_get_cube_contaminants,
 * src/bubbles/function3d.F90:1570-1624); 0 for a centre outside the grid.
 * DAGE_DEVICE_PTRS: `cube` is a device pointer (centres and contams stay on
 * the host). */
int dage_cube_contaminants(const dage_grid1d grid[3], const double *cube, int natom,
                           const double *centers, int tmax, unsigned flags, double *contams);

/* Taylor bubbles from contaminants (Bubbles_make_taylor,
 * src/bubbles/bubbles.F90:1435-1530): a new set on b's atoms and radial grids
 * with lmax = max(lmax_b, tmax) and k = k_b whose radial functions are
 *   f_lm(r) = sum_kappa (Cb + Cc)_kappa r^(|kappa|-k) w(r) / |kappa|! S_lm(kappa)
 * with w(r) = erfc(r - 2/r) / 2 (1 at r = 0) and x^kappa = r^|kappa| sum S_lm Y_lm
 * (Cart2SphIter, src/bubbles/harmonic.F90:1096-1265, looked up through the
 * reference's dvpos, which for |kappa| = 3 takes the expansion of the
 * preceding monomial).  Either contaminant array may be NULL (zero).
 * DAGE_TAYLOR_EXACT: 1/kappa! and the exact expansion, i.e. the true
 * truncated Taylor series of the contaminated function times w. */
int dage_bubbles_make_taylor(const dage_bubbles *b, const double *bubble_contams,
                             const double *cube_contams, int tmax, unsigned flags,
                             dage_bubbles **out);

/* Contaminants and Taylor bubbles in one call, with the contaminants kept on
 * the GPU (Function3D_get_taylor_series_bubbles,
 * src/bubbles/function3d.F90:1332-1405; the reference's default order is 2).
 * cube (with its grid) may be NULL: no cube contaminants (ignore_cube).
 * Flags: DAGE_DEVICE_PTRS (cube on the device), DAGE_TAYLOR_IGNORE_BUBBLES,
 * DAGE_TAYLOR_EXACT.  The reference's non_overlapping switch selects between
 * two identical damping functions and has no counterpart. */
int dage_bubbles_taylor(const dage_bubbles *b, const dage_grid1d grid[3], const double *cube,
                        int tmax, unsigned flags, dage_bubbles **out);

/* Bubble product with Taylor series (option (1) of BubblesMultiplier_multiply,
 * src/bubbles/bubbles.F90:3567-3640; BubblesMultiplier::multiplyBubble,
 * src/bubbles/bubbles_multiplier.cu:240-292):
 *   (b1 + t1)(b2 + t2) - t1 t2 = b1 b2 + b1 t2 + t1 b2
 * on the radial points, each Taylor set cut at its bubble set's lmax; the
 * result has lmax = lmax1 + lmax2 (<= 12) and k = k1 + k2.  All four sets
 * share atoms and radial grids, and t_i has b_i's k.  Its result is the
 * `br` of dage_function3d_multiply for a product of cuspy functions.
 * DAGE_PRODUCT_COMPLETE as in dage_bubbles_multiply. */
int dage_bubbles_multiply_taylor(const dage_bubbles *b1, const dage_bubbles *b2,
                                 const dage_bubbles *t1, const dage_bubbles *t2, unsigned flags,
                                 dage_bubbles **out);

/* The monomial -> harmonic table make_taylor uses (host only, no GPU call):
 * entry e says that multi-index kappa_index[e] (CartIter position) adds
 * c[e] * Y_lm[e].  Sets *n; fills the arrays when cap >= *n.
 * DAGE_TAYLOR_EXACT as above. */
int dage_cart2sph_table(int tmax, unsigned flags, int cap, int *kappa_index, int *lm, double *c,
                        int *n);


/* ---------------------------------------------------------------------------
 * Integration (Function3D_integrate / Function3D_dot_product cube part)
 * ------------------------------------------------------------------------ */

/* out = integral of f (or of f1*f2 when f2 != NULL) over the grid with LIP
 * weights.  Replaces integrator3d_integrate / SerialInfo_integrate_cube
 * (src/bubbles/parallel_info.F90:512-528, src/bubbles/integrator.cu:321-372)
 * and the cube part of Function3D_dot_product (function3d.F90:1499-1523). */
int dage_integrate(const dage_grid1d grid[3], const double *f1, const double *f2,
                   unsigned flags, double *out);

/* ---------------------------------------------------------------------------
 * Allocation-free FP64 apply
 * ------------------------------------------------------------------------ */

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory around an operator call (a caching allocator or fixed pool owns the
 * free memory, or the loop must not hit cudaFree, which synchronises the
 * device): V = sum_p w[p] (Tx_p (x) Ty_p (x) Tz_p) rho in FP64 (no coda),
 * allocating nothing.  All pointers except w are device pointers on the
 * current device: Tx/Ty/Tz hold P matrices laid out T[p][i_out][j_in]
 * (j_in fastest), rho is nix*niy*niz and V nox*noy*noz (x fastest); w holds
 * P host weights; stream may be NULL.  The two intermediate cubes live in one
 * fixed device array of 4 Mi doubles (32 MiB) that every GPU loading the
 * library keeps until exit: niy*niz*nox + niz*nox*noy must not exceed it, or
 * the call fails with DAGE_E_INVALID.  The first call on a device looks up
 * that array's device address (cudaGetSymbolAddress), so make it before any
 * stream capture.  Every call shares the array: calls that overlap on the
 * GPU race.  The array needs no clearing (each call overwrites what it
 * reads), and V is overwritten. */
int dage_op3d_apply_fp64_noalloc(int nix, int niy, int niz, int nox, int noy, int noz, int P,
                                 const double *Tx, const double *Ty, const double *Tz,
                                 const double *w, const double *rho, double *V, void *stream);

/* ---------------------------------------------------------------------------
 * Library
 * ------------------------------------------------------------------------ */
const char *dage_last_error(void);
/* Autotuner cache file (no reference counterpart: the reference has no
 * autotuner).  Launch choices the library times (tile widths of the FP64
 * contraction stages and of the GBFMM near field) are keyed on the problem
 * (points per axis, t-points, boxes or batch) and the device, kept for the
 * process and, with a path, read from and appended to this text file so that
 * later processes skip the timing.  NULL or "" keeps choices in the process
 * only.  The DAGE_TUNE_CACHE environment variable sets the path when this is
 * never called. */
int dage_set_tune_cache(const char *path);
int dage_abi_version(void);
/* Device-side timeout (in device clock cycles) for bounded waits. */
int dage_set_wait_limit(long long cycles);

#ifdef __cplusplus
}
#endif
#endif /* DAGE_GPU_H */
