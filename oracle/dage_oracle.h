/*
 * dage_oracle.h -- CPU FP64 oracle for the DAGE grid-based Coulomb/Helmholtz
 * operator path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA
 * product is compared against.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load it.  The product library
 * (dage_b200/libdagegpu.so) never links, loads or calls it.
 *
 * Every routine restates, in plain C++, the algorithm of the reference
 * Fortran file named in its comment (paths relative to the DAGE source tree).
 * Layout conventions follow the reference: cubes are Fortran column-major
 * cube(x, y, z) with x fastest; matrices are column-major.
 */
#ifndef DAGE_ORACLE_H
#define DAGE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Gaussian quadrature in t (src/bubbles/gauss.F90:81-122, 307-383) --- */
/* nlin Gauss-Legendre points on [tstart, tlin] followed by nlog log-mapped
 * points on [tlin, tlog].  tp, tw: nlin+nlog values. */
void orc_gauss_quad(int nlin, int nlog, double tstart, double tlin, double tlog,
                    double *tp, double *tw);
/* plain Gauss-Legendre rule on [-1, 1] (gauss.F90:344-383) */
void orc_gauleg(int n, double *x, double *w);

/* ---- LIP basis (src/bubbles/lip.F90) ------------------------------------ */
/* coeffs: nlip*nlip, column-major p(j,k) = coefficient of x^(nlip-k) of basis
 * polynomial j (lip.F90:285-362).  first/last: cell extent in cell units. */
int orc_lip_coeffs(int nlip, int grid_type, double *coeffs, double *first,
                   double *last);
/* integrals of each basis polynomial over [first, last] (lip.F90:392-411) */
int orc_lip_integrals(int nlip, int grid_type, double *ints);

/* ---- 1-D grids (src/bubbles/grid.F90) ----------------------------------- */
/* Grid1D_init_step (grid.F90:446-534): points (ncell*(nlip-1)+1 values) and
 * cell starts celld (ncell values). */
int orc_grid1d_points(double qmin, int ncell, int nlip, int grid_type,
                      const double *cell_scales, double *points, double *celld);
/* Grid1D_init_spheres + Grid1D_init_equidistant (grid.F90:539-640): the
 * default grid of a Gaussian generator along one axis.  Returns ncell. */
int orc_grid1d_spheres(int n, const double *centers, const double *radii,
                       double step, int nlip, double *qmin, double *cell_scale);
/* LIP-weighted integration weights per grid point (sum over the cells that
 * share a point; the weights the reference Integrator applies,
 * src/bubbles/evaluators.F90:1023-1098). */
int orc_grid1d_weights(int ncell, int nlip, int grid_type,
                       const double *cell_scales, double *weights);

/* ---- Coulomb operator matrices (src/bubbles/exponentials.F90) ----------- */
/* integrals(a,b,t,p,n) (exponentials.F90:647-666): values[n-1-i] =
 * int_a^b x^i exp(-t^2 (x-p)^2) dx, i = 0..n-1. */
void orc_expo_integrals(double a, double b, double t, double p, int n,
                        double *values);
/* exponentials() (exponentials.F90:178-346) for one axis, no PBC images.
 * Input grid: (qmin_in, ncell_in, nlip, grid_type, cell_scales_in).  Output
 * points: n_out coordinates.  T: n_out x n_in x P, column-major,
 * T(i_out, j_in, p).  The reference stores the y and z matrices transposed
 * (trsp='t'); callers transpose as needed. */
int orc_coulomb_matrix(double qmin_in, int ncell_in, int nlip, int grid_type,
                       const double *cell_scales_in, int n_out,
                       const double *out_points, int P, const double *tp,
                       double *T);
/* Same, but only the border rows/columns that border_exponentials()
 * (exponentials.F90:348-600) evaluates; other entries are zero. */
int orc_coulomb_border_matrix(double qmin_in, int ncell_in, int nlip,
                              int grid_type, const double *cell_scales_in,
                              int n_out, const double *out_points, int P,
                              const double *tp, double *T);

/* ---- Operator application (src/bubbles/function3d.F90:4230-4349) ------- */
/* V = sum_p w[p] (Tx_p (x) Ty_p (x) Tz_p) rho + coda * rho.
 * Tx: nox x nix x P  (T(i_out, j_in, p) for x)
 * Ty: noy x niy x P, Tz: noz x niz x P  (same orientation; NOT transposed).
 * rho: nix*niy*niz (x fastest); V: nox*noy*noz (overwritten).
 * coda is added only when the input and output grids coincide
 * (cube_project of identical grids is a copy); pass 0 to skip it. */
int orc_transform_cube(int nix, int niy, int niz, int nox, int noy, int noz,
                       int P, const double *Tx, const double *Ty,
                       const double *Tz, const double *w, double coda,
                       const double *rho, double *V);

/* Integrator_eval (src/bubbles/evaluators.F90:1064-1098): integral of a cube
 * with LIP weights, contracted x, then y, then z. */
double orc_integrate_cube(int nlip, int grid_type, int ncx, const double *hx,
                          int ncy, const double *hy, int ncz, const double *hz,
                          const double *f);

/* ---- Test densities (src/bubbles/gauss_generator.F90, analytical.F90) --- */
/* GaussGenerator_gen_cubef (gauss_generator.F90:291-318) */
void orc_gauss_cube(int ng, const double *q, const double *alpha,
                    const double *centers, int nx, const double *x, int ny,
                    const double *y, int nz, const double *z, double *cube);
/* GaussPotGenerator_gen_cubef (gauss_generator.F90:384-429) */
void orc_gauss_pot_cube(int ng, const double *q, const double *alpha,
                        const double *centers, int nx, const double *x, int ny,
                        const double *y, int nz, const double *z, double *cube);
/* gauss_analytical_energy without PBC (analytical.F90:308-420) */
double orc_gauss_analytical_energy(int ng, const double *q, const double *alpha,
                                   const double *centers);
/* extent of each Gaussian shell (gauss_generator.F90:262-281) */
void orc_gauss_extent(int ng, const double *q, const double *alpha,
                      double thres, double *extent);

/* ---- GBFMM pieces (src/bubbles/multipole.F90, harmonics.F90,
 *      src/gbfmm/gbfmm_parallel_info.F90) ---------------------------------- */
/* Racah-normalised real regular solid harmonics S_lm, lm = l(l+1)+m. */
void orc_solid_harmonics(int lmax, double x, double y, double z, double *S);
/* M2L interaction matrix T(d), N x N column-major, N = (lmax+1)^2. */
int orc_interaction_matrix(int lmax, const double *d, double *T);
/* M2M/L2L translation matrix, packed lower triangle (N(N+1)/2). */
int orc_translation_matrix(int lmax, const double *d, double *W);
void orc_dtpmv_lower_unit(int n, const double *A, double *x);
/* octree boxes (1-based indices; 2^level boxes per axis) */
void orc_box_vector(int ibox, int level, int *v);
int orc_box_index(const int *v, int level);
int orc_nearest_neighbors(int ibox, int level, int *out);
int orc_local_farfield(int ibox, int level, int *out);
/* multipole moments of one box and local-expansion evaluation */
int orc_box_multipoles(int lmax, int nx, const double *px, const double *wx, int ny,
                       const double *py, const double *wy, int nz, const double *pz,
                       const double *wz, const double *cube, const double *center, double *q);
int orc_l2p(int lmax, const double *L, const double *center, int nx, const double *px, int ny,
            const double *py, int nz, const double *pz, double *out);

/* ---- bubbles -> cube injection (src/bubbles/bubbles.F90:1904-1975) ------ */
/* cube += factor * sum_atoms sum_{l >= lmin} [r^k f_lm](|r - R|) Y_lm.
 * Atom a: radial grid of ncell[a] equidistant-LIP cells starting at r = 0
 * (cell_scales concatenated over atoms); f: per atom (lmax+1)^2 rows of the
 * radial grid's points, atoms concatenated. */
int orc_bubbles_inject(int natom, const double *centers, const int *ncell,
                       const double *cell_scales, int nlip, int lmax, int lmin, int k,
                       const double *f, int nx, const double *x, int ny, const double *y,
                       int nz, const double *z, double factor, double *cube);

/* Helmholtz (Yukawa) far field (helmholtz_ref.cpp) */
void orc_bessel_i(double x, int lmax, double *out);
void orc_bessel_k(double x, int lmax, double *out);
void orc_aligned_ml(const double *bessel, int lmax, int lin, double *out);
void orc_rotation(const double *dhat, int lmax, double *out);
void orc_ref_real_rotation(double alpha, double beta, double gamma, int lmax, int repaired,
                           double *out);
int orc_helm_m2l_lsq(int lmax, int lin, double kappa, const double *M, const double *src,
                     const double *dst, double *L);
int orc_helm_m2l(int lmax, int lin, double kappa, const double *M, const double *src,
                 const double *dst, double *L);
void orc_aligned_mm(const double *bessel, int lmax, int lin, double *out);
int orc_helm_m2m(int lmax, int lin, double kappa, const double *M, const double *src,
                 const double *dst, double *out);
int orc_helm_matrix(int kind, int lmax, int lin, double kappa, const double *src,
                    const double *dst, double *out);
int orc_helm_box_multipoles(int lmax, double kappa, int nx, const double *px, const double *wx,
                            int ny, const double *py, const double *wy, int nz, const double *pz,
                            const double *wz, const double *rho, const double *center, double *q);
int orc_helm_l2p(int lmax, double kappa, const double *L, const double *center, int nx,
                 const double *px, int ny, const double *py, int nz, const double *pz, double *V);

#ifdef __cplusplus
}
#endif
#endif
