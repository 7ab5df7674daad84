// taylor.cu -- Taylor-series contaminant bubbles on one B200.
//
// Near a nucleus B the smooth part of a function -- its cube and the bubbles
// of every OTHER atom -- is replaced by its truncated Taylor series around
// R_B and carried as a bubble on B (Function3D_get_taylor_series_bubbles,
// src/bubbles/function3d.F90:1332-1405).  Three steps, three kernels:
//
//   bubble contaminants  C^b_kappa(B) = sum_{A != B} d^kappa [ sum_lm (r^k f_A,lm)(r_A) Y_lm ](R_B)
//                        (Bubbles_get_contaminants, src/bubbles/bubbles.F90:2844-2910)
//   cube contaminants    C^c_kappa(B) = d^kappa [ 3-D LIP interpolant of the cube ](R_B)
//                        (Function3D_get_cube_contaminants, function3d.F90:1570-1624)
//   make_taylor          t_B,lm(r) = sum_kappa (C^b + C^c) r^(|kappa|-k) w(r) / |kappa|! S_lm(kappa)
//                        (Bubbles_make_taylor, bubbles.F90:1435-1530)
//
// kappa runs over the multi-indices with |kappa| <= T in the reference's
// CartIter order (last index fastest, src/bubbles/cartiter.F90:169-223), w is
// the damping 0.5 erfc(r - 2/r) (1 at r <= DBL_EPSILON, bubbles.F90:1532-1558),
// and S_lm(kappa) expands the monomial x^kappa = r^|kappa| sum S_lm(kappa) Y_lm
// in the Racah-normalised real harmonics (Cart2SphIter, harmonic.F90:
// 1096-1265).  Two properties of the reference are kept by default:
//   * the series divides by |kappa|!, not kappa!, so mixed terms are scaled
//     down (by 2 for |kappa| = 2);
//   * the harmonic expansion is looked up through dvpos, whose shell offset
//     |kappa|^2 equals the true offset |kappa|(|kappa|+1)(|kappa|+2)/6 only
//     for |kappa| <= 2, so a third-order term takes the expansion of the
//     monomial one place before it.
// DAGE_TAYLOR_EXACT replaces both by the true Taylor series.
//
// The derivatives are exact: the bubble kernel carries every quantity as a
// truncated multivariate Taylor polynomial (a "jet") in the displacement
// (dx, dy, dz) about R_B -- r^2, r = sqrt(r^2), 1/r, the unit vector, the
// harmonics by their recursion, the radial LIP polynomial composed with
// r - |R_B - R_A| -- so d^kappa = kappa! x the jet's kappa coefficient.  The
// reference forms the same derivatives symbolically (Y_eval_coeffs,
// harmonic.F90:806-860, times LIP derivatives of the radial function,
// Bubbles_get_radial_derivatives, bubbles.F90:2272-2340).
//
// The bubble product of option (1) of BubblesMultiplier_multiply
// (bubbles.F90:3567-3640; BubblesMultiplier::multiplyBubble,
// src/bubbles/bubbles_multiplier.cu:240-292),
//   (b1 + t1)(b2 + t2) - t1 t2 = b1 b2 + b1 t2 + t1 b2,
// runs as one pass over the radial points (the right-hand form: no
// cancellation of t1 t2), each Taylor set cut at its bubble set's lmax as the
// reference's device arrays cut it (Bubble::add, bubbles_cuda.cu:2629-2680).
#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <vector>

#include "bubbles.cuh"

namespace dage {
namespace {

constexpr int kMaxTaylor = 3;

__host__ __device__ constexpr int ncart(int T) { return (T + 1) * (T + 2) * (T + 3) / 6; }

// Position of (a, b, c), a + b + c <= T, in CartIter order.
__host__ __device__ constexpr int cart_index(int T, int a, int b, int c) {
  int i = 0;
  for (int a2 = 0; a2 < a; ++a2) i += (T - a2 + 1) * (T - a2 + 2) / 2;
  for (int b2 = 0; b2 < b; ++b2) i += T - a - b2 + 1;
  return i + c;
}

// The multi-index at CartIter position i.
__host__ __device__ inline void cart_decode(int T, int i, int &a, int &b, int &c) {
  for (a = 0; a <= T; ++a)
    for (b = 0; a + b <= T; ++b)
      for (c = 0; a + b + c <= T; ++c)
        if (cart_index(T, a, b, c) == i) return;
  a = b = c = 0;
}

// ---------------------------------------------------------------- jets
// A jet is a truncated Taylor polynomial in (dx, dy, dz) of total degree
// <= T, its ncart(T) coefficients in CartIter order, held in a double[kNC].
// The jet product runs from a table of the (i, j, k) index triples with
// monomial_i * monomial_j = monomial_k built once per block in shared memory
// (84 triples for T = 3), so that the device code stays small.
constexpr int kNC = 20;     // ncart(kMaxTaylor)
constexpr int kNProd = 84;  // products of monomials of total degree <= 3

struct JetCtx {
  int nc, np;
  const unsigned char *pi, *pj, *pk;
};

// Thread 0 of the block fills the product table of order T.
__device__ void jet_tables(int T, unsigned char *pi, unsigned char *pj, unsigned char *pk,
                           int *np) {
  if (threadIdx.x != 0) return;
  int n = 0;
  for (int a1 = 0; a1 <= T; ++a1)
    for (int b1 = 0; a1 + b1 <= T; ++b1)
      for (int c1 = 0; a1 + b1 + c1 <= T; ++c1)
        for (int a2 = 0; a1 + b1 + c1 + a2 <= T; ++a2)
          for (int b2 = 0; a1 + b1 + c1 + a2 + b2 <= T; ++b2)
            for (int c2 = 0; a1 + b1 + c1 + a2 + b2 + c2 <= T; ++c2) {
              pi[n] = (unsigned char)cart_index(T, a1, b1, c1);
              pj[n] = (unsigned char)cart_index(T, a2, b2, c2);
              pk[n] = (unsigned char)cart_index(T, a1 + a2, b1 + b2, c1 + c2);
              ++n;
            }
  *np = n;
}

__device__ __noinline__ void jset(const JetCtx &J, double v, double *r) {
  for (int i = 0; i < J.nc; ++i) r[i] = 0.0;
  r[0] = v;
}

__device__ __noinline__ void jcopy(const JetCtx &J, const double *x, double *r) {
  for (int i = 0; i < J.nc; ++i) r[i] = x[i];
}

// r = x * y (r must not alias x or y)
__device__ __noinline__ void jmul(const JetCtx &J, const double *x, const double *y, double *r) {
  for (int i = 0; i < J.nc; ++i) r[i] = 0.0;
  for (int p = 0; p < J.np; ++p) r[J.pk[p]] += x[J.pi[p]] * y[J.pj[p]];
}

// r = alpha x + beta y (r may alias x or y)
__device__ __noinline__ void jlin(const JetCtx &J, double alpha, const double *x, double beta,
                                  const double *y, double *r) {
  for (int i = 0; i < J.nc; ++i) r[i] = alpha * x[i] + beta * y[i];
}

// r = sum_j f[j] p[j], j <= T, over the powers p[j] = e^j of a jet e with no
// constant term (p[0] = 1): the composition F(v0 + e), f[j] = F^(j)(v0)/j!.
__device__ __noinline__ void jcompose(const JetCtx &J, int T, const double *f,
                                      const double (*p)[kNC], double *r) {
  for (int i = 0; i < J.nc; ++i) r[i] = 0.0;
  for (int j = 0; j <= T; ++j)
    for (int i = 0; i < J.nc; ++i) r[i] += f[j] * p[j][i];
}

// p[j] = e^j, j <= T
__device__ __noinline__ void jpowers(const JetCtx &J, int T, const double *e, double (*p)[kNC]) {
  jset(J, 1.0, p[0]);
  if (T >= 1) jcopy(J, e, p[1]);
  for (int j = 2; j <= T; ++j) jmul(J, p[j - 1], e, p[j]);
}

// Racah-normalised real spherical harmonics of a unit-vector jet: the
// recursion of unit_harmonics on jets (|u|^2 = 1 holds as a jet); f(lm, Y).
template <class F>
__device__ void jet_harmonics(const JetCtx &J, int lmax, const double *x, const double *y,
                              const double *z, F &&f) {
  double p1[kNC], p2[kNC], cur[kNC], t1[kNC], t2[kNC], top[kNC], bot[kNC];
  jset(J, 1.0, cur);
  f(0, cur);
  if (lmax == 0) return;
  jset(J, 1.0, p2);
  jcopy(J, z, p1);
  f(2, p1);
  for (int l = 2; l <= lmax; ++l) {
    jmul(J, z, p1, t1);
    jlin(J, (2.0 * l - 1.0) / sqrt((double)(l * l)), t1,
         -sqrt((double)((l - 1) * (l - 1))) / sqrt((double)(l * l)), p2, cur);
    f(l * (l + 1), cur);
    jcopy(J, p1, p2);
    jcopy(J, cur, p1);
  }
  jcopy(J, x, top);
  jcopy(J, y, bot);
  for (int mm = 1; mm <= lmax; ++mm) {
    if (mm >= 2) {
      const double c = sqrt(1.0 - 0.5 / mm);
      jmul(J, top, y, t1);
      jmul(J, bot, x, t2);
      jlin(J, c, t1, c, t2, cur);  // new bot
      jmul(J, top, x, t1);
      jmul(J, bot, y, t2);
      jlin(J, c, t1, -c, t2, top);
      jcopy(J, cur, bot);
    }
    f(mm * (mm + 1) + mm, top);
    f(mm * (mm + 1) - mm, bot);
    for (int sg = 0; sg < 2; ++sg) {
      const int m = sg ? -mm : mm;
      jset(J, 0.0, p2);
      jcopy(J, sg ? bot : top, p1);
      for (int l = mm + 1; l <= lmax; ++l) {
        const double s = 1.0 / sqrt(1.0 * (l - m) * (l + m));
        jmul(J, p1, z, t1);
        if (l - mm > 1)
          jlin(J, (2.0 * l - 1.0) * s, t1, -sqrt((l + m - 1.0) * (l - m - 1.0)) * s, p2, cur);
        else
          jlin(J, (2.0 * l - 1.0) * s, t1, 0.0, t1, cur);
        f(l * (l + 1) + m, cur);
        jcopy(J, p1, p2);
        jcopy(J, cur, p1);
      }
    }
  }
}

// Taylor coefficients q[j] = p^(j)(t) / j!, j <= T, of a polynomial given by
// its coefficients c[0..n] (highest power first), by repeated synthetic
// division.
__host__ __device__ inline void poly_taylor(const double *c, int n, double t, int T, double *q) {
  double a[8];
  for (int i = 0; i <= n; ++i) a[i] = c[i];
  for (int j = 0; j <= T; ++j) {
    if (j > n) {
      q[j] = 0.0;
      continue;
    }
    for (int i = 1; i <= n - j; ++i) a[i] += a[i - 1] * t;
    q[j] = a[n - j];
  }
}

__host__ __device__ inline double ifact(int n) {
  double f = 1.0;
  for (int i = 2; i <= n; ++i) f *= i;
  return f;
}

// One block per evaluation atom B; its threads take the source atoms A and
// the block sums their jets in a fixed order.
constexpr int kContamThreads = 128;

__global__ void __launch_bounds__(kContamThreads)
    bubble_contaminants_kernel(const AtomTab *__restrict__ atoms, int natom,
                               const double *__restrict__ celld, const double *__restrict__ hcell,
                               const double *__restrict__ coef, int N, int lmax, int nlip,
                               double first, int T, double *__restrict__ contams) {
  __shared__ double red[kNC][kContamThreads];
  __shared__ unsigned char pi[kNProd], pj[kNProd], pk[kNProd];
  __shared__ int nprod;
  jet_tables(T, pi, pj, pk, &nprod);
  __syncthreads();
  const JetCtx J{ncart(T), nprod, pi, pj, pk};
  const int B = blockIdx.x;
  const AtomTab tb = atoms[B];
  double acc[kNC];
  jset(J, 0.0, acc);
  for (int A = threadIdx.x; A < natom; A += blockDim.x) {
    if (A == B) continue;
    const AtomTab ta = atoms[A];
    const double dx = tb.cx - ta.cx, dy = tb.cy - ta.cy, dz = tb.cz - ta.cz;
    const double d2 = dx * dx + dy * dy + dz * dz, d = sqrt(d2);
    // outside A's radial grid the interpolant is 0 (Grid1D_get_icell)
    if (!(d <= ta.rmax) || !(d > 0.0)) continue;
    const double *cd = celld + ta.cell0;
    const int ic = radial_cell(cd, ta.ncell, d);
    if (!ic) continue;
    const double h = hcell[ta.cell0 + ic - 1];
    const double t = (d - cd[ic - 1]) / h + first;
    // coordinates about R_A as jets in the displacement e about R_B, and
    // r^2 - d^2 = 2 d.e + |e|^2
    double X[kNC], Y[kNC], Z[kNC], del[kNC];
    jset(J, dx, X);
    jset(J, dy, Y);
    jset(J, dz, Z);
    jset(J, 0.0, del);
    if (T >= 1) {
      X[cart_index(T, 1, 0, 0)] = 1.0;
      Y[cart_index(T, 0, 1, 0)] = 1.0;
      Z[cart_index(T, 0, 0, 1)] = 1.0;
      del[cart_index(T, 1, 0, 0)] = 2.0 * dx;
      del[cart_index(T, 0, 1, 0)] = 2.0 * dy;
      del[cart_index(T, 0, 0, 1)] = 2.0 * dz;
    }
    if (T >= 2) {
      del[cart_index(T, 2, 0, 0)] = 1.0;
      del[cart_index(T, 0, 2, 0)] = 1.0;
      del[cart_index(T, 0, 0, 2)] = 1.0;
    }
    double pw[kMaxTaylor + 1][kNC];
    jpowers(J, T, del, pw);
    // sqrt(v) and v^-1/2 at v = d^2: binomial series in del / d^2
    double fs[kMaxTaylor + 1], fi[kMaxTaylor + 1];
    {
      double bs = 1.0, bi = 1.0, vp = 1.0;  // binomial(1/2, j), binomial(-1/2, j), d2^-j
      for (int j = 0; j <= T; ++j) {
        fs[j] = bs * d * vp;
        fi[j] = bi / d * vp;
        bs *= (0.5 - j) / (j + 1);
        bi *= (-0.5 - j) / (j + 1);
        vp /= d2;
      }
    }
    double r[kNC], rinv[kNC], ux[kNC], uy[kNC], uz[kNC];
    jcompose(J, T, fs, pw, r);
    jcompose(J, T, fi, pw, rinv);
    jmul(J, X, rinv, ux);
    jmul(J, Y, rinv, uy);
    jmul(J, Z, rinv, uz);
    r[0] = 0.0;  // r - d
    double ep[kMaxTaylor + 1][kNC];
    jpowers(J, T, r, ep);
    const double *cf = coef + (size_t)(ta.cell0 + ic - 1) * N * 8;
    double hinv[kMaxTaylor + 1];
    hinv[0] = 1.0;
    for (int j = 1; j <= T; ++j) hinv[j] = hinv[j - 1] / h;
    jet_harmonics(J, lmax, ux, uy, uz, [&](int lm, const double *Ylm) {
      double q[kMaxTaylor + 1], g[kNC], gy[kNC];
      poly_taylor(cf + (size_t)lm * 8, nlip - 1, t, T, q);
      for (int j = 0; j <= T; ++j) q[j] *= hinv[j];
      jcompose(J, T, q, ep, g);
      jmul(J, g, Ylm, gy);
      jlin(J, 1.0, acc, 1.0, gy, acc);
    });
  }
  for (int i = 0; i < J.nc; ++i) red[i][threadIdx.x] = acc[i];
  __syncthreads();
  if (threadIdx.x < J.nc) {
    const int i = threadIdx.x;
    double s = 0.0;
    for (int k = 0; k < kContamThreads; ++k) s += red[i][k];
    int a, b, c;
    cart_decode(T, i, a, b, c);
    contams[(size_t)B * J.nc + i] = ifact(a) * ifact(b) * ifact(c) * s;
  }
}

// One axis of the cube grid for the interpolant.
struct CubeAxis {
  const double *celld, *h;
  double qmin, qmax;
  int ncell;
};
struct CubeAxes {
  CubeAxis ax[3];
};

// Derivatives of the cube's 3-D LIP interpolant at each atom centre (the
// Interpolator of evaluators.F90:853-1000 with derivative order T): one block
// per atom; threads 0-2 find the cell of each coordinate and the basis
// polynomials' derivatives there, the block stages the nlip^3 values of the
// cell, and thread i contracts them for multi-index i (x innermost).
__global__ void __launch_bounds__(64)
    cube_contaminants_kernel(CubeAxes axes, const double *__restrict__ lipc, int nlip, double first,
                             const double *__restrict__ centers, const double *__restrict__ cube,
                             int nx, int ny, int T, double *__restrict__ contams) {
  const int NC = ncart(T);
  __shared__ double P[3][kMaxTaylor + 1][8];
  __shared__ int start[3], inside[3];
  __shared__ double vals[8 * 8 * 8];
  const int B = blockIdx.x;
  if (threadIdx.x < 3) {
    const int d = threadIdx.x;
    const CubeAxis A = axes.ax[d];
    const double x = centers[3 * B + d];
    int ic = 0;
    if (!(x > A.qmax || x < A.qmin)) ic = radial_cell(A.celld, A.ncell, x);
    inside[d] = ic > 0;
    start[d] = ic > 0 ? (ic - 1) * (nlip - 1) : 0;
    if (ic > 0) {
      const double h = A.h[ic - 1], t = (x - A.celld[ic - 1]) / h + first;
      for (int i = 0; i < nlip; ++i) {
        // basis polynomial i: coefficients lipc[k * nlip + i], highest first
        double c[8], q[kMaxTaylor + 1];
        for (int k = 0; k < nlip; ++k) c[k] = lipc[k * nlip + i];
        poly_taylor(c, nlip - 1, t, T, q);
        double hp = 1.0;
        for (int j = 0; j <= T; ++j) {
          P[d][j][i] = ifact(j) * q[j] * hp;
          hp /= h;
        }
      }
    }
  }
  __syncthreads();
  const bool in = inside[0] && inside[1] && inside[2];
  if (in) {
    const int n3 = nlip * nlip * nlip;
    for (int e = threadIdx.x; e < n3; e += blockDim.x) {
      const int i = e % nlip, j = (e / nlip) % nlip, k = e / (nlip * nlip);
      vals[e] = cube[(size_t)(start[0] + i) +
                     (size_t)nx * ((size_t)(start[1] + j) + (size_t)ny * (start[2] + k))];
    }
  }
  __syncthreads();
  if (threadIdx.x < NC) {
    const int id = threadIdx.x;
    double s = 0.0;
    if (in) {
      int a, b, c;
      cart_decode(T, id, a, b, c);
      for (int k = 0; k < nlip; ++k) {
        double sy = 0.0;
        for (int j = 0; j < nlip; ++j) {
          double sx = 0.0;
          for (int i = 0; i < nlip; ++i) sx += vals[(k * nlip + j) * nlip + i] * P[0][a][i];
          sy += sx * P[1][b][j];
        }
        s += sy * P[2][c][k];
      }
    }
    contams[(size_t)B * NC + id] = s;
  }
}

// Radial functions of the Taylor bubbles: one thread per (atom, radial
// point).  f_lm(r) = sum_kappa sum_{(lm, s) of kappa} s * [(Cb + Cc) *
// (rpow(r, |kappa| - k) * w(r) * fac(kappa))], accumulated kappa by kappa
// as Bubbles_make_taylor does.
__global__ void make_taylor_kernel(const double *__restrict__ rpts, const int *__restrict__ np,
                                   const int *__restrict__ poff, int natom,
                                   const double *__restrict__ cb, const double *__restrict__ cc,
                                   int NC, const int *__restrict__ kabs,
                                   const double *__restrict__ fac, const int *__restrict__ sptr,
                                   const int *__restrict__ slm, const double *__restrict__ sval,
                                   int Nn, int k, double *__restrict__ out) {
  const int total = poff[natom];
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  int a = 0;
  while (poff[a + 1] <= idx) ++a;
  const int j = idx - poff[a], npts = np[a];
  const double r = rpts[idx];
  const double w = r > DBL_EPSILON ? 0.5 * erfc(r - 2.0 / r) : 1.0;
  double *o = out + (size_t)Nn * poff[a] + j;
  for (int i = 0; i < NC; ++i) {
    const double c = (cb ? cb[(size_t)a * NC + i] : 0.0) + (cc ? cc[(size_t)a * NC + i] : 0.0);
    const int n = kabs[i] - k;
    double rp;
    if (n >= 0) {
      rp = 1.0;
      for (int e = 0; e < n; ++e) rp *= r;
    } else if (j == 0) {
      rp = 0.0;  // Bubbles_rpow: negative powers are 0 at the first point
    } else {
      double q = 1.0;
      for (int e = 0; e < -n; ++e) q *= r;
      rp = 1.0 / q;
    }
    const double v = c * (rp * w * fac[i]);
    for (int e = sptr[i]; e < sptr[i + 1]; ++e) o[(size_t)slm[e] * npts] += sval[e] * v;
  }
}

// Option (1) product: out_LM += C (b1_a (b2_b + t2_b) + t1_a b2_b + [a <-> b]).
// The Taylor sets are read with their own row counts (Rt1, Rt2) but only
// for lm below the bubble sets' N1, N2.
__global__ void bubbles_product_taylor_kernel(const double *__restrict__ f1, int N1,
                                              const double *__restrict__ u1, int Rt1,
                                              const double *__restrict__ f2, int N2,
                                              const double *__restrict__ u2, int Rt2,
                                              const int *__restrict__ np,
                                              const int *__restrict__ poff, int natom,
                                              const ProdTerm *__restrict__ terms, int nterms,
                                              int Nr, double *out) {
  const int total = poff[natom];
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  int a = 0;
  while (poff[a + 1] <= idx) ++a;
  const int j = idx - poff[a], npts = np[a];
  const double *g1 = f1 + (size_t)N1 * poff[a] + j;
  const double *g2 = f2 + (size_t)N2 * poff[a] + j;
  const double *h1 = u1 + (size_t)Rt1 * poff[a] + j;
  const double *h2 = u2 + (size_t)Rt2 * poff[a] + j;
  double *o = out + (size_t)Nr * poff[a] + j;
  for (int t = 0; t < nterms; ++t) {
    const ProdTerm T = terms[t];
    double s = 0.0;
    if (T.a < N1 && T.b < N2) {
      const size_t pa = (size_t)T.a * npts, pb = (size_t)T.b * npts;
      s += g1[pa] * (g2[pb] + h2[pb]) + h1[pa] * g2[pb];
    }
    if (T.a != T.b && T.b < N1 && T.a < N2) {
      const size_t pa = (size_t)T.a * npts, pb = (size_t)T.b * npts;
      s += g1[pb] * (g2[pa] + h2[pa]) + h1[pb] * g2[pa];
    }
    o[(size_t)T.lm * npts] += T.c * s;
  }
}

// ------------------------------------------------------------ host tables
// Dense polynomial in x, y, z of degree <= 3.
struct Poly3 {
  double c[4][4][4] = {};
  Poly3 times(int axis) const {  // * x, * y or * z
    Poly3 r;
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b)
        for (int e = 0; e < 4; ++e) {
          if (c[a][b][e] == 0.0) continue;
          const int a2 = a + (axis == 0), b2 = b + (axis == 1), e2 = e + (axis == 2);
          if (a2 < 4 && b2 < 4 && e2 < 4) r.c[a2][b2][e2] += c[a][b][e];
        }
    return r;
  }
  Poly3 r2() const {
    Poly3 x = times(0).times(0), y = times(1).times(1), z = times(2).times(2);
    return x.lin(1.0, y, 1.0).lin(1.0, z, 1.0);
  }
  Poly3 lin(double alpha, const Poly3 &o, double beta) const {
    Poly3 r;
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b)
        for (int e = 0; e < 4; ++e) r.c[a][b][e] = alpha * c[a][b][e] + beta * o.c[a][b][e];
    return r;
  }
};

// Racah-normalised real solid harmonics S_lm (l <= 3) as polynomials: the
// recursion of unit_harmonics with r^2 = x^2 + y^2 + z^2 kept.
void solid_polys(std::vector<Poly3> &S) {
  const int L = 3;
  S.assign((L + 1) * (L + 1), Poly3());
  Poly3 one;
  one.c[0][0][0] = 1.0;
  S[0] = one;
  Poly3 x = one.times(0), y = one.times(1), z = one.times(2);
  S[2] = z;
  for (int l = 2; l <= L; ++l)
    S[l * (l + 1)] = S[(l - 1) * l].times(2).lin((2.0 * l - 1.0) / l, S[(l - 2) * (l - 1)].r2(),
                                                 -(l - 1.0) / l);
  Poly3 top = x, bot = y;
  for (int mm = 1; mm <= L; ++mm) {
    if (mm >= 2) {
      const double c = std::sqrt(1.0 - 0.5 / mm);
      const Poly3 nb = top.times(1).lin(c, bot.times(0), c);
      const Poly3 nt = top.times(0).lin(c, bot.times(1), -c);
      top = nt;
      bot = nb;
    }
    S[mm * (mm + 1) + mm] = top;
    S[mm * (mm + 1) - mm] = bot;
    for (int sg = 0; sg < 2; ++sg) {
      const int m = sg ? -mm : mm;
      for (int l = mm + 1; l <= L; ++l) {
        Poly3 cur = S[(l - 1) * l + m].times(2).lin(2.0 * l - 1.0, Poly3(), 0.0);
        if (l - mm > 1)
          cur = cur.lin(1.0, S[(l - 2) * (l - 1) + m].r2(), -std::sqrt((l + m - 1.0) * (l - m - 1.0)));
        S[l * (l + 1) + m] = cur.lin(1.0 / std::sqrt(1.0 * (l - m) * (l + m)), Poly3(), 0.0);
      }
    }
  }
}

// The monomials of shell k in the reference's in-shell order (dvpos_shell,
// harmonic.F90:1378-1385: first index outer, second inner).
void shell_monomials(int k, std::vector<std::array<int, 3>> &mono) {
  mono.clear();
  for (int a = 0; a <= k; ++a)
    for (int b = 0; a + b <= k; ++b) mono.push_back({a, b, k - a - b});
}

// Cart2SphIter_init (harmonic.F90:1096-1165) for shells 0..3: per shell k,
// the matrix of the monomial coefficients of r^(k-l) S_lm (l = k, k-2, ...)
// is inverted; column `col` of the result (shell-grouped, 0-based) lists
// the (lm, coefficient) pairs with |coefficient| > 1e-16.
struct C2SCol {
  std::vector<std::pair<int, double>> e;
};
int cart_to_sph_columns(std::vector<C2SCol> &cols) {
  std::vector<Poly3> S;
  solid_polys(S);
  cols.assign(ncart(kMaxTaylor), C2SCol());
  for (int k = 0; k <= kMaxTaylor; ++k) {
    std::vector<std::array<int, 3>> mono;
    shell_monomials(k, mono);
    const int n = (int)mono.size();
    std::vector<int> sph;  // lm of each matrix column, l ascending then m
    for (int l = k % 2; l <= k; l += 2)
      for (int m = -l; m <= l; ++m) sph.push_back(l * (l + 1) + m);
    if ((int)sph.size() != n) return fail(DAGE_E_INVALID, "Cart2Sph shell size");
    // M[row = monomial][col = harmonic]
    std::vector<double> M((size_t)n * n, 0.0), Inv((size_t)n * n, 0.0);
    for (int s = 0; s < n; ++s) {
      const int lm = sph[s], l = (int)std::sqrt((double)lm);
      Poly3 p = S[lm];
      for (int e = l; e < k; e += 2) p = p.r2();
      for (int r = 0; r < n; ++r) M[(size_t)r * n + s] = p.c[mono[r][0]][mono[r][1]][mono[r][2]];
    }
    // Gauss-Jordan with partial pivoting
    for (int i = 0; i < n; ++i) Inv[(size_t)i * n + i] = 1.0;
    for (int col = 0; col < n; ++col) {
      int piv = col;
      for (int r = col + 1; r < n; ++r)
        if (std::fabs(M[(size_t)r * n + col]) > std::fabs(M[(size_t)piv * n + col])) piv = r;
      if (M[(size_t)piv * n + col] == 0.0) return fail(DAGE_E_INVALID, "Cart2Sph singular shell");
      for (int c = 0; c < n; ++c) {
        std::swap(M[(size_t)piv * n + c], M[(size_t)col * n + c]);
        std::swap(Inv[(size_t)piv * n + c], Inv[(size_t)col * n + c]);
      }
      const double d = M[(size_t)col * n + col];
      for (int c = 0; c < n; ++c) {
        M[(size_t)col * n + c] /= d;
        Inv[(size_t)col * n + c] /= d;
      }
      for (int r = 0; r < n; ++r) {
        if (r == col) continue;
        const double f = M[(size_t)r * n + col];
        if (f == 0.0) continue;
        for (int c = 0; c < n; ++c) {
          M[(size_t)r * n + c] -= f * M[(size_t)col * n + c];
          Inv[(size_t)r * n + c] -= f * Inv[(size_t)col * n + c];
        }
      }
    }
    // Inv[harmonic][monomial]: harmonic coefficients of each monomial
    const int base = k * (k + 1) * (k + 2) / 6;
    for (int r = 0; r < n; ++r) {
      std::vector<std::pair<int, double>> e;
      for (int s = 0; s < n; ++s) {
        const double v = Inv[(size_t)s * n + r];
        if (std::fabs(v) > 1e-16) e.push_back({sph[s], v});
      }
      std::sort(e.begin(), e.end());
      cols[base + r].e = e;
    }
  }
  return 0;
}

// Per multi-index (CartIter order, |kappa| <= T): |kappa|, the series factor
// (1/|kappa|! or, exact, 1/kappa!) and its harmonic expansion.
struct TaylorTables {
  int T = 0, NC = 0;
  std::vector<int> kabs, sptr, slm;
  std::vector<double> fac, sval;
};
int taylor_tables(int T, bool exact, TaylorTables &tt) {
  std::vector<C2SCol> cols;
  DAGE_TRY(cart_to_sph_columns(cols));
  tt.T = T;
  tt.NC = ncart(T);
  tt.kabs.clear();
  tt.fac.clear();
  tt.sptr.assign(1, 0);
  tt.slm.clear();
  tt.sval.clear();
  for (int i = 0; i < tt.NC; ++i) {
    int a, b, c;
    cart_decode(T, i, a, b, c);
    const int K = a + b + c;
    tt.kabs.push_back(K);
    tt.fac.push_back(exact ? 1.0 / (ifact(a) * ifact(b) * ifact(c)) : 1.0 / ifact(K));
    // dvpos_shell (1-based) + shell offset: |kappa|^2 in the reference's
    // dvpos (harmonic.F90:1369-1376), the true offset when exact
    const int pos = (a * (3 + 2 * K - a) + 2) / 2 + b;
    const int col = (exact ? K * (K + 1) * (K + 2) / 6 : K * K) + pos - 1;
    for (const auto &e : cols[col].e) {
      tt.slm.push_back(e.first);
      tt.sval.push_back(e.second);
    }
    tt.sptr.push_back((int)tt.slm.size());
  }
  return 0;
}

// Bubble contaminants of every atom into a device array [natom][ncart(T)].
int bubble_contaminants_launch(const dage_bubbles *b, int T, double *d_out, cudaStream_t s) {
  for (int i = 0; i < b->natom; ++i)
    for (int j = 0; j < i; ++j) {
      const double *p = &b->centers[3 * i], *q = &b->centers[3 * j];
      if (p[0] == q[0] && p[1] == q[1] && p[2] == q[2])
        return fail(DAGE_E_INVALID, "contaminants: atoms %d and %d share a centre", j, i);
    }
  bubble_contaminants_kernel<<<b->natom, kContamThreads, 0, s>>>(
      b->atoms.as<AtomTab>(), b->natom, b->celld.as<double>(), b->hcell.as<double>(),
      b->coef.as<double>(), b->N, b->lmax, b->nlip, b->first, T, d_out);
  DAGE_CUDA_TRY(cudaGetLastError());
  return 0;
}

// Cube contaminants at `natom` device centres into d_out [natom][ncart(T)];
// the cube is a device pointer.  The grid tables live in `keep` until the
// caller has synchronised.
int cube_contaminants_launch(const dage_grid1d grid[3], const double *d_cube, int natom,
                             const double *d_centers, int T, double *d_out, TmpBuf &keep,
                             cudaStream_t s) {
  Axis ax[3];
  for (int d = 0; d < 3; ++d) DAGE_TRY(make_axis(grid[d], ax[d]));
  for (int d = 1; d < 3; ++d)
    if (ax[d].nlip != ax[0].nlip || ax[d].grid_type != ax[0].grid_type)
      return fail(DAGE_E_UNSUPPORTED, "cube contaminants: the axes need one nlip and grid type");
  if (ax[0].nlip > 8) return fail(DAGE_E_UNSUPPORTED, "cube contaminants: nlip <= 8");
  LipBasis L;
  DAGE_TRY(make_lip_basis(ax[0].nlip, ax[0].grid_type, L));
  size_t tot = L.coeff.size();
  for (int d = 0; d < 3; ++d) tot += 2 * (size_t)ax[d].ncell;
  std::vector<double> host;
  host.reserve(tot);
  host.insert(host.end(), L.coeff.begin(), L.coeff.end());
  size_t off[3];
  for (int d = 0; d < 3; ++d) {
    off[d] = host.size();
    host.insert(host.end(), ax[d].celld.begin(), ax[d].celld.end());
    host.insert(host.end(), ax[d].h.begin(), ax[d].h.end());
  }
  DAGE_TRY(keep.alloc(sizeof(double) * host.size()));
  DAGE_CUDA_TRY(cudaMemcpyAsync(keep.ptr, host.data(), sizeof(double) * host.size(),
                                cudaMemcpyHostToDevice, s));
  const double *base = keep.as<double>();
  CubeAxes A;
  for (int d = 0; d < 3; ++d) {
    A.ax[d].celld = base + off[d];
    A.ax[d].h = base + off[d] + ax[d].ncell;
    A.ax[d].qmin = ax[d].points.front();
    A.ax[d].qmax = ax[d].points.back();
    A.ax[d].ncell = ax[d].ncell;
  }
  cube_contaminants_kernel<<<natom, 64, 0, s>>>(A, base, ax[0].nlip, L.first, d_centers, d_cube,
                                                 ax[0].n(), ax[1].n(), T, d_out);
  DAGE_CUDA_TRY(cudaGetLastError());
  return 0;
}

// Taylor bubbles from device contaminant arrays (either may be null).
int make_taylor_impl(const dage_bubbles *b, const double *d_cb, const double *d_cc, int T,
                     bool exact, dage_bubbles **out) {
  TaylorTables tt;
  DAGE_TRY(taylor_tables(T, exact, tt));
  const int lnew = std::max(b->lmax, T), Nn = (lnew + 1) * (lnew + 1);
  std::vector<int> np(b->natom), poff(b->natom + 1, 0);
  for (int a = 0; a < b->natom; ++a) {
    np[a] = b->radial[a].ncell * (b->nlip - 1) + 1;
    poff[a + 1] = poff[a] + np[a];
  }
  const int total = poff[b->natom];
  const size_t nout = (size_t)Nn * total;
  TmpBuf ints, dbls, d_out;
  std::vector<int> hi;
  hi.insert(hi.end(), np.begin(), np.end());
  hi.insert(hi.end(), poff.begin(), poff.end());
  const size_t o_kabs = hi.size();
  hi.insert(hi.end(), tt.kabs.begin(), tt.kabs.end());
  const size_t o_sptr = hi.size();
  hi.insert(hi.end(), tt.sptr.begin(), tt.sptr.end());
  const size_t o_slm = hi.size();
  hi.insert(hi.end(), tt.slm.begin(), tt.slm.end());
  std::vector<double> hd(tt.fac);
  const size_t o_sval = hd.size();
  hd.insert(hd.end(), tt.sval.begin(), tt.sval.end());
  DAGE_TRY(ints.alloc(sizeof(int) * hi.size()));
  DAGE_TRY(dbls.alloc(sizeof(double) * std::max<size_t>(hd.size(), 1)));
  DAGE_TRY(d_out.alloc(sizeof(double) * nout));
  DAGE_CUDA_TRY(cudaMemcpy(ints.ptr, hi.data(), sizeof(int) * hi.size(), cudaMemcpyHostToDevice));
  DAGE_CUDA_TRY(cudaMemcpy(dbls.ptr, hd.data(), sizeof(double) * hd.size(), cudaMemcpyHostToDevice));
  DAGE_CUDA_TRY(cudaMemset(d_out.ptr, 0, sizeof(double) * nout));
  const int *I = ints.as<int>();
  const double *D = dbls.as<double>();
  make_taylor_kernel<<<(total + 127) / 128, 128>>>(
      b->rpts.as<double>(), I, I + b->natom, b->natom, d_cb, d_cc, tt.NC, I + o_kabs, D,
      I + o_sptr, I + o_slm, D + o_sval, Nn, b->k, d_out.as<double>());
  DAGE_CUDA_TRY(cudaGetLastError());
  std::vector<double> f(nout);
  DAGE_CUDA_TRY(cudaMemcpy(f.data(), d_out.ptr, sizeof(double) * nout, cudaMemcpyDeviceToHost));
  return dage_bubbles_create(b->natom, b->centers.data(), b->radial.data(), lnew, b->k, f.data(),
                             out);
}

}  // namespace
}  // namespace dage

using namespace dage;

extern "C" {

int dage_bubbles_contaminants(const dage_bubbles *b, int tmax, double *contams) {
  clear_error();
  if (!b || !contams) return fail(DAGE_E_INVALID, "null argument");
  if (tmax < 0 || tmax > kMaxTaylor) return fail(DAGE_E_UNSUPPORTED, "need 0 <= tmax <= 3");
  DAGE_CUDA_TRY(cudaSetDevice(b->device));
  const size_t n = (size_t)b->natom * ncart(tmax);
  TmpBuf d;
  DAGE_TRY(d.alloc(sizeof(double) * n));
  DAGE_TRY(bubble_contaminants_launch(b, tmax, d.as<double>(), 0));
  DAGE_CUDA_TRY(cudaMemcpy(contams, d.ptr, sizeof(double) * n, cudaMemcpyDeviceToHost));
  return 0;
}

int dage_cube_contaminants(const dage_grid1d grid[3], const double *cube, int natom,
                           const double *centers, int tmax, unsigned flags, double *contams) {
  clear_error();
  if (!grid || !cube || !centers || !contams || natom < 1)
    return fail(DAGE_E_INVALID, "null argument or natom < 1");
  if (tmax < 0 || tmax > kMaxTaylor) return fail(DAGE_E_UNSUPPORTED, "need 0 <= tmax <= 3");
  Axis ax[3];
  for (int d = 0; d < 3; ++d) DAGE_TRY(make_axis(grid[d], ax[d]));
  const size_t npts = (size_t)ax[0].n() * ax[1].n() * ax[2].n();
  const size_t n = (size_t)natom * ncart(tmax);
  TmpBuf d_out, d_cent, d_cube, keep;
  DAGE_TRY(d_out.alloc(sizeof(double) * n));
  DAGE_TRY(d_cent.alloc(sizeof(double) * 3 * natom));
  DAGE_CUDA_TRY(cudaMemcpy(d_cent.ptr, centers, sizeof(double) * 3 * natom, cudaMemcpyHostToDevice));
  const double *dc = cube;
  if (!(flags & DAGE_DEVICE_PTRS)) {
    DAGE_TRY(d_cube.alloc(sizeof(double) * npts));
    DAGE_CUDA_TRY(cudaMemcpy(d_cube.ptr, cube, sizeof(double) * npts, cudaMemcpyHostToDevice));
    dc = d_cube.as<double>();
  }
  DAGE_TRY(cube_contaminants_launch(grid, dc, natom, d_cent.as<double>(), tmax, d_out.as<double>(),
                                    keep, 0));
  DAGE_CUDA_TRY(cudaMemcpy(contams, d_out.ptr, sizeof(double) * n, cudaMemcpyDeviceToHost));
  return 0;
}

int dage_bubbles_make_taylor(const dage_bubbles *b, const double *bubble_contams,
                             const double *cube_contams, int tmax, unsigned flags,
                             dage_bubbles **out) {
  clear_error();
  if (!b || !out) return fail(DAGE_E_INVALID, "null argument");
  *out = nullptr;
  if (tmax < 0 || tmax > kMaxTaylor) return fail(DAGE_E_UNSUPPORTED, "need 0 <= tmax <= 3");
  if (std::max(b->lmax, tmax) > 12) return fail(DAGE_E_INVALID, "Taylor bubbles: lmax <= 12");
  DAGE_CUDA_TRY(cudaSetDevice(b->device));
  const size_t n = (size_t)b->natom * ncart(tmax);
  TmpBuf cb, cc;
  if (bubble_contams) {
    DAGE_TRY(cb.alloc(sizeof(double) * n));
    DAGE_CUDA_TRY(cudaMemcpy(cb.ptr, bubble_contams, sizeof(double) * n, cudaMemcpyHostToDevice));
  }
  if (cube_contams) {
    DAGE_TRY(cc.alloc(sizeof(double) * n));
    DAGE_CUDA_TRY(cudaMemcpy(cc.ptr, cube_contams, sizeof(double) * n, cudaMemcpyHostToDevice));
  }
  return make_taylor_impl(b, cb.as<double>(), cc.as<double>(), tmax,
                          (flags & DAGE_TAYLOR_EXACT) != 0, out);
}

int dage_bubbles_taylor(const dage_bubbles *b, const dage_grid1d grid[3], const double *cube,
                        int tmax, unsigned flags, dage_bubbles **out) {
  clear_error();
  if (!b || !out) return fail(DAGE_E_INVALID, "null argument");
  *out = nullptr;
  if (cube && !grid) return fail(DAGE_E_INVALID, "a cube needs its grid");
  if (tmax < 0 || tmax > kMaxTaylor) return fail(DAGE_E_UNSUPPORTED, "need 0 <= tmax <= 3");
  if (std::max(b->lmax, tmax) > 12) return fail(DAGE_E_INVALID, "Taylor bubbles: lmax <= 12");
  DAGE_CUDA_TRY(cudaSetDevice(b->device));
  const size_t n = (size_t)b->natom * ncart(tmax);
  TmpBuf cb, cc, d_cent, d_cube, keep;
  if (!(flags & DAGE_TAYLOR_IGNORE_BUBBLES)) {
    DAGE_TRY(cb.alloc(sizeof(double) * n));
    DAGE_TRY(bubble_contaminants_launch(b, tmax, cb.as<double>(), 0));
  }
  if (cube) {
    Axis ax[3];
    for (int d = 0; d < 3; ++d) DAGE_TRY(make_axis(grid[d], ax[d]));
    const size_t npts = (size_t)ax[0].n() * ax[1].n() * ax[2].n();
    const double *dc = cube;
    if (!(flags & DAGE_DEVICE_PTRS)) {
      DAGE_TRY(d_cube.alloc(sizeof(double) * npts));
      DAGE_CUDA_TRY(cudaMemcpy(d_cube.ptr, cube, sizeof(double) * npts, cudaMemcpyHostToDevice));
      dc = d_cube.as<double>();
    }
    DAGE_TRY(cc.alloc(sizeof(double) * n));
    DAGE_TRY(d_cent.alloc(sizeof(double) * 3 * b->natom));
    DAGE_CUDA_TRY(cudaMemcpy(d_cent.ptr, b->centers.data(), sizeof(double) * 3 * b->natom,
                             cudaMemcpyHostToDevice));
    DAGE_TRY(cube_contaminants_launch(grid, dc, b->natom, d_cent.as<double>(), tmax,
                                      cc.as<double>(), keep, 0));
  }
  return make_taylor_impl(b, cb.as<double>(), cc.as<double>(), tmax,
                          (flags & DAGE_TAYLOR_EXACT) != 0, out);
}

int dage_bubbles_multiply_taylor(const dage_bubbles *b1, const dage_bubbles *b2,
                                 const dage_bubbles *t1, const dage_bubbles *t2, unsigned flags,
                                 dage_bubbles **out) {
  clear_error();
  if (!b1 || !b2 || !t1 || !t2 || !out) return fail(DAGE_E_INVALID, "null argument");
  *out = nullptr;
  for (const dage_bubbles *x : {b2, t1, t2})
    if (!same_layout(b1, x))
      return fail(DAGE_E_UNSUPPORTED,
                  "Taylor product: the four sets need the same atoms and radial grids");
  if (t1->k != b1->k || t2->k != b2->k)
    return fail(DAGE_E_UNSUPPORTED, "Taylor product: each Taylor set needs its bubbles' k");
  if (t1->lmax < b1->lmax || t2->lmax < b2->lmax)
    return fail(DAGE_E_INVALID, "Taylor product: a Taylor set's lmax is below its bubbles'");
  const int lr = b1->lmax + b2->lmax;
  if (lr > 12) return fail(DAGE_E_INVALID, "Taylor product: lmax1 + lmax2 > 12");
  DAGE_CUDA_TRY(cudaSetDevice(b1->device));
  const std::vector<ProdTerm> terms =
      product_table(std::max(b1->lmax, b2->lmax), lr, (flags & DAGE_PRODUCT_COMPLETE) != 0);
  const int Nr = (lr + 1) * (lr + 1);
  std::vector<int> hi(2 * b1->natom + 1, 0);
  int *np = hi.data(), *poff = hi.data() + b1->natom;
  for (int a = 0; a < b1->natom; ++a) {
    np[a] = b1->radial[a].ncell * (b1->nlip - 1) + 1;
    poff[a + 1] = poff[a] + np[a];
  }
  const int total = poff[b1->natom];
  const size_t nout = (size_t)Nr * total;
  TmpBuf d_terms, d_ints, d_out;
  DAGE_TRY(d_terms.alloc(sizeof(ProdTerm) * std::max<size_t>(terms.size(), 1)));
  DAGE_TRY(d_ints.alloc(sizeof(int) * hi.size()));
  DAGE_TRY(d_out.alloc(sizeof(double) * nout));
  DAGE_CUDA_TRY(cudaMemcpy(d_terms.ptr, terms.data(), sizeof(ProdTerm) * terms.size(),
                           cudaMemcpyHostToDevice));
  DAGE_CUDA_TRY(cudaMemcpy(d_ints.ptr, hi.data(), sizeof(int) * hi.size(), cudaMemcpyHostToDevice));
  DAGE_CUDA_TRY(cudaMemset(d_out.ptr, 0, sizeof(double) * nout));
  bubbles_product_taylor_kernel<<<(total + 127) / 128, 128>>>(
      b1->fraw.as<double>(), b1->N, t1->fraw.as<double>(), t1->N, b2->fraw.as<double>(), b2->N,
      t2->fraw.as<double>(), t2->N, d_ints.as<int>(), d_ints.as<int>() + b1->natom, b1->natom,
      d_terms.as<ProdTerm>(), (int)terms.size(), Nr, d_out.as<double>());
  DAGE_CUDA_TRY(cudaGetLastError());
  std::vector<double> prod(nout);
  DAGE_CUDA_TRY(cudaMemcpy(prod.data(), d_out.ptr, sizeof(double) * nout, cudaMemcpyDeviceToHost));
  return dage_bubbles_create(b1->natom, b1->centers.data(), b1->radial.data(), lr,
                             b1->k + b2->k, prod.data(), out);
}

int dage_cart2sph_table(int tmax, unsigned flags, int cap, int *kappa_index, int *lm, double *c,
                        int *n) {
  clear_error();
  if (!n) return fail(DAGE_E_INVALID, "null argument");
  if (tmax < 0 || tmax > kMaxTaylor) return fail(DAGE_E_UNSUPPORTED, "need 0 <= tmax <= 3");
  TaylorTables tt;
  DAGE_TRY(taylor_tables(tmax, (flags & DAGE_TAYLOR_EXACT) != 0, tt));
  *n = (int)tt.slm.size();
  if (cap < *n || !kappa_index || !lm || !c) return 0;
  for (int i = 0; i < tt.NC; ++i)
    for (int e = tt.sptr[i]; e < tt.sptr[i + 1]; ++e) {
      kappa_index[e] = i;
      lm[e] = tt.slm[e];
      c[e] = tt.sval[e];
    }
  return 0;
}

}  // extern "C"
