"""ctypes wrapper of the CPU FP64 oracle (oracle/_build/libdage_oracle.so).

TEST INFRASTRUCTURE ONLY: the checker the CUDA product is compared against.
Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.  The product library never loads it.

The routines restate the reference Fortran CPU path (file:line cited in
``dage_oracle.h`` and ``operator_ref.cpp``).  Cubes are numpy arrays in
Fortran order (``order='F'``), shape ``(nx, ny, nz)``, x fastest, matching
the reference's ``cube(x, y, z)``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libdage_oracle.so")
_LIB_1ULP_PATH = os.path.join(_HERE, "_build", "libdage_oracle_1ulp.so")
_libs = {}

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.c_int
_F = ctypes.c_double


def build(force: bool = False) -> str:
    """Compile the oracle with ``make -C oracle`` (make rebuilds what is out
    of date); returns the library path."""
    if force:
        subprocess.run(["make", "-s", "-C", _HERE, "clean"], check=True)
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib(libm_1ulp: bool = False):
    """The oracle library; ``libm_1ulp`` selects the build whose erf/exp
    results are moved by +-1 ulp (see operator_ref.cpp)."""
    path = _LIB_1ULP_PATH if libm_1ulp else _LIB_PATH
    if path not in _libs:
        build()
        L = ctypes.CDLL(path)
        sig = {
            "orc_gauss_quad": (None, [_I, _I, _F, _F, _F, _D, _D]),
            "orc_bessel_i": (None, [_F, _I, _D]),
            "orc_bessel_k": (None, [_F, _I, _D]),
            "orc_aligned_ml": (None, [_D, _I, _I, _D]),
            "orc_rotation": (None, [_D, _I, _D]),
            "orc_helm_m2l": (_I, [_I, _I, _F, _D, _D, _D, _D]),
            "orc_helm_m2l_lsq": (_I, [_I, _I, _F, _D, _D, _D, _D]),
            "orc_helm_m2m": (_I, [_I, _I, _F, _D, _D, _D, _D]),
            "orc_helm_matrix": (_I, [_I, _I, _I, _F, _D, _D, _D]),
            "orc_aligned_mm": (None, [_D, _I, _I, _D]),
            "orc_ref_real_rotation": (None, [_F, _F, _F, _I, _I, _D]),
            "orc_helm_box_multipoles": (_I, [_I, _F, _I, _D, _D, _I, _D, _D, _I, _D, _D, _D, _D,
                                             _D]),
            "orc_helm_l2p": (_I, [_I, _F, _D, _D, _I, _D, _I, _D, _I, _D, _D]),
            "orc_gauleg": (None, [_I, _D, _D]),
            "orc_lip_coeffs": (_I, [_I, _I, _D, _D, _D]),
            "orc_lip_integrals": (_I, [_I, _I, _D]),
            "orc_grid1d_points": (_I, [_F, _I, _I, _I, _D, _D, _D]),
            "orc_grid1d_spheres": (_I, [_I, _D, _D, _F, _I, _D, _D]),
            "orc_grid1d_weights": (_I, [_I, _I, _I, _D, _D]),
            "orc_expo_integrals": (None, [_F, _F, _F, _F, _I, _D]),
            "orc_coulomb_matrix": (_I, [_F, _I, _I, _I, _D, _I, _D, _I, _D, _D]),
            "orc_coulomb_border_matrix": (_I, [_F, _I, _I, _I, _D, _I, _D, _I, _D, _D]),
            "orc_transform_cube": (_I, [_I, _I, _I, _I, _I, _I, _I, _D, _D, _D, _D, _F, _D, _D]),
            "orc_integrate_cube": (_F, [_I, _I, _I, _D, _I, _D, _I, _D, _D]),
            "orc_gauss_cube": (None, [_I, _D, _D, _D, _I, _D, _I, _D, _I, _D, _D]),
            "orc_gauss_pot_cube": (None, [_I, _D, _D, _D, _I, _D, _I, _D, _I, _D, _D]),
            "orc_gauss_analytical_energy": (_F, [_I, _D, _D, _D]),
            "orc_gauss_extent": (None, [_I, _D, _D, _F, _D]),
            "orc_solid_harmonics": (None, [_I, _F, _F, _F, _D]),
            "orc_interaction_matrix": (_I, [_I, _D, _D]),
            "orc_translation_matrix": (_I, [_I, _D, _D]),
            "orc_dtpmv_lower_unit": (None, [_I, _D, _D]),
            "orc_box_vector": (None, [_I, _I, ctypes.POINTER(_I)]),
            "orc_box_index": (_I, [ctypes.POINTER(_I), _I]),
            "orc_nearest_neighbors": (_I, [_I, _I, ctypes.POINTER(_I)]),
            "orc_local_farfield": (_I, [_I, _I, ctypes.POINTER(_I)]),
            "orc_box_multipoles": (_I, [_I, _I, _D, _D, _I, _D, _D, _I, _D, _D, _D, _D, _D]),
            "orc_l2p": (_I, [_I, _D, _D, _I, _D, _I, _D, _I, _D, _D]),
            "orc_bubbles_inject": (_I, [_I, _D, ctypes.POINTER(_I), _D, _I, _I, _I, _I, _D, _I, _D,
                                        _I, _D, _I, _D, _F, _D]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _libs[path] = L
    return _libs[path]


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and (a.flags.c_contiguous or a.flags.f_contiguous)
    return a.ctypes.data_as(_D)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


# ---------------------------------------------------------------------------
# Quadrature, LIP basis, grids
# ---------------------------------------------------------------------------
def gauss_quad(nlin=10, nlog=8, tstart=0.0, tlin=2.0, tlog=1.0e3):
    """GaussQuad(nlin, nlog, tlin, tlog, tstart) (gauss.F90:81-122)."""
    n = nlin + nlog
    tp = np.zeros(n)
    tw = np.zeros(n)
    lib().orc_gauss_quad(nlin, nlog, tstart, tlin, tlog, _p(tp), _p(tw))
    return tp, tw


def lip_coeffs(nlip=7, grid_type=1):
    c = np.zeros((nlip, nlip), order="F")
    first = ctypes.c_double()
    last = ctypes.c_double()
    rc = lib().orc_lip_coeffs(nlip, grid_type, _p(c), ctypes.byref(first), ctypes.byref(last))
    if rc:
        raise ValueError("unsupported LIP basis")
    return c, first.value, last.value


def lip_integrals(nlip=7, grid_type=1):
    v = np.zeros(nlip)
    if lib().orc_lip_integrals(nlip, grid_type, _p(v)):
        raise ValueError("unsupported LIP basis")
    return v


@dataclass
class Grid1D:
    """Grid1D (grid.F90:446-534): ``ncell`` LIP cells of ``nlip`` points."""

    qmin: float
    ncell: int
    nlip: int = 7
    grid_type: int = 1
    cell_scales: np.ndarray = field(default=None)

    def __post_init__(self):
        if self.cell_scales is None:
            raise ValueError("cell_scales required")
        self.cell_scales = _f64(np.broadcast_to(self.cell_scales, (self.ncell,)))
        self.points = np.zeros(self.ncell * (self.nlip - 1) + 1)
        self.celld = np.zeros(self.ncell)
        rc = lib().orc_grid1d_points(self.qmin, self.ncell, self.nlip, self.grid_type,
                                     _p(self.cell_scales), _p(self.points), _p(self.celld))
        if rc:
            raise ValueError("unsupported grid")

    @property
    def n(self) -> int:
        return self.ncell * (self.nlip - 1) + 1

    @classmethod
    def equidistant(cls, qmin, ncell, step, nlip=7, grid_type=1):
        return cls(qmin, ncell, nlip, grid_type, np.full(ncell, float(step)))

    @classmethod
    def spheres(cls, centers, radii, step, nlip=7, grid_type=1):
        """Default generator grid (grid.F90:604-640 then :539-564)."""
        c = _f64(centers)
        r = _f64(radii)
        qmin = ctypes.c_double()
        s = ctypes.c_double()
        nc = lib().orc_grid1d_spheres(len(c), _p(c), _p(r), float(step), nlip,
                                      ctypes.byref(qmin), ctypes.byref(s))
        return cls.equidistant(qmin.value, nc, s.value, nlip, grid_type)

    def weights(self) -> np.ndarray:
        w = np.zeros(self.n)
        lib().orc_grid1d_weights(self.ncell, self.nlip, self.grid_type, _p(self.cell_scales), _p(w))
        return w


@dataclass
class Grid3D:
    axes: tuple

    @property
    def shape(self):
        return tuple(a.n for a in self.axes)

    @classmethod
    def cube(cls, qmin, ncell, step, nlip=7, grid_type=1):
        ax = Grid1D.equidistant(qmin, ncell, step, nlip, grid_type)
        return cls((ax, ax, ax))

    @classmethod
    def gauss_default(cls, q, alpha, centers, step=0.2, nlip=7, thres=1e-12, grid_type=1):
        """GaussGenerator_gen_cubegrid (gauss_generator.F90:262-281)."""
        ext = gauss_extent(q, alpha, thres)
        cen = np.asarray(centers, dtype=np.float64).reshape(-1, 3)
        return cls(tuple(Grid1D.spheres(cen[:, d], ext, step, nlip, grid_type) for d in range(3)))


# ---------------------------------------------------------------------------
# Operator matrices and application
# ---------------------------------------------------------------------------
def expo_integrals(a, b, t, p, n=7):
    v = np.zeros(n)
    lib().orc_expo_integrals(a, b, t, p, n, _p(v))
    return v


def coulomb_matrix(grid_in: Grid1D, out_points, tp, border_only=False,
                   libm_1ulp=False) -> np.ndarray:
    """T(i_out, j_in, p) for one axis (exponentials.F90:178-346)."""
    out = _f64(out_points)
    tp = _f64(tp)
    T = np.zeros((len(out), grid_in.n, len(tp)), order="F")
    L = lib(libm_1ulp)
    fn = L.orc_coulomb_border_matrix if border_only else L.orc_coulomb_matrix
    rc = fn(grid_in.qmin, grid_in.ncell, grid_in.nlip, grid_in.grid_type,
            _p(grid_in.cell_scales), len(out), _p(out), len(tp), _p(tp), _p(T))
    if rc:
        raise ValueError("unsupported grid")
    return T


def coulomb_weights(tw):
    """w_p = 2/sqrt(pi) * tw_p (coulomb.F90:150)."""
    return (2.0 / np.sqrt(np.pi)) * np.asarray(tw)


def helmholtz_weights(tp, tw, energy):
    """Helmholtz3D_set_energy (helmholtz3d.F90:411-444)."""
    tw = np.asarray(tw, dtype=np.float64).copy()
    tp = np.asarray(tp, dtype=np.float64)
    if energy < -0.005:
        tw = tw * np.exp(2.0 * energy / (4.0 * tp ** 2))
    return (2.0 / np.sqrt(np.pi)) * tw


def coda_of(tlog):
    """coda = pi / tlog^2 (coulomb.F90:151)."""
    return np.pi / tlog ** 2


def transform_cube(Tx, Ty, Tz, w, rho, coda=0.0) -> np.ndarray:
    """Operator3D_transform_cube CPU branch (function3d.F90:4230-4349)."""
    Tx = np.asfortranarray(Tx, dtype=np.float64)
    Ty = np.asfortranarray(Ty, dtype=np.float64)
    Tz = np.asfortranarray(Tz, dtype=np.float64)
    rho = np.asfortranarray(rho, dtype=np.float64)
    w = _f64(w)
    nox, nix, P = Tx.shape
    noy, niy, _ = Ty.shape
    noz, niz, _ = Tz.shape
    assert rho.shape == (nix, niy, niz)
    V = np.zeros((nox, noy, noz), order="F")
    lib().orc_transform_cube(nix, niy, niz, nox, noy, noz, P, _p(Tx), _p(Ty), _p(Tz), _p(w),
                             float(coda), _p(rho), _p(V))
    return V


def transform_cube_blas(Tx, Ty, Tz, w, rho, coda=0.0, p_subset=None) -> np.ndarray:
    """Same contraction as :func:`transform_cube` with every mode product a
    BLAS DGEMM (numpy's bundled OpenBLAS, all host threads), the way the
    reference's xmatmul reaches DGEMM (xmatrix.F90:72-100).  ``p_subset``
    restricts the t-point loop (used to time a bounded sample)."""
    rho = np.asfortranarray(rho, dtype=np.float64)
    nox, nix, P = Tx.shape
    noy, niy, _ = Ty.shape
    noz, niz, _ = Tz.shape
    r = rho.reshape(-1, order="F").reshape(niz, niy, nix)  # C view (z, y, x)
    V = np.zeros((noz, noy, nox))
    ps = range(P) if p_subset is None else p_subset
    for ip in ps:
        tx = np.ascontiguousarray(Tx[:, :, ip])
        ty = np.ascontiguousarray(Ty[:, :, ip])
        tz = np.ascontiguousarray(Tz[:, :, ip])
        u = (r.reshape(-1, nix) @ tx.T).reshape(niz, niy, nox)
        u = np.matmul(ty, u)  # (noy x niy) @ (niz, niy, nox) -> (niz, noy, nox)
        V.reshape(noz, -1)[...] += w[ip] * (tz @ u.reshape(niz, -1))
    out = np.asfortranarray(V.reshape(-1).reshape((nox, noy, noz), order="F"))
    if coda != 0.0 and out.shape == rho.shape:
        out = out + coda * rho
    return out


def integrate_cube(grid: Grid3D, f) -> float:
    """Integrator_eval (evaluators.F90:1064-1098)."""
    f = np.asfortranarray(f, dtype=np.float64)
    gx, gy, gz = grid.axes
    return lib().orc_integrate_cube(gx.nlip, gx.grid_type, gx.ncell, _p(gx.cell_scales),
                                    gy.ncell, _p(gy.cell_scales), gz.ncell,
                                    _p(gz.cell_scales), _p(f))


# ---------------------------------------------------------------------------
# Test densities
# ---------------------------------------------------------------------------
def slater_dens(zeta, l, r):
    """Radial Slater density 2 zeta^(l+3) (1+2l) / (pi (l+2)!) r^l e^(-2 zeta r)
    (slater_generator.F90:453-464, slater_dens)."""
    norm = 2.0 * zeta ** (l + 3) * (1.0 + 2 * l) / np.pi / float(np.prod(np.arange(2, l + 3)))
    return norm * np.asarray(r, dtype=np.float64) ** l * np.exp(-2.0 * zeta * np.asarray(r))


def slater_analytical_energy(coeffs, expos, centers) -> float:
    """Self-interaction of Slater s-densities (slater_analytical_energy,
    analytical.F90:70-188, without periodic images): sum_i U_i + 2 sum_{i<j}
    U_ij, U_i = q^2 5 zeta / 8, U_ij the closed form for equal or unequal
    exponents (:155-187)."""
    q = [float(x) for x in coeffs]
    z = [float(x) for x in expos]
    C = np.asarray(centers, dtype=np.float64).reshape(-1, 3)

    def uij(zi, zj, qi, qj, r):
        if r <= 1e-14:
            return qi * qj * zi * zj * (zi ** 2 + 3.0 * zi * zj + zj ** 2) / (zi + zj) ** 3
        if zi == zj:
            ei = np.exp(-2.0 * zi * r)
            f = zi * r
            return qi * qj * (1.0 - ei * (1.0 + 11.0 / 8.0 * f + 3.0 / 4.0 * f ** 2
                                          + 1.0 / 6.0 * f ** 3)) / r
        f = 1.0 / (zi * zi - zj * zj)
        ei = np.exp(-2.0 * zi * r)
        ej = np.exp(-2.0 * zj * r)
        return (qi * qj / r) * (1.0 - zi ** 4 * zj ** 4 * f ** 2 * (ei * (1.0 + zi * r) / zi ** 4
                                                                     - ej * (1.0 + zj * r) / zj ** 4)
                                - 2.0 * zi ** 4 * zj ** 4 * f ** 3 * (ei / zi ** 2 - ej / zj ** 2))

    E = 0.0
    for i in range(len(q)):
        E += q[i] ** 2 * 5.0 / 8.0 * z[i]
        for j in range(i + 1, len(q)):
            E += 2.0 * uij(z[i], z[j], q[i], q[j], float(np.sqrt(((C[i] - C[j]) ** 2).sum())))
    return float(E)


def radial_grid_charge(z, n0=100, nlip=7, r_max=20.0) -> Grid1D:
    """Grid1D_init_radial (grid.F90:568-599): int(n0 z^(1/4)) cells whose ends
    follow x_i = c / ((r_max + c) / (i dx) - 1), c = 8 z^(-3/2), dx = r_max /
    ncell; equidistant points inside each cell."""
    ncell = int(n0 * z ** 0.25)
    const = 8.0 * z ** (-1.5)
    dx = r_max / ncell
    x0, scales = 0.0, []
    for i in range(1, ncell + 1):
        x1 = const / ((r_max + const) / (i * dx) - 1.0)
        scales.append((x1 - x0) / (nlip - 1))
        x0 = x1
    return Grid1D(0.0, ncell, nlip, 1, np.array(scales))


def gauss_extent(q, alpha, thres=1e-12):
    q = _f64(q)
    a = _f64(alpha)
    e = np.zeros(len(q))
    lib().orc_gauss_extent(len(q), _p(q), _p(a), thres, _p(e))
    return e


def gauss_cube(grid: Grid3D, q, alpha, centers) -> np.ndarray:
    q = _f64(q)
    a = _f64(alpha)
    c = _f64(np.asarray(centers, dtype=np.float64).reshape(-1, 3))
    gx, gy, gz = grid.axes
    out = np.zeros(grid.shape, order="F")
    lib().orc_gauss_cube(len(q), _p(q), _p(a), _p(c), gx.n, _p(gx.points), gy.n,
                         _p(gy.points), gz.n, _p(gz.points), _p(out))
    return out


def gauss_pot_cube(grid: Grid3D, q, alpha, centers) -> np.ndarray:
    q = _f64(q)
    a = _f64(alpha)
    c = _f64(np.asarray(centers, dtype=np.float64).reshape(-1, 3))
    gx, gy, gz = grid.axes
    out = np.zeros(grid.shape, order="F")
    lib().orc_gauss_pot_cube(len(q), _p(q), _p(a), _p(c), gx.n, _p(gx.points), gy.n,
                             _p(gy.points), gz.n, _p(gz.points), _p(out))
    return out


def gauss_analytical_energy(q, alpha, centers) -> float:
    q = _f64(q)
    a = _f64(alpha)
    c = _f64(np.asarray(centers, dtype=np.float64).reshape(-1, 3))
    return lib().orc_gauss_analytical_energy(len(q), _p(q), _p(a), _p(c))


# ---------------------------------------------------------------------------
# Whole-operator helpers
# ---------------------------------------------------------------------------
def coulomb_operator_matrices(grid_in: Grid3D, grid_out: Grid3D, tp, libm_1ulp=False):
    """make_Coulomb3D_matrices (exponentials.F90:602-639), all three axes in
    the T(i_out, j_in, p) orientation."""
    return tuple(coulomb_matrix(grid_in.axes[d], grid_out.axes[d].points, tp,
                                libm_1ulp=libm_1ulp) for d in range(3))


def coulomb_apply(grid: Grid3D, rho, quad=(10, 8, 0.0, 2.0, 1.0e3), coda=True, weights=None,
                  libm_1ulp=False):
    """V = Coulomb3D(grid) .apply. rho (cube part), CPU semantics."""
    nlin, nlog, tstart, tlin, tlog = quad
    tp, tw = gauss_quad(nlin, nlog, tstart, tlin, tlog)
    Tx, Ty, Tz = coulomb_operator_matrices(grid, grid, tp, libm_1ulp)
    w = coulomb_weights(tw) if weights is None else weights
    return transform_cube(Tx, Ty, Tz, w, rho, coda_of(tlog) if coda else 0.0)


def selfint(grid: Grid3D, rho, quad=(10, 8, 0.0, 2.0, 1.0e3), coda=True) -> float:
    """rho .dot. (Coulomb3D .apply. rho) as tests/gauss_test.F90 computes it."""
    V = coulomb_apply(grid, rho, quad, coda)
    return integrate_cube(grid, rho * V)


def matrix_noise_envelope(T: np.ndarray, T1: np.ndarray, band: int = 6) -> np.ndarray:
    """Per-entry tolerance for comparing operator matrices from two FP64
    implementations: for each t-point slice and each band of |i - j|
    (``band`` points wide) the largest |T - T1| inside the band, where T1
    comes from the +-1 ulp oracle.  The reference's closed-form integrals
    (exponentials.F90:695-1297) cancel heavily for t*h just above 0.1, so
    their last bits -- and the matrices -- move by this much with the libm."""
    no, ni, P = T.shape
    I, J = np.meshgrid(np.arange(no), np.arange(ni), indexing="ij")
    bands = np.abs(I - J) // band
    env = np.zeros_like(T)
    d = np.abs(T - T1)
    for p in range(P):
        dp = d[:, :, p]
        mx = np.zeros(bands.max() + 1)
        np.maximum.at(mx, bands.ravel(), dp.ravel())
        # noise grows with distance: take the running max over nearer bands too
        env[:, :, p] = np.maximum.accumulate(mx)[bands]
    return env


# ---------------------------------------------------------------------------
# GBFMM pieces
# ---------------------------------------------------------------------------
def solid_harmonics(lmax, xyz) -> np.ndarray:
    """Racah-normalised real regular solid harmonics, lm = l(l+1)+m."""
    out = np.zeros((lmax + 1) ** 2)
    lib().orc_solid_harmonics(lmax, float(xyz[0]), float(xyz[1]), float(xyz[2]), _p(out))
    return out


def interaction_matrix(lmax, d) -> np.ndarray:
    """M2L matrix T(d) (multipole.F90:81-303): L_i += T(c_j - c_i) q_j."""
    N = (lmax + 1) ** 2
    T = np.zeros((N, N), order="F")
    if lib().orc_interaction_matrix(lmax, _p(_f64(d)), _p(T)):
        raise ValueError("interaction matrix undefined at d = 0")
    return T


def translation_matrix(lmax, d) -> np.ndarray:
    """M2M/L2L matrix (multipole.F90:344-515), packed lower triangle."""
    N = (lmax + 1) ** 2
    W = np.zeros(N * (N + 1) // 2)
    lib().orc_translation_matrix(lmax, _p(_f64(d)), _p(W))
    return W


def translate(lmax, q, frm, to) -> np.ndarray:
    """TranslationMatrix_apply: q expanded about `frm` -> about `to`."""
    W = translation_matrix(lmax, np.asarray(frm, float) - np.asarray(to, float))
    x = _f64(q).copy()
    lib().orc_dtpmv_lower_unit(len(x), _p(W), _p(x))
    return x


def translation_dense(lmax, d) -> np.ndarray:
    """The translation matrix W(d) as a dense lower-triangular matrix with
    unit diagonal (dtpmv('L', *, 'U') semantics of TranslationMatrix)."""
    N = (lmax + 1) ** 2
    Wp = translation_matrix(lmax, d)
    W = np.eye(N)
    k = 0
    for j in range(N):  # packed by columns
        k += 1  # the (unit) diagonal element
        for i in range(j + 1, N):
            W[i, j] = Wp[k]
            k += 1
    return W


def translate_local(lmax, L, child, parent) -> np.ndarray:
    """L2L of GBFMMCoulomb3D_translate_potential (gbfmm_coulomb3d.F90:1565-1621):
    the transposed translation matrix of the displacement child - parent
    applied to the parent's local expansion."""
    W = translation_dense(lmax, np.asarray(child, float) - np.asarray(parent, float))
    return W.T @ _f64(L)


_IP = ctypes.POINTER(ctypes.c_int)


def box_vector(ibox, level):
    v = (ctypes.c_int * 3)()
    lib().orc_box_vector(ibox, level, v)
    return tuple(v)


def box_index(v, level):
    a = (ctypes.c_int * 3)(*v)
    return lib().orc_box_index(a, level)


def nearest_neighbors(ibox, level):
    out = (ctypes.c_int * 26)()
    n = lib().orc_nearest_neighbors(ibox, level, out)
    return list(out[:n])


def local_farfield(ibox, level):
    out = (ctypes.c_int * 1024)()
    n = lib().orc_local_farfield(ibox, level, out)
    return list(out[:n])


def local_farfield_adaptive(ibox, level):
    """The adaptive mode's far field of box `ibox` of `level`
    (GBFMMParallelInfo_get_local_farfield_indices evaluation types 1 and 2,
    gbfmm_parallel_info.F90:827-983, used at gbfmm_coulomb3d.F90:1386-1433):
    (boxes of `level`: the children of the parent's neighbours that contain
    one of ibox's nearest neighbours, minus those neighbours; boxes of
    level - 1: the parent's other neighbours)."""
    if level < 2:
        return [], []
    nn = set(nearest_neighbors(ibox, level))
    partial, whole = [], []
    for p in nearest_neighbors((ibox - 1) // 8 + 1, level - 1):
        kids = range((p - 1) * 8 + 1, p * 8 + 1)
        if any(c in nn for c in kids):
            partial += [c for c in kids if c not in nn]
        else:
            whole.append(p)
    return partial, whole


def box_multipoles(lmax, px, wx, py, wy, pz, wz, cube_sub, center):
    q = np.zeros((lmax + 1) ** 2)
    c = np.asfortranarray(cube_sub, dtype=np.float64)
    px, wx, py, wy, pz, wz = (_f64(a) for a in (px, wx, py, wy, pz, wz))
    lib().orc_box_multipoles(lmax, len(px), _p(px), _p(wx), len(py), _p(py), _p(wy), len(pz),
                             _p(pz), _p(wz), _p(c), _p(_f64(center)), _p(q))
    return q


def l2p(lmax, L, center, px, py, pz, out):
    """out += sum_lm L_lm S_lm(r - center) over the product grid."""
    px, py, pz = (_f64(a) for a in (px, py, pz))
    assert out.flags.f_contiguous and out.shape == (len(px), len(py), len(pz))
    lib().orc_l2p(lmax, _p(_f64(L)), _p(_f64(center)), len(px), _p(px), len(py), _p(py),
                  len(pz), _p(pz), _p(out))
    return out


def bessel_i(x, lmax):
    """i_0..i_lmax(x) (helmholtz3d.F90:879-971)."""
    out = np.zeros(lmax + 1)
    lib().orc_bessel_i(float(x), lmax, _p(out))
    return out


def bessel_k(x, lmax):
    """k_0..k_lmax(x), k_0 = (pi/2) e^-x / x (helmholtz3d.F90:1133-1174)."""
    out = np.zeros(lmax + 1)
    lib().orc_bessel_k(float(x), lmax, _p(out))
    return out


def helm_box_multipoles(lmax, kappa, px, wx, py, wy, pz, wz, cube_sub, center):
    """Helmholtz box moments sum rho w i_l(kappa r) Y_lm (gbfmm_helmholtz3d.F90:1491-1577)."""
    q = np.zeros((lmax + 1) ** 2)
    c = np.asfortranarray(cube_sub, dtype=np.float64)
    px, wx, py, wy, pz, wz = (_f64(a) for a in (px, wx, py, wy, pz, wz))
    lib().orc_helm_box_multipoles(lmax, float(kappa), len(px), _p(px), _p(wx), len(py), _p(py),
                                  _p(wy), len(pz), _p(pz), _p(wz), _p(c), _p(_f64(center)), _p(q))
    return q


def helm_m2l(lmax, kappa, M, src, dst, lin=None, least_squares=False):
    """Local expansion at dst of the Helmholtz multipoles M at src
    (HelmholtzMultipoleConverter, helmholtz_multipole_tools.F90:172-511),
    rotating with the reference's recursions (:911-1200); least_squares:
    with the independent least-squares rotation instead."""
    lin = lmax if lin is None else lin
    L = np.zeros((lmax + 1) ** 2)
    fn = lib().orc_helm_m2l_lsq if least_squares else lib().orc_helm_m2l
    rc = fn(lmax, lin, float(kappa), _p(_f64(M)), _p(_f64(src)), _p(_f64(dst)), _p(L))
    if rc:
        raise ValueError("zero translation distance")
    return L


def helm_m2m(lmax, kappa, M, src, dst):
    """Helmholtz multipoles M about src moved to dst (the reference's
    HelmholtzMultipoleTranslator, helmholtz_multipole_tools.F90:172-278 and
    :338-378, first-kind Bessel functions and the coaxial recurrence
    :513-588; rotations by the reference's recursions, repaired)."""
    out = np.zeros((lmax + 1) ** 2)
    rc = lib().orc_helm_m2m(lmax, lmax, float(kappa), _p(_f64(M)), _p(_f64(src)), _p(_f64(dst)),
                            _p(out))
    if rc:
        raise ValueError("zero translation distance")
    return out


_HELM_MATS = {}


def helm_matrix(kind, lmax, kappa, src, dst):
    """Matrix (N x N, column k = image of unit input k) of the converter
    (kind "m2l") or the translator (kind "m2m") from src to dst; cached per
    displacement."""
    d = np.asarray(dst, dtype=np.float64) - np.asarray(src, dtype=np.float64)
    key = (kind, lmax, float(kappa), tuple(np.round(d, 12)))
    T = _HELM_MATS.get(key)
    if T is None:
        N = (lmax + 1) ** 2
        out = np.zeros(N * N)
        rc = lib().orc_helm_matrix(0 if kind == "m2l" else 1, lmax, lmax, float(kappa),
                                   _p(np.zeros(3)), _p(_f64(d)), _p(out))
        if rc:
            raise ValueError("zero translation distance")
        T = out.reshape(N, N).T.copy()  # T[i, k]
        _HELM_MATS[key] = T
    return T


def helm_l2l(lmax, kappa, Lp, parent, child):
    """Local expansion of the child box from its parent's.  The reference has
    no Helmholtz L2L (its level loop, gbfmm_helmholtz3d.F90:789-937, adds
    every level's local expansions into the finest level's box slots about
    the wrong centres); this is the translation the moments' M2M implies:
    with q(parent) = W q(child) for the regular basis i_l Y_lm and the L2P
    factor (2l+1) of local expansions (:1019-1105), L(child)_i =
    sum_j W_ji (2 l_j + 1) L(parent)_j / (2 l_i + 1)."""
    W = helm_matrix("m2m", lmax, kappa, child, parent)
    ls = np.repeat(np.arange(lmax + 1), 2 * np.arange(lmax + 1) + 1)
    c = 2.0 * ls + 1.0
    return (W.T @ (c * Lp)) / c


def _far_field_levels_helm(plan, q_fine, lmax, kappa, adaptive=False):
    """Multi-level Helmholtz far field: the levels of _far_field_levels with
    the reference's Helmholtz M2M (translate_multipoles, gbfmm_helmholtz3d.F90:
    598-601, 1223-1278), the Helmholtz converter at every level (and, in the
    adaptive mode, from whole parent-level boxes, :811-937) and helm_l2l."""
    N = (lmax + 1) ** 2
    top = plan.level
    q = {top: q_fine}
    for lev in range(top - 1, 0 if adaptive else 1, -1):
        nb = 8 ** lev
        ql = np.zeros((N, nb))
        for p in range(1, nb + 1):
            cp = plan.center_at(p, lev)
            for c in range((p - 1) * 8 + 1, p * 8 + 1):
                ql[:, p - 1] += helm_matrix("m2m", lmax, kappa, plan.center_at(c, lev + 1), cp) @ \
                    q[lev + 1][:, c - 1]
        q[lev] = ql
    Lprev = None
    for lev in range(2, top + 1):
        nb = 8 ** lev
        Ll = np.zeros((N, nb))
        for i in range(1, nb + 1):
            ci = plan.center_at(i, lev)
            if Lprev is not None:
                par = (i - 1) // 8 + 1
                Ll[:, i - 1] += helm_l2l(lmax, kappa, Lprev[:, par - 1], plan.center_at(par, lev - 1), ci)
            if adaptive:
                partial, whole = local_farfield_adaptive(i, lev)
                srcs = [(j, lev) for j in partial] + [(j, lev - 1) for j in whole]
            else:
                srcs = [(j, lev) for j in local_farfield(i, lev)]
            for j, lj in srcs:
                Ll[:, i - 1] += helm_matrix("m2l", lmax, kappa, plan.center_at(j, lj), ci) @ q[lj][:, j - 1]
        Lprev = Ll
    return Lprev


def ref_real_rotation(alpha, beta, gamma, lmax, repaired=True):
    """The reference's real spherical-harmonic rotation coefficients
    (get_real_spherical_harmonic_rotation_coefficients,
    helmholtz_multipole_tools.F90:911-1001): a list over l of (2l+1, 2l+1)
    arrays [m' + l, m + l].  repaired=False: exactly as the reference computes
    them, with its single-precision sqrt(2.0) and the 0/0 of its eq. 68 step."""
    out = np.zeros(sum((2 * l + 1) ** 2 for l in range(lmax + 1)))
    lib().orc_ref_real_rotation(float(alpha), float(beta), float(gamma), lmax, int(repaired),
                                _p(out))
    blocks, off = [], 0
    for l in range(lmax + 1):
        w = 2 * l + 1
        blocks.append(out[off:off + w * w].reshape(w, w))
        off += w * w
    return blocks


def helm_l2p(lmax, kappa, L, center, px, py, pz, out):
    """out += 8 kappa sum (2l+1)/(4 pi) i_l(kappa r) Y_lm L_lm
    (gbfmm_helmholtz3d.F90:1019-1105)."""
    px, py, pz = (_f64(a) for a in (px, py, pz))
    assert out.flags.f_contiguous and out.shape == (len(px), len(py), len(pz))
    lib().orc_helm_l2p(lmax, float(kappa), _p(_f64(L)), _p(_f64(center)), len(px), _p(px),
                       len(py), _p(py), len(pz), _p(pz), _p(out))
    return out


def subgrid(g1: Grid1D, c0: int, c1: int) -> Grid1D:
    """Cells c0..c1 (1-based, inclusive) of an axis as a grid of its own
    (Grid3D_get_subgrid: the same points and cell steps)."""
    return Grid1D(float(g1.points[(c0 - 1) * (g1.nlip - 1)]), c1 - c0 + 1, g1.nlip,
                  g1.grid_type, g1.cell_scales[c0 - 1:c1])


class GBFMMPlan:
    """Octree box bookkeeping of GBFMMParallelInfo / GBFMMCoulomb3D for one
    grid (src/gbfmm/gbfmm_parallel_info.F90, gbfmm_coulomb3d.F90:417-508):
    boxes at `maxlevel` (2^maxlevel per axis), near-field cell ranges (box
    plus its nearest neighbours), local far-field lists and the points each
    box owns (its last point per axis belongs to the next box unless it is
    the grid's last point).

    Cells per box: ncell // 2^maxlevel, as the reference's integer division
    (gbfmm_parallel_info.F90:1072-1084) when it divides evenly.  When it does
    not, the reference leaves the trailing cells in no box; the policy shared
    by this oracle and the GPU code gives the first (ncell mod 2^maxlevel)
    boxes along the axis one extra cell and centres each box on the midpoint
    of its points."""

    def __init__(self, grid: Grid3D, maxlevel: int = 2):
        self.grid = grid
        self.level = maxlevel
        self.nb = 2 ** maxlevel
        self.nbox = self.nb ** 3
        self.ranges = [(a.points[0], a.points[-1]) for a in grid.axes]
        self.vec = [box_vector(i, maxlevel) for i in range(1, self.nbox + 1)]

    def _axis_cells(self, d, v):
        """1-based (first, last) cell of box position v along axis d."""
        nc = self.grid.axes[d].ncell
        base, rem = divmod(nc, self.nb)
        c0 = v * base + min(v, rem)
        return c0 + 1, c0 + base + (1 if v < rem else 0)

    def cells(self, ibox):
        v = self.vec[ibox - 1]
        return [self._axis_cells(d, v[d]) for d in range(3)]

    def near_cells(self, ibox):
        v = self.vec[ibox - 1]
        return [(self._axis_cells(d, max(v[d] - 1, 0))[0],
                 self._axis_cells(d, min(v[d] + 1, self.nb - 1))[1]) for d in range(3)]

    def center(self, ibox):
        v = self.vec[ibox - 1]
        c = np.zeros(3)
        for d in range(3):
            a = self.grid.axes[d]
            if a.ncell % self.nb == 0:  # gbfmm_parallel_info.F90:1290-1299
                c[d] = self.ranges[d][0] + (v[d] + 0.5) * ((self.ranges[d][1] - self.ranges[d][0]) / self.nb)
            else:
                (p0, p1) = self.points(ibox)[d]
                c[d] = 0.5 * (a.points[p0] + a.points[p1 - 1])
        return c

    def cells_at(self, ibox, level):
        """Cells (1-based first, last) per axis of box `ibox` of a coarser
        `level` (2 <= level <= maxlevel): the union of its descendants at
        the finest level, so that the levels nest also when the finest split
        is uneven (for evenly divisible grids this is the reference's split
        at that level)."""
        v = box_vector(ibox, level)
        f = 2 ** (self.level - level)
        return [(self._axis_cells(d, v[d] * f)[0], self._axis_cells(d, v[d] * f + f - 1)[1])
                for d in range(3)]

    def center_at(self, ibox, level):
        """Expansion centre of a box of any level (as `center` at maxlevel)."""
        if level == self.level:
            return self.center(ibox)
        v = box_vector(ibox, level)
        nbl = 2 ** level
        c = np.zeros(3)
        for d, (c0, c1) in enumerate(self.cells_at(ibox, level)):
            a = self.grid.axes[d]
            if a.ncell % self.nb == 0:  # gbfmm_parallel_info.F90:1290-1299
                c[d] = self.ranges[d][0] + (v[d] + 0.5) * ((self.ranges[d][1] - self.ranges[d][0]) / nbl)
            else:
                p0, p1 = (c0 - 1) * (a.nlip - 1), c1 * (a.nlip - 1)
                c[d] = 0.5 * (a.points[p0] + a.points[p1])
        return c

    def points(self, ibox):
        """0-based point index range [p0, p1) per axis of the box's sub-grid."""
        return [((c0 - 1) * (a.nlip - 1), c1 * (a.nlip - 1) + 1)
                for (c0, c1), a in zip(self.cells(ibox), self.grid.axes)]

    def owned(self, ibox):
        out = []
        for (c0, c1), a, (p0, p1) in zip(self.cells(ibox), self.grid.axes, self.points(ibox)):
            out.append((p0, p1 if c1 == a.ncell else p1 - 1))
        return out


def _far_field_levels(plan, q_fine, lmax, adaptive=False):
    """Local expansions at the finest level of a multi-level GBFMM
    (gbfmm_coulomb3d.F90:650-905): upward pass q(parent) += W(c_child -
    c_parent) q(child) (translate_multipoles, :1502-1562) from maxlevel - 1
    down to level 2 (1 in the adaptive mode); M2L over the local far field
    at level 2; then for each finer level the parent's local expansion
    translated down (L2L, translate_potential, :1565-1621) plus that level's
    own local far field (adaptive: local_farfield_adaptive, the level - 1
    boxes about their own centres)."""
    N = (lmax + 1) ** 2
    top = plan.level
    q = {top: q_fine}
    for lev in range(top - 1, 0 if adaptive else 1, -1):
        nb = 8 ** lev
        ql = np.zeros((N, nb))
        for p in range(1, nb + 1):
            cp = plan.center_at(p, lev)
            for c in range((p - 1) * 8 + 1, p * 8 + 1):
                ql[:, p - 1] += translate(lmax, q[lev + 1][:, c - 1], plan.center_at(c, lev + 1), cp)
        q[lev] = ql
    Lprev = None
    for lev in range(2, top + 1):
        nb = 8 ** lev
        Ll = np.zeros((N, nb))
        for i in range(1, nb + 1):
            ci = plan.center_at(i, lev)
            if Lprev is not None:
                par = (i - 1) // 8 + 1
                Ll[:, i - 1] += translate_local(lmax, Lprev[:, par - 1], ci, plan.center_at(par, lev - 1))
            if adaptive:
                partial, whole = local_farfield_adaptive(i, lev)
                srcs = [(j, lev) for j in partial] + [(j, lev - 1) for j in whole]
            else:
                srcs = [(j, lev) for j in local_farfield(i, lev)]
            for j, lj in srcs:
                Ll[:, i - 1] += interaction_matrix(lmax, plan.center_at(j, lj) - ci) @ q[lj][:, j - 1]
        Lprev = Ll
    return Lprev


def gbfmm_near_field(grid: Grid3D, rho, maxlevel=2, quad=(25, 25, 0.0, 2.0, 1.0e3),
                     libm_1ulp=False, energy=0.0, blas=False) -> np.ndarray:
    """Near-field part of the GBFMM potential (gbfmm_coulomb3d.F90:933-1098):
    each box's sub-operator (coulomb.F90:517-635) applied to the density on
    the box's near-field cells, written to the points the box owns (no coda).
    energy < 0: Helmholtz weights.  blas: the contractions as DGEMMs."""
    plan = GBFMMPlan(grid, maxlevel)
    rho = np.asfortranarray(rho)
    tp, tw = gauss_quad(*quad)
    w = helmholtz_weights(tp, tw, energy) if energy < 0.0 else coulomb_weights(tw)
    Vnear = np.zeros(grid.shape, order="F")
    for b in range(1, plan.nbox + 1):
        ncl = plan.near_cells(b)
        gin = [subgrid(a, c0, c1) for a, (c0, c1) in zip(grid.axes, ncl)]
        own = plan.owned(b)
        outs = [grid.axes[d].points[own[d][0]:own[d][1]] for d in range(3)]
        Ts = [coulomb_matrix(gin[d], outs[d], tp, libm_1ulp=libm_1ulp) for d in range(3)]
        pin = [((c0 - 1) * (a.nlip - 1), c1 * (a.nlip - 1) + 1) for a, (c0, c1) in zip(grid.axes, ncl)]
        sub = np.asfortranarray(rho[pin[0][0]:pin[0][1], pin[1][0]:pin[1][1], pin[2][0]:pin[2][1]])
        vn = (transform_cube_blas if blas else transform_cube)(*Ts, w, sub, 0.0)
        Vnear[tuple(slice(o0, o1) for o0, o1 in own)] = vn
    return Vnear


def gbfmm_apply(grid: Grid3D, rho, lmax=12, maxlevel=2, quad=(25, 25, 0.0, 2.0, 1.0e3),
                return_parts=False, libm_1ulp=False, energy=0.0, adaptive=False, blas=False):
    """GBFMMCoulomb3D_calculate_potential along the reference's CUDA path
    (gbfmm_coulomb3d.F90:650-819, gbfmm_coulomb3d.cu:478-573): multipoles per
    box, M2L over the local far field, near field by the sub-operator of
    each box (no coda), L2P of the far field; each grid point takes the near
    and far contributions of the box that owns it.  energy < 0: the
    GBFMMHelmholtz3D kernel e^(-kappa r)/r, kappa = sqrt(-2 energy)
    (gbfmm_helmholtz3d.F90:478-1105): Helmholtz near-field weights, Bessel
    multipoles, the Helmholtz multipole-to-local converter and L2P.
    adaptive: the reference's adaptive mode (_far_field_levels, and
    _far_field_levels_helm for the Helmholtz kernel).
    blas: each box's near-field contraction as DGEMMs (transform_cube_blas,
    the same sums in BLAS order; for grids of 181^3 and more)."""
    plan = GBFMMPlan(grid, maxlevel)
    rho = np.asfortranarray(rho)
    N = (lmax + 1) ** 2
    helm = energy < 0.0
    kappa = np.sqrt(-2.0 * energy) if helm else 0.0
    q = np.zeros((N, plan.nbox))
    for b in range(1, plan.nbox + 1):
        (x0, x1), (y0, y1), (z0, z1) = plan.points(b)
        subs = [subgrid(a, c0, c1) for a, (c0, c1) in zip(grid.axes, plan.cells(b))]
        args = (subs[0].points, subs[0].weights(), subs[1].points, subs[1].weights(),
                subs[2].points, subs[2].weights(), rho[x0:x1, y0:y1, z0:z1], plan.center(b))
        q[:, b - 1] = (helm_box_multipoles(lmax, kappa, *args) if helm
                       else box_multipoles(lmax, *args))
    if maxlevel > 2 or adaptive:
        L = (_far_field_levels_helm(plan, q, lmax, kappa, adaptive) if helm
             else _far_field_levels(plan, q, lmax, adaptive))
    else:
        L = np.zeros((N, plan.nbox))
        for i in range(1, plan.nbox + 1):
            ci = plan.center(i)
            for j in local_farfield(i, maxlevel):
                if helm:
                    L[:, i - 1] += helm_m2l(lmax, kappa, q[:, j - 1], plan.center(j), ci)
                else:
                    L[:, i - 1] += interaction_matrix(lmax, plan.center(j) - ci) @ q[:, j - 1]
    Vnear = gbfmm_near_field(grid, rho, maxlevel, quad, libm_1ulp, energy, blas)
    V = Vnear.copy(order="F")
    for b in range(1, plan.nbox + 1):
        own = plan.owned(b)
        outs = [grid.axes[d].points[own[d][0]:own[d][1]] for d in range(3)]
        far = np.zeros(tuple(len(o) for o in outs), order="F")
        if helm:
            helm_l2p(lmax, kappa, L[:, b - 1], plan.center(b), outs[0], outs[1], outs[2], far)
        else:
            l2p(lmax, L[:, b - 1], plan.center(b), outs[0], outs[1], outs[2], far)
        V[tuple(slice(o0, o1) for o0, o1 in own)] += far
    if return_parts:
        return V, q, L, Vnear
    return V


# ---------------------------------------------------------------------------
# Bubbles
# ---------------------------------------------------------------------------
def bubbles_inject(centers, ncells, cell_scales, lmax, f, grid: Grid3D, lmin=0, k=0,
                   factor=1.0, cube=None, nlip=7):
    """cube += factor * sum of the atom-centred bubbles (Bubbles_eval_pick,
    bubbles.F90:1904-1975).  f: list over atoms of ((lmax+1)^2, npoints)."""
    centers = _f64(np.asarray(centers, dtype=np.float64).reshape(-1, 3))
    nc = (ctypes.c_int * len(ncells))(*ncells)
    cs = _f64(np.concatenate([np.asarray(c, dtype=np.float64) for c in cell_scales]))
    ff = _f64(np.concatenate([np.asarray(a, dtype=np.float64).reshape(-1) for a in f]))
    if cube is None:
        cube = np.zeros(grid.shape, order="F")
    gx, gy, gz = grid.axes
    rc = lib().orc_bubbles_inject(len(ncells), _p(centers), nc, _p(cs), nlip, lmax, lmin, k,
                                  _p(ff), gx.n, _p(gx.points), gy.n, _p(gy.points), gz.n,
                                  _p(gz.points), float(factor), _p(cube))
    if rc:
        raise ValueError("bad bubbles input")
    return cube


def log_radial_grid(ncell=33, r0=1e-5, r1=15.0, nlip=7):
    """Cell steps of a radial LIP grid from r = 0 whose cell ends are
    log-spaced on [r0, r1] (ncell cells, ncell*(nlip-1)+1 points)."""
    edges = np.concatenate([[0.0], r0 * (r1 / r0) ** (np.arange(ncell) / (ncell - 1))])
    return np.diff(edges) / (nlip - 1)


def lip_partial_integrals(nlip):
    """LIPBasis outward/inward integrals (lip.F90:414-480) of the
    equidistant basis on local nodes first, first+1, ..., first+nlip-1:
    out[i, j-1] = int_{x_0}^{x_j} chi_i, inn[i, j] = int_{x_j}^{x_n} chi_i."""
    first = -((nlip - 1) // 2)
    x = first + np.arange(nlip, dtype=np.float64)
    out = np.zeros((nlip, nlip - 1))
    inn = np.zeros((nlip, nlip - 1))
    for i in range(nlip):
        others = np.delete(x, i)
        P = np.poly1d(others, r=True) / np.prod(x[i] - others)
        A = np.polyint(P)
        for j in range(1, nlip):
            out[i, j - 1] = A(x[j]) - A(x[0])
        for j in range(nlip - 1):
            inn[i, j] = A(x[-1]) - A(x[j])
    return out, inn


def bubbles_coulomb_potential(ncell, cell_scales, lmax, f, k=0, nlip=7):
    """Coulomb3D_evaluate_bubbles_potential (coulomb.F90:222-336) for one atom:
    V_lm(r) = 4 pi/(2l+1) [ r^-(l+1) int_0^r f_lm s^(l+2+k) ds
                            + r^l int_r^inf f_lm s^(1-l+k) ds ]
    with the cumulative LIP integrals of InOutIntegrator1D
    (evaluators.F90:1263-1318); negative powers are 0 at r = 0
    (Bubbles_rpow, bubbles.F90:3363-3378).  f: ((lmax+1)^2, npts)."""
    h = _f64(np.broadcast_to(cell_scales, (ncell,)))
    n = nlip - 1
    r = Grid1D(0.0, ncell, nlip, 1, h).points
    npts = r.size
    out_i, in_i = lip_partial_integrals(nlip)

    def rpow(p):
        if p >= 0:
            return r ** p
        v = np.zeros_like(r)
        v[1:] = r[1:] ** p
        return v

    def outwards(g):
        res = np.zeros(npts)
        for c in range(ncell):
            s = c * n
            res[s + 1:s + n + 1] = (g[s:s + n + 1] @ out_i) * h[c] + res[s]
        return res

    def inwards(g):
        res = np.zeros(npts)
        for c in range(ncell - 1, -1, -1):
            s = c * n
            res[s:s + n] = (g[s:s + n + 1] @ in_i) * h[c] + res[s + n]
        return res

    f = np.asarray(f, dtype=np.float64).reshape((lmax + 1) ** 2, npts)
    V = np.zeros_like(f)
    for l in range(lmax + 1):
        r1, r2, r3, r4 = rpow(-(l + 1)), rpow(l + 2 + k), rpow(l), rpow(-(l + 1) + 2 + k)
        for m in range(-l, l + 1):
            lm = l * (l + 1) + m
            V[lm] = 4 * np.pi / (2 * l + 1) * (r1 * outwards(f[lm] * r2) + r3 * inwards(f[lm] * r4))
    return V


# ---------------------------------------------------------------------------
# Products of functions (the density producer)
# ---------------------------------------------------------------------------
def _clebsch_gordan(l1, m1, l2, m2, l, m):
    """<l1 m1 l2 m2 | l m> by Racah's closed formula (harmonic.F90:991-1031)."""
    from math import factorial as F, sqrt
    if l < abs(l1 - l2) or l > l1 + l2 or abs(m1) > l1 or abs(m2) > l2 or abs(m) > l \
            or m != m1 + m2:
        return 0.0
    pre = sqrt((2 * l + 1.0) / F(l1 + l2 + l + 1) * F(l1 + l2 - l) * F(l2 + l - l1)
               * F(l + l1 - l2) * F(l1 + m1) * F(l1 - m1) * F(l2 + m2) * F(l2 - m2)
               * F(l + m) * F(l - m))
    s = 0.0
    for kk in range(max(l1 + m2 - l, l2 - m1 - l, 0), min(l1 + l2 - l, l1 - m1, l2 + m2) + 1):
        t = (F(l1 + l2 - l - kk) * F(l - l1 - m2 + kk) * F(l - l2 + m1 + kk)
             * F(l1 - m1 - kk) * F(l2 + m2 - kk) * F(kk))
        s += (-1.0 if kk % 2 else 1.0) / t
    return pre * s


def _real_product_coeff(l1, m1, l2, m2, l, m):
    """Coefficient of Y_lm in Y_l1m1 * Y_l2m2 for the Racah-normalised real
    harmonics (prod_coeff, harmonic.F90:1034-1089): a product of two
    Clebsch-Gordan coefficients with the real-harmonic phase rule."""
    sgn = lambda v: 1 if v >= 0 else -1  # Fortran sign(1, v)
    cp = lambda v: 0.5 if v < 0 else float(v)
    cm = lambda v: v - 0.5 if v < 0 else 0.0
    if (l - l1 - l2) % 2 or sgn(m1) * sgn(m2) * sgn(m) < 0:
        return 0.0
    if m == m1 + m2:
        f, a, b = cp(m1) + cp(m2) - cp(m), m1, m2
    elif m == m1 - m2:
        f, a, b = cp(m1) + cm(m2) - cp(m), m1, -m2
    elif m == -m1 + m2:
        f, a, b = cm(m1) + cp(m2) - cp(m), -m1, m2
    elif m == -m1 - m2:
        f, a, b = cm(m1) + cm(m2) - cp(m), -m1, -m2
    else:
        return 0.0
    # Fortran nint of a REAL32 half-integer rounds away from zero
    e = int(np.floor(abs(f) + 0.5)) * (1 if f >= 0 else -1)
    res = _clebsch_gordan(l1, 0, l2, 0, l, 0) * _clebsch_gordan(l1, a, l2, b, l, m) * (-1.0) ** e
    if m1 * m2 * m != 0:
        res /= np.sqrt(2.0)
    return res


def yproduct(lmax, result_lmax=None):
    """YProduct_init (harmonic.F90:884-951): for every unordered pair of
    harmonic indices a <= b (lm = l(l+1)+m, 0-based) the list of
    (result index, coefficient) with Y_a Y_b = sum C Y_LM."""
    if result_lmax is None:
        result_lmax = 2 * lmax
    table = {}
    for l1 in range(lmax + 1):
        for m1 in range(-l1, l1 + 1):
            for l2 in range(l1, lmax + 1):
                for m2 in range(m1 if l1 == l2 else -l2, l2 + 1):
                    sgn = (1 if m1 >= 0 else -1) * (1 if m2 >= 0 else -1)
                    terms = []
                    for l in range(abs(l1 - l2), min(result_lmax, l1 + l2) + 1, 2):
                        m = sgn * abs(m1 - m2)
                        if abs(m) > l:
                            continue
                        terms.append((l * (l + 1) + m, _real_product_coeff(l1, m1, l2, m2, l, m)))
                        if m1 * m2 != 0 and (sgn == 1 or m1 + m2 != 0):
                            m = sgn * abs(m1 + m2)
                            if abs(m) > l:
                                continue
                            terms.append((l * (l + 1) + m,
                                          _real_product_coeff(l1, m1, l2, m2, l, m)))
                    table[(l1 * (l1 + 1) + m1, l2 * (l2 + 1) + m2)] = terms
    return table


def bubbles_multiply(f1, lmax1, f2, lmax2):
    """Radial product of two bubbles on one atom (Bubble_product_kernel,
    bubbles_multiplier.cu:65-106, option (2) of BubblesMultiplier_multiply,
    bubbles.F90:3567-3690): result ((lmax1+lmax2+1)^2, npts) with
    r_LM = sum_{a<=b} C_ab^LM (f1_a f2_b + f1_b f2_a [a != b]); k adds."""
    f1 = np.asarray(f1, dtype=np.float64)
    f2 = np.asarray(f2, dtype=np.float64)
    N1, N2 = (lmax1 + 1) ** 2, (lmax2 + 1) ** 2
    lr = lmax1 + lmax2
    out = np.zeros(((lr + 1) ** 2, f1.shape[1]))
    for (a, b), terms in yproduct(max(lmax1, lmax2), lr).items():
        s = np.zeros(f1.shape[1])
        if a < N1 and b < N2:
            s = s + f1[a] * f2[b]
        if a != b and b < N1 and a < N2:
            s = s + f1[b] * f2[a]
        for LM, C in terms:
            out[LM] += C * s
    return out


def function3d_multiply(grid: Grid3D, cube1, cube2, bubbles1=None, bubbles2=None,
                        result_bubbles=None):
    """Cube part of Function3D_multiply (function3d.F90:1097-1409, the
    non-CUDA branch at :1372-1390): (cube1 + bubbles1)(cube2 + bubbles2)
    - result_bubbles on the grid.  Each bubbles argument is a dict of
    bubbles_inject keyword arguments (centers, ncells, cell_scales, lmax, f, k)."""
    def with_bubbles(cube, b, factor=1.0):
        c = np.array(cube, dtype=np.float64, order="F", copy=True)
        if b is not None:
            bubbles_inject(grid=grid, cube=c, factor=factor, **b)
        return c
    out = with_bubbles(cube1, bubbles1) * with_bubbles(cube2, bubbles2)
    if result_bubbles is not None:
        bubbles_inject(grid=grid, cube=out, factor=-1.0, **result_bubbles)
    return out


def bubbles_helmholtz_potential(ncell, cell_scales, lmax, f, kappa, k=0, nlip=7):
    """Helmholtz3D_transform_bubbles_sub (helmholtz3d.F90:519-650) for one
    atom: with i_l, k_l the modified spherical Bessel functions
    (i_0 = sinh x / x, k_0 = pi/2 e^-x / x; both 0 except i_0 = 1 at x = 0,
    helmholtz3d.F90:851-1060),
      V_lm(r) = 8 kappa [ k_l(kr) int_0^r i_l(ks) f s^(2+k) ds
                          + i_l(kr) int_r^inf k_l(ks) f s^(2+k) ds ],
    the inward integrand's value at r = 0 replaced by the 3-point
    extrapolation 3 g1 - 3 g2 + g3 for l = 0 and by 0 otherwise
    (extrapolate_first_nlip7, evaluators.F90:1588-1600).  The cumulative
    integrals are those of bubbles_coulomb_potential."""
    from scipy.special import spherical_in, spherical_kn
    h = _f64(np.broadcast_to(cell_scales, (ncell,)))
    n = nlip - 1
    r = Grid1D(0.0, ncell, nlip, 1, h).points
    npts = r.size
    out_i, in_i = lip_partial_integrals(nlip)
    x = kappa * r
    I = np.zeros((lmax + 1, npts))
    K = np.zeros((lmax + 1, npts))
    nz = x > np.finfo(np.float64).eps
    for l in range(lmax + 1):
        I[l, nz] = spherical_in(l, x[nz])
        K[l, nz] = spherical_kn(l, x[nz])
    I[0, ~nz] = 1.0
    rp = r ** (2 + k)

    def outwards(g):
        res = np.zeros(npts)
        for c in range(ncell):
            s = c * n
            res[s + 1:s + n + 1] = (g[s:s + n + 1] @ out_i) * h[c] + res[s]
        return res

    def inwards(g):
        res = np.zeros(npts)
        for c in range(ncell - 1, -1, -1):
            s = c * n
            res[s:s + n] = (g[s:s + n + 1] @ in_i) * h[c] + res[s + n]
        return res

    f = np.asarray(f, dtype=np.float64).reshape((lmax + 1) ** 2, npts)
    V = np.zeros_like(f)
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            lm = l * (l + 1) + m
            t1 = rp * I[l] * f[lm]
            t2 = rp * K[l] * f[lm]
            t2[0] = 3 * t2[1] - 3 * t2[2] + t2[3] if l == 0 else 0.0
            V[lm] = 8 * kappa * (K[l] * outwards(t1) + I[l] * inwards(t2))
    return V


# ---------------------------------------------------------------------------
# Taylor-series contaminant bubbles
# ---------------------------------------------------------------------------
def cart_iter(tmax):
    """CartIter(3, tmax) (cartiter.F90:169-223): the multi-indices with
    |kappa| <= tmax, the last index running fastest."""
    return [(a, b, c) for a in range(tmax + 1) for b in range(tmax + 1 - a)
            for c in range(tmax + 1 - a - b)]


def dvpos_shell(dv):
    """Position (1-based) of dv in its shell (harmonic.F90:1378-1385)."""
    k = sum(dv)
    return (dv[0] * (3 + 2 * k - dv[0]) + 2) // 2 + dv[1]


def dvpos(dv):
    """The reference's position of dv in the shell-grouped series
    (harmonic.F90:1369-1376): dvpos_shell + |dv|^2, which is the true offset
    |dv|(|dv|+1)(|dv|+2)/6 for |dv| <= 2 only."""
    return dvpos_shell(dv) + sum(dv) ** 2


def grid1d_icell(celld, qmin, qmax, x):
    """Grid1D_get_icell (grid.F90:1212-1245): 1-based cell of x, 0 outside."""
    ncell = len(celld)
    if x > qmax or x < qmin:
        return 0
    if celld[ncell - 1] <= x:
        return ncell
    icell, maxi, mini = ncell // 2, ncell - 1, 1
    while True:
        if x >= celld[icell]:
            if x < celld[icell + 1]:
                return icell + 1
            mini = icell + 2
            icell = (mini + maxi) // 2
        else:
            if x >= celld[icell - 1]:
                return icell
            maxi = icell - 1
            icell = (mini + maxi) // 2


def lip_interp_derivatives(g: Grid1D, vals, x, order):
    """Interpolator1D_eval (evaluators.F90:766-830): d^j/dx^j, j <= order, of
    the LIP interpolant of the point values ``vals`` (shape (..., g.n)) at
    x; zeros outside the grid."""
    vals = np.asarray(vals, dtype=np.float64)
    out = np.zeros(vals.shape[:-1] + (order + 1,))
    ic = grid1d_icell(g.celld, g.points[0], g.points[-1], x)
    if ic == 0:
        return out
    c, first, _ = lip_coeffs(g.nlip, g.grid_type)
    h = g.cell_scales[ic - 1]
    crd = (x - g.celld[ic - 1]) / h + first
    s = (ic - 1) * (g.nlip - 1)
    block = vals[..., s:s + g.nlip]
    for j in range(order + 1):
        pv = np.array([np.polyval(np.polyder(c[i], j) if j else c[i], crd) for i in range(g.nlip)])
        out[..., j] = (block @ pv) * h ** (-j)
    return out


def _sympy_xyzr():
    import sympy as sp
    return sp, sp.symbols("x y z r", real=True)


def ybundle_polys(lmax):
    """YBundle_init (harmonic.F90:612-660): the Racah-normalised real
    harmonics as polynomials in x/r, y/r, z/r (the recursion's r2 monomial is
    1), exact sympy expressions in x, y, z, r; index lm = l(l+1)+m."""
    sp, (x, y, z, r) = _sympy_xyzr()
    X, Y, Z = x / r, y / r, z / r
    N = (lmax + 1) ** 2
    P = [None] * N
    P[0] = sp.Integer(1)
    if lmax > 0:
        P[1], P[2], P[3] = Y, Z, X
    for l in range(2, lmax + 1):
        f1 = sp.sqrt(1 - sp.Rational(1, 2 * l))
        P[l * (l + 1) - l] = f1 * (P[(l - 1) * l + (l - 1)] * Y + P[(l - 1) * l - (l - 1)] * X)
        for m in range(-(l - 1), l):
            e = (2 * l - 1) * P[(l - 1) * l + m] * Z
            if l - abs(m) > 1:
                e = e - sp.sqrt((l + m - 1) * (l - m - 1)) * P[(l - 2) * (l - 1) + m]
            P[l * (l + 1) + m] = e / sp.sqrt((l - m) * (l + m))
        P[l * (l + 1) + l] = f1 * (P[(l - 1) * l + (l - 1)] * X - P[(l - 1) * l - (l - 1)] * Y)
    return [sp.expand(p) for p in P]


_EVAL_COEFFS = {}


def y_eval_coeffs(lmax, dv):
    """Y_eval_coeffs (harmonic.F90:806-860): for every lm, the polynomials
    P_i(x, y, z, r), i <= |dv|, with d^dv [Y_lm f(r)] = sum_i P_i f^(i)(r);
    returned as numpy callables of (x, y, z, r).  Differentiating in x_m a
    term P f^(i) gives (dP/dx_m + dP/dr x_m/r) f^(i) + P x_m/r f^(i+1)."""
    key = (lmax, tuple(dv))
    if key in _EVAL_COEFFS:
        return _EVAL_COEFFS[key]
    sp, (x, y, z, r) = _sympy_xyzr()
    xs = (x, y, z)
    out = []
    for Y in ybundle_polys(lmax):
        prev = [Y]
        for m in range(3):
            for _ in range(dv[m]):
                new = [sp.Integer(0)] * (len(prev) + 1)
                for i, p in enumerate(prev):
                    new[i] += sp.diff(p, xs[m]) + sp.diff(p, r) * xs[m] / r
                    new[i + 1] += p * xs[m] / r
                prev = new
        out.append([sp.lambdify((x, y, z, r), p, "numpy") for p in prev])
    _EVAL_COEFFS[key] = out
    return out


def bubble_contaminants(centers, grids, lmax, f, k, tmax):
    """Bubbles_get_contaminants (bubbles.F90:2844-2910) with the radial
    derivatives of Bubbles_get_radial_derivatives (bubbles.F90:2272-2300,
    k >= 0: derivatives of the LIP interpolant of r^k f): contams[B, i] =
    sum_{A != B} sum_lm d^kappa_i [(r^k f_A,lm)(r_A) Y_lm](R_B)."""
    centers = np.asarray(centers, dtype=np.float64).reshape(-1, 3)
    nat = len(centers)
    kap = cart_iter(tmax)
    out = np.zeros((nat, len(kap)))
    polys = [y_eval_coeffs(lmax, dv) for dv in kap]
    for A in range(nat):
        g = grids[A]
        rk = np.asarray(f[A], dtype=np.float64) * g.points ** k
        for B in range(nat):
            if A == B:
                continue
            v = centers[B] - centers[A]
            d = float(np.sqrt(v @ v))
            rfs = lip_interp_derivatives(g, rk, d, tmax)  # (N, tmax+1)
            for i, dv in enumerate(kap):
                s = 0.0
                for lm, P in enumerate(polys[i]):
                    s += sum(float(Pi(v[0], v[1], v[2], d)) * rfs[lm, j] for j, Pi in enumerate(P))
                out[B, i] += s
    return out


def cube_contaminants(grid: Grid3D, cube, centers, tmax):
    """Function3D_get_cube_contaminants (function3d.F90:1570-1624) through
    the Interpolator (evaluators.F90:853-1000): partial derivatives of the
    cube's LIP interpolant at the centres (x's LIP basis for every axis),
    0 for a centre outside the grid."""
    centers = np.asarray(centers, dtype=np.float64).reshape(-1, 3)
    kap = cart_iter(tmax)
    out = np.zeros((len(centers), len(kap)))
    nlip = grid.axes[0].nlip
    c, first, _ = lip_coeffs(nlip, grid.axes[0].grid_type)
    for B, R in enumerate(centers):
        P, s = [], []
        for d, g in enumerate(grid.axes):
            ic = grid1d_icell(g.celld, g.points[0], g.points[-1], R[d])
            if ic == 0:
                break
            h = g.cell_scales[ic - 1]
            crd = (R[d] - g.celld[ic - 1]) / h + first
            P.append([np.array([np.polyval(np.polyder(c[i], j) if j else c[i], crd)
                                for i in range(nlip)]) * h ** (-j) for j in range(tmax + 1)])
            s.append((ic - 1) * (nlip - 1))
        if len(P) < 3:
            continue
        blk = np.asarray(cube)[s[0]:s[0] + nlip, s[1]:s[1] + nlip, s[2]:s[2] + nlip]
        for i, (a, b, cc) in enumerate(kap):
            out[B, i] = np.einsum("ijk,i,j,k->", blk, P[0][a], P[1][b], P[2][cc])
    return out


def cart_to_sph(lmax):
    """Cart2SphIter_init (harmonic.F90:1096-1165): the (lmax+1)^2 x ncart
    matrix whose column for a monomial x^kappa (columns grouped by shell,
    dvpos_shell order within a shell) holds its expansion
    x^kappa = r^|kappa| sum_lm S_lm Y_lm, from the inverse of each shell's
    matrix of the monomial coefficients of r^(k-l) S_lm."""
    sp, (x, y, z, r) = _sympy_xyzr()
    Y = ybundle_polys(lmax)
    ncart = (lmax + 1) * (lmax + 2) * (lmax + 3) // 6
    out = np.zeros(((lmax + 1) ** 2, ncart))
    for k in range(lmax + 1):
        mono = [(a, b, k - a - b) for a in range(k + 1) for b in range(k + 1 - a)]
        sph = [(l, m) for l in range(k % 2, k + 1, 2) for m in range(-l, l + 1)]
        M = np.zeros((len(mono), len(sph)))
        for s, (l, m) in enumerate(sph):
            # r^k Y_lm: the reference's poly%extend(k)
            e = sp.expand(sp.expand(Y[l * (l + 1) + m] * r ** k).subs(r, sp.sqrt(x * x + y * y + z * z)))
            poly = sp.Poly(e, x, y, z)
            for row, (a, b, c) in enumerate(mono):
                M[row, s] = float(poly.coeff_monomial(x ** a * y ** b * z ** c))
        inv = np.linalg.inv(M)
        base = k * (k + 1) * (k + 2) // 6
        for s, (l, m) in enumerate(sph):
            out[l * (l + 1) + m, base:base + len(mono)] = inv[s]
    out[np.abs(out) <= 1e-16] = 0.0
    return out


def make_taylor(grids, lmax, k, bubble_contams, cube_contams, tmax, exact=False):
    """Bubbles_make_taylor (bubbles.F90:1435-1530) with the damping w
    (bubbles.F90:1532-1558) and Bubbles_rpow (bubbles.F90:3363-3378): per
    atom, ((max(lmax, tmax)+1)^2, npoints) radial values (without r^k).
    ``exact``: 1/kappa! and the shell-grouped column instead of 1/|kappa|!
    and dvpos."""
    import math
    lnew = max(lmax, tmax)
    C = cart_to_sph(max(lnew, 3))
    out = []
    for A, g in enumerate(grids):
        rr = g.points
        w = np.array([0.5 * math.erfc(v - 2.0 / v) if v > np.finfo(float).eps else 1.0 for v in rr])
        f = np.zeros(((lnew + 1) ** 2, g.n))
        for kappa in cart_iter(tmax):
            K = sum(kappa)
            n = K - k
            if n >= 0:
                rp = rr ** n
            else:
                rp = np.concatenate([[0.0], rr[1:] ** n])
            if exact:
                fac = 1.0 / (math.factorial(kappa[0]) * math.factorial(kappa[1]) * math.factorial(kappa[2]))
                col = K * (K + 1) * (K + 2) // 6 + dvpos_shell(kappa) - 1
            else:
                fac = 1.0 / math.factorial(K)
                col = dvpos(kappa) - 1
            i = cart_iter(tmax).index(kappa)
            cval = (bubble_contams[A][i] if bubble_contams is not None else 0.0) + \
                (cube_contams[A][i] if cube_contams is not None else 0.0)
            val = cval * (rp * w * fac)
            for lm in np.nonzero(C[:, col])[0]:
                if lm < f.shape[0]:
                    f[lm] += C[lm, col] * val
        out.append(f)
    return out


def bubbles_multiply_taylor(f1, lmax1, t1, f2, lmax2, t2):
    """Option (1) of BubblesMultiplier_multiply (bubbles.F90:3567-3640;
    BubblesMultiplier::multiplyBubble, bubbles_multiplier.cu:240-292) for one
    atom: (b1 + t1)(b2 + t2) - t1 t2 with each Taylor set cut at its bubbles'
    lmax (Bubble::add, bubbles_cuda.cu:2629-2680)."""
    N1, N2 = (lmax1 + 1) ** 2, (lmax2 + 1) ** 2
    f1, f2 = np.asarray(f1, dtype=np.float64), np.asarray(f2, dtype=np.float64)
    u1, u2 = np.asarray(t1, dtype=np.float64)[:N1], np.asarray(t2, dtype=np.float64)[:N2]
    return bubbles_multiply(f1 + u1, lmax1, f2 + u2, lmax2) - bubbles_multiply(u1, lmax1, u2, lmax2)


def bubbles_integrate(grids, f, k=0):
    """Bubbles_integrate_all (bubbles.F90:3146-3240): 4 pi sum_A
    int r^(2+k) f_A,00(r) dr with each radial grid's LIP weights."""
    return float(sum(4.0 * np.pi * np.sum(g.weights() * (np.asarray(fa)[0] * g.points ** (2 + k)))
                     for g, fa in zip(grids, f)))
