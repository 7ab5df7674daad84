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
_lib = None

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.c_int
_F = ctypes.c_double


def build(force: bool = False) -> str:
    """Compile the oracle with ``make -C oracle``; returns the library path."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        sig = {
            "orc_gauss_quad": (None, [_I, _I, _F, _F, _F, _D, _D]),
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
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


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


def coulomb_matrix(grid_in: Grid1D, out_points, tp, border_only=False) -> np.ndarray:
    """T(i_out, j_in, p) for one axis (exponentials.F90:178-346)."""
    out = _f64(out_points)
    tp = _f64(tp)
    T = np.zeros((len(out), grid_in.n, len(tp)), order="F")
    fn = lib().orc_coulomb_border_matrix if border_only else lib().orc_coulomb_matrix
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
def coulomb_operator_matrices(grid_in: Grid3D, grid_out: Grid3D, tp):
    """make_Coulomb3D_matrices (exponentials.F90:602-639), all three axes in
    the T(i_out, j_in, p) orientation."""
    return tuple(coulomb_matrix(grid_in.axes[d], grid_out.axes[d].points, tp) for d in range(3))


def coulomb_apply(grid: Grid3D, rho, quad=(10, 8, 0.0, 2.0, 1.0e3), coda=True, weights=None):
    """V = Coulomb3D(grid) .apply. rho (cube part), CPU semantics."""
    nlin, nlog, tstart, tlin, tlog = quad
    tp, tw = gauss_quad(nlin, nlog, tstart, tlin, tlog)
    Tx, Ty, Tz = coulomb_operator_matrices(grid, grid, tp)
    w = coulomb_weights(tw) if weights is None else weights
    return transform_cube(Tx, Ty, Tz, w, rho, coda_of(tlog) if coda else 0.0)


def selfint(grid: Grid3D, rho, quad=(10, 8, 0.0, 2.0, 1.0e3), coda=True) -> float:
    """rho .dot. (Coulomb3D .apply. rho) as tests/gauss_test.F90 computes it."""
    V = coulomb_apply(grid, rho, quad, coda)
    return integrate_cube(grid, rho * V)
