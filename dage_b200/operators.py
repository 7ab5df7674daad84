"""Host-side mirror of the reference's operator interface for this path.

The names follow DAGE's Fortran types (``GaussQuad``, ``Grid1D``,
``Grid3D``, ``Coulomb3D``, ``Helmholtz3D``, ``Function3D``-style
``dot``/``integrate``) so that code written against the reference's
``Operator3D``/``Function3D`` API reads the same:

    V = Coulomb3D(grid) .apply(rho)           # Operator3D .apply.
    E = integrate(grid, rho, V)               # rho .dot. V

Cubes are numpy arrays in Fortran order ``(nx, ny, nz)`` (host memory) or
torch CUDA tensors whose storage is the same column-major cube (device
memory, e.g. ``t = torch.empty(nz, ny, nx)``; x fastest).  All arithmetic
runs in libdagegpu.so on the GPU.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _capi
from ._capi import DageGrid1D, DageQuad, check, load

PRECISIONS = {
    "fp64": _capi.DAGE_FP64,
    "bf16x3": _capi.DAGE_MIXED_BF16X3,
    "bf16x6": _capi.DAGE_MIXED_BF16X6,
    "fp16x3": _capi.DAGE_MIXED_FP16X3,
}


@dataclass
class GaussQuad:
    """GaussQuad (src/bubbles/gauss.F90:55-122); same defaults."""

    nlin: int = 10
    nlog: int = 8
    tstart: float = 0.0
    tlin: float = 2.0
    tlog: float = 1.0e3

    def c(self) -> DageQuad:
        return DageQuad(self.nlin, self.nlog, self.tstart, self.tlin, self.tlog)

    @property
    def npoints(self) -> int:
        return self.nlin + self.nlog


@dataclass
class Grid1D:
    """One axis of LIP cells (src/bubbles/grid.F90:446-534)."""

    qmin: float
    ncell: int
    nlip: int = 7
    grid_type: int = 1
    cell_scales: np.ndarray = field(default=None)

    def __post_init__(self):
        if self.cell_scales is None:
            raise ValueError("cell_scales required")
        self.cell_scales = np.ascontiguousarray(
            np.broadcast_to(np.asarray(self.cell_scales, dtype=np.float64), (self.ncell,)))

    @classmethod
    def equidistant(cls, qmin: float, ncell: int, step: float, nlip: int = 7, grid_type: int = 1):
        return cls(float(qmin), int(ncell), nlip, grid_type, np.full(ncell, float(step)))

    @property
    def n(self) -> int:
        return self.ncell * (self.nlip - 1) + 1

    def c(self) -> DageGrid1D:
        return DageGrid1D(self.ncell, self.nlip, self.grid_type, self.qmin,
                          self.cell_scales.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))

    def coordinates(self) -> np.ndarray:
        """Grid point coordinates (equidistant cells only)."""
        if self.grid_type != 1:
            raise NotImplementedError("coordinates() for equidistant cells")
        pts = [self.qmin]
        x = self.qmin
        for h in self.cell_scales:
            start = x
            for k in range(1, self.nlip):
                pts.append(start + k * h)
            x = pts[-1]
        return np.asarray(pts)


@dataclass
class Grid3D:
    axes: tuple

    @classmethod
    def cube(cls, qmin: float, ncell: int, step: float, nlip: int = 7, grid_type: int = 1):
        ax = Grid1D.equidistant(qmin, ncell, step, nlip, grid_type)
        return cls((ax, ax, ax))

    @property
    def shape(self):
        return tuple(a.n for a in self.axes)

    def c(self):
        arr = (DageGrid1D * 3)(*[a.c() for a in self.axes])
        return arr


def _ptr(a, nelem: int):
    """(pointer, is_device) of a float64 cube with nelem elements."""
    try:
        import torch  # noqa: F401

        if hasattr(a, "is_cuda"):
            if a.dtype != torch.float64 or not a.is_contiguous():
                raise TypeError("torch cube must be contiguous float64")
            if a.numel() != nelem:
                raise ValueError(f"cube has {a.numel()} elements, expected {nelem}")
            return ctypes.c_void_p(a.data_ptr()), a.is_cuda
    except ImportError:
        pass
    if not isinstance(a, np.ndarray) or a.dtype != np.float64:
        raise TypeError("cube must be a float64 numpy array or torch tensor")
    if not a.flags.f_contiguous:
        raise TypeError("numpy cube must be Fortran-ordered (x fastest)")
    if a.size != nelem:
        raise ValueError(f"cube has {a.size} elements, expected {nelem}")
    return ctypes.c_void_p(a.ctypes.data), False


class Operator3D:
    """Tensor-product cube operator, V = sum_p w_p (T^x_p (x) T^y_p (x) T^z_p) rho
    (+ coda rho).  ``Coulomb3D`` and ``Helmholtz3D`` are its two kernels."""

    def __init__(self, gridin: Grid3D, gridout: Grid3D | None = None,
                 quad: GaussQuad | None = None, precision: str = "fp64",
                 cache_dir: str | None = None):
        """``cache_dir``: on-disk cache of the operator matrices keyed by the
        grids and the quadrature (read when present, written otherwise;
        ``from_cache`` tells which)."""
        lib = load()
        self.gridin = gridin
        self.gridout = gridout if gridout is not None else gridin
        self.quad = quad if quad is not None else GaussQuad()
        self.precision = precision
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {list(PRECISIONS)}")
        self._keep = (self.gridin.c(), self.gridout.c(), self.quad.c())
        h = ctypes.c_void_p()
        self.from_cache = False
        if cache_dir:
            fc = ctypes.c_int(0)
            check(lib.dage_op3d_create_cached(self._keep[0], self._keep[1],
                                              ctypes.byref(self._keep[2]), PRECISIONS[precision],
                                              cache_dir.encode(), ctypes.byref(fc),
                                              ctypes.byref(h)))
            self.from_cache = bool(fc.value)
        else:
            check(lib.dage_op3d_create(self._keep[0], self._keep[1], ctypes.byref(self._keep[2]),
                                       PRECISIONS[precision], ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                load().dage_op3d_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def tiles(self):
        """Contraction tile widths of the three stages (FP64: the autotuner's
        choice, keyed on points per axis and t-points)."""
        t = (ctypes.c_int * 3)()
        check(load().dage_op3d_tiles(self._h, t))
        return tuple(t)

    @property
    def schedule(self):
        """Split-precision operators: (ring stages, t-points per last-stage
        pass) of the tensor-core stages as the autotuner chose them; None in
        FP64."""
        if self.precision == _capi.DAGE_FP64:
            return None
        ns, g = ctypes.c_int(), ctypes.c_int()
        check(load().dage_op3d_mixed_schedule(self._h, ctypes.byref(ns), ctypes.byref(g)))
        return ns.value, g.value

    # -- quadrature -------------------------------------------------------
    def quadrature(self):
        P = self.quad.npoints
        tp = np.zeros(P)
        w = np.zeros(P)
        n = ctypes.c_int()
        dp = ctypes.POINTER(ctypes.c_double)
        check(load().dage_op3d_get_quadrature(self._h, ctypes.byref(n), tp.ctypes.data_as(dp),
                                              w.ctypes.data_as(dp)))
        return tp, w

    @property
    def tpoints(self):
        return self.quadrature()[0]

    @property
    def weights(self):
        return self.quadrature()[1]

    def set_transformation_weights(self, w) -> None:
        w = np.ascontiguousarray(w, dtype=np.float64)
        check(load().dage_op3d_set_weights(self._h, len(w),
                                           w.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))

    def set_coda(self, coda: float) -> None:
        check(load().dage_op3d_set_coda(self._h, float(coda)))

    def set_stream(self, stream) -> None:
        """Run on a caller's CUDA stream (a torch.cuda.Stream or raw handle)."""
        handle = getattr(stream, "cuda_stream", stream)
        check(load().dage_op3d_set_stream(self._h, ctypes.c_void_p(handle or 0)))

    def matrix(self, axis: int) -> np.ndarray:
        """FP64 matrix of one axis, T(i_out, j_in, p)."""
        no = self.gridout.axes[axis].n
        ni = self.gridin.axes[axis].n
        T = np.zeros((no, ni, self.quad.npoints), order="F")
        check(load().dage_op3d_get_matrix(self._h, axis,
                                          T.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return T

    def set_timing(self, enable: bool = True) -> None:
        """Per-kernel CUDA-event timing of later applies (resets totals)."""
        check(load().dage_op3d_set_timing(self._h, int(bool(enable))))

    def timing(self, kind: int = 0):
        """(launches, total ms) of one kernel kind since set_timing():
        0 = contraction stages, 1 = precision split, 2 = finalize."""
        n = ctypes.c_longlong()
        ms = ctypes.c_double()
        check(load().dage_op3d_get_timing(self._h, kind, ctypes.byref(n), ctypes.byref(ms)))
        return n.value, ms.value

    @property
    def last_time_ms(self) -> float:
        v = ctypes.c_float()
        check(load().dage_op3d_last_time_ms(self._h, ctypes.byref(v)))
        return v.value

    # -- application ------------------------------------------------------
    def apply(self, rho, out=None, energy: bool = False, coda: bool = True,
              accumulate: bool = False):
        """V = self .apply. rho.  Returns V, or (V, integral of rho*V) when
        ``energy`` is set.  ``rho``/``out`` may be host (numpy, Fortran
        order) or device (torch CUDA) cubes; the output follows the input."""
        nin = int(np.prod(self.gridin.shape))
        nout = int(np.prod(self.gridout.shape))
        rp, rdev = _ptr(rho, nin)
        if out is None:
            if rdev:
                import torch

                out = torch.zeros(self.gridout.shape[::-1], dtype=torch.float64,
                                  device=rho.device)
            else:
                out = np.zeros(self.gridout.shape, order="F")
        vp, vdev = _ptr(out, nout)
        if rdev != vdev:
            raise ValueError("rho and out must both be host or both be device cubes")
        flags = (_capi.DAGE_DEVICE_PTRS if rdev else 0) | (_capi.DAGE_ENERGY if energy else 0)
        flags |= 0 if coda else _capi.DAGE_NO_CODA
        flags |= _capi.DAGE_ACCUMULATE if accumulate else 0
        e = ctypes.c_double(0.0)
        check(load().dage_op3d_apply(self._h, rp, vp, flags, ctypes.byref(e)))
        return (out, e.value) if energy else out

    __call__ = apply

    def operate_on(self, cube, bubbles: "Bubbles | None" = None, out=None):
        """Operator3D_operate_on_Function3D (function3d.F90:3727-3882) for a
        function held as a cube plus bubbles: (V cube, V bubbles) with the
        cube operator applied to the cube and the radial Coulomb potential
        of the bubbles (coulomb.F90:222-336; None without bubbles)."""
        V = self.apply(cube, out)
        return V, (bubbles.coulomb_potential() if bubbles is not None else None)


def apply_batched(ops, rhos, outs, energy: bool = False, coda: bool = True):
    """Applies ops[i] to rhos[i] into outs[i] for every i, all queued before
    one wait per distinct operator (applies on distinct operators overlap on
    their streams).  Cubes: all host or all device.  Returns the energies
    (numpy array) when ``energy`` is set."""
    n = len(ops)
    if not (len(rhos) == len(outs) == n):
        raise ValueError("ops, rhos and outs need the same length")
    rp, vp, devs = [], [], set()
    for op, r, v in zip(ops, rhos, outs):
        p1, d1 = _ptr(r, int(np.prod(op.gridin.shape)))
        p2, d2 = _ptr(v, int(np.prod(op.gridout.shape)))
        rp.append(p1.value)
        vp.append(p2.value)
        devs.update((d1, d2))
    if len(devs) > 1:
        raise ValueError("cubes must all be host arrays or all CUDA tensors")
    dev = devs.pop() if devs else False
    flags = (_capi.DAGE_DEVICE_PTRS if dev else 0) | (_capi.DAGE_ENERGY if energy else 0)
    flags |= 0 if coda else _capi.DAGE_NO_CODA
    arr = lambda xs: (ctypes.c_void_p * n)(*xs)
    e = np.zeros(max(n, 1))
    check(load().dage_op3d_apply_batched(n, arr([op._h.value for op in ops]), arr(rp), arr(vp),
                                         flags, e.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    return e[:n] if energy else None


class Coulomb3D(Operator3D):
    """Coulomb3D (src/bubbles/coulomb.F90:109-195), cube part:
    w_p = 2/sqrt(pi) tw_p, coda = pi/tlog^2."""


class Helmholtz3D:
    """Helmholtz3D (src/bubbles/helmholtz3d.F90:367-481): a Coulomb operator
    whose weights are rescaled to 2/sqrt(pi) tw_p exp(2E/(4 t_p^2)) for the
    duration of one application, then reset to E = 0."""

    def __init__(self, coulomb_operator: Operator3D, energy: float):
        self.coulomb_operator = coulomb_operator
        self.energy = energy

    def set_energy(self, energy: float) -> None:
        self.energy = energy
        check(load().dage_op3d_set_energy(self.coulomb_operator._h, float(energy)))

    def apply(self, rho, out=None, energy: bool = False, coda: bool = True):
        self.set_energy(self.energy)
        try:
            return self.coulomb_operator.apply(rho, out, energy=energy, coda=coda)
        finally:
            check(load().dage_op3d_set_energy(self.coulomb_operator._h, 0.0))

    __call__ = apply

    def operate_on(self, cube, bubbles: "Bubbles | None" = None, out=None):
        """Helmholtz3D_operate (helmholtz3d.F90:445-481): the cube operator at
        this energy applied to the cube, and the radial Helmholtz potential
        of the bubbles (Helmholtz3D_transform_bubbles_sub, :519-650; None
        without bubbles)."""
        V = self.apply(cube, out)
        return V, (bubbles.helmholtz_potential(self.energy) if bubbles is not None else None)


def set_tune_cache(path: str | None) -> None:
    """Autotuner cache file: tile-width choices are read from it and appended
    to it, keyed on the problem and the device (None: this process only)."""
    check(load().dage_set_tune_cache(path.encode() if path else None))


def integrate(grid: Grid3D, f1, f2=None) -> float:
    """Cube part of Function3D_integrate / Function3D_dot_product: the
    LIP-weighted integral of f1 (times f2 when given)."""
    n = int(np.prod(grid.shape))
    p1, d1 = _ptr(f1, n)
    p2, d2 = (ctypes.c_void_p(0), d1) if f2 is None else _ptr(f2, n)
    if d1 != d2:
        raise ValueError("f1 and f2 must both be host or both be device cubes")
    out = ctypes.c_double()
    g = grid.c()
    check(load().dage_integrate(g, p1, p2, _capi.DAGE_DEVICE_PTRS if d1 else 0,
                                ctypes.byref(out)))
    return out.value


dot = integrate


class GBFMMCoulomb3D:
    """GBFMMCoulomb3D (src/gbfmm/gbfmm_coulomb3d.F90:331-819), FP64: near
    field by per-box sub-operators, far field by multipoles (lmax) and M2L,
    2^maxlevel boxes per axis.  The near-field quadrature defaults to the
    reference's GaussQuad(25, 25).  ``adaptive_mode``: the reference's
    adaptive mode (gbfmm_coulomb3d.F90:374-384, 1386-1433): multipoles up to
    level 1, and neighbours of a box's parent that hold none of the box's
    nearest neighbours interact as whole parent-level boxes.
    ``precision``: "fp64" (the drop-in) or "fp16x3" (the near field on the
    tensor cores in the split precision; multipoles, M2L and L2P stay FP64)."""

    def __init__(self, grid: Grid3D, lmax: int = 12, maxlevel: int = 2,
                 quad: GaussQuad | None = None, adaptive_mode: bool = False,
                 precision: str = "fp64"):
        lib = load()
        self.grid = grid
        self.lmax = lmax
        self.maxlevel = maxlevel
        self.adaptive_mode = adaptive_mode
        if precision not in ("fp64", "fp16x3"):
            raise ValueError("GBFMM precision must be 'fp64' or 'fp16x3'")
        self.precision = precision
        self.quad = quad if quad is not None else GaussQuad(25, 25)
        self._keep = (grid.c(), self.quad.c())
        h = ctypes.c_void_p()
        create = lib.dage_gbfmm_create_adaptive if adaptive_mode else lib.dage_gbfmm_create
        check(create(self._keep[0], maxlevel, lmax, ctypes.byref(self._keep[1]),
                     PRECISIONS[precision], ctypes.byref(h)))
        self._h = h
        nb, nlm = ctypes.c_int(), ctypes.c_int()
        check(lib.dage_gbfmm_box_count(h, ctypes.byref(nb), ctypes.byref(nlm)))
        self.nbox, self.nlm = nb.value, nlm.value

    @property
    def tiles(self):
        """Near-field stage tile widths chosen by the autotuner (x, y, z)."""
        t = (ctypes.c_int * 3)()
        check(load().dage_gbfmm_tiles(self._h, t))
        return tuple(t)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                load().dage_gbfmm_destroy(h)
            except Exception:
                pass
            self._h = None

    def apply(self, rho, out=None, energy: bool = False):
        n = int(np.prod(self.grid.shape))
        rp, rdev = _ptr(rho, n)
        if out is None:
            if rdev:
                import torch

                out = torch.zeros(self.grid.shape[::-1], dtype=torch.float64, device=rho.device)
            else:
                out = np.zeros(self.grid.shape, order="F")
        vp, vdev = _ptr(out, n)
        if rdev != vdev:
            raise ValueError("rho and out must both be host or both be device cubes")
        flags = (_capi.DAGE_DEVICE_PTRS if rdev else 0) | (_capi.DAGE_ENERGY if energy else 0)
        e = ctypes.c_double(0.0)
        check(load().dage_gbfmm_apply(self._h, rp, vp, flags, ctypes.byref(e)))
        return (out, e.value) if energy else out

    __call__ = apply

    def multipole_moments(self, rho) -> np.ndarray:
        """(N_lm, nbox) moments, boxes in the reference's octree order."""
        n = int(np.prod(self.grid.shape))
        rp, rdev = _ptr(rho, n)
        q = np.zeros((self.nlm, self.nbox), order="F")
        check(load().dage_gbfmm_multipole_moments(
            self._h, rp, _capi.DAGE_DEVICE_PTRS if rdev else 0,
            q.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return q

    def local_expansions(self) -> np.ndarray:
        L = np.zeros((self.nlm, self.nbox), order="F")
        check(load().dage_gbfmm_local_expansions(self._h,
                                                 L.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return L

    def evaluate_local_expansions(self, L, V):
        """V += far-field potential of the local expansions L (N_lm, nbox)."""
        L = np.asfortranarray(L, dtype=np.float64)
        n = int(np.prod(self.grid.shape))
        vp, vdev = _ptr(V, n)
        check(load().dage_gbfmm_evaluate_le(self._h, L.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                            vp, _capi.DAGE_DEVICE_PTRS if vdev else 0))
        return V

    @property
    def last_time_ms(self) -> float:
        v = ctypes.c_float()
        check(load().dage_gbfmm_last_time_ms(self._h, ctypes.byref(v)))
        return v.value




class GBFMMHelmholtz3D(GBFMMCoulomb3D):
    """GBFMMHelmholtz3D (src/gbfmm/gbfmm_helmholtz3d.F90:241-1105): the GBFMM
    operator with the kernel e^(-kappa r)/r, kappa = sqrt(-2 energy)."""

    def __init__(self, grid: Grid3D, energy: float, lmax: int = 12, maxlevel: int = 2,
                 quad: GaussQuad | None = None, precision: str = "fp64",
                 adaptive_mode: bool = False):
        super().__init__(grid, lmax=lmax, maxlevel=maxlevel, quad=quad, precision=precision,
                         adaptive_mode=adaptive_mode)
        self.set_energy(energy)

    def set_energy(self, energy: float) -> None:
        check(load().dage_gbfmm_set_energy(self._h, float(energy)))
        self.energy = float(energy)

class GBFMMBatch:
    """Many independent densities through the GBFMM Coulomb operator at once
    (config: hundreds of orbitals of uneven grid sizes in one SCF step).
    Densities on equal grids share one plan; each pipeline stage is one
    launch over all densities, and the pipeline runs as a CUDA graph
    captured for the set of device cubes it is given.  ``precision``:
    "fp64" or "fp16x3" (near field on the tensor cores)."""

    def __init__(self, grids, lmax: int = 12, maxlevel: int = 2,
                 quad: GaussQuad | None = None, near_budget_bytes: int = 0,
                 precision: str = "fp64"):
        lib = load()
        if precision not in ("fp64", "fp16x3"):
            raise ValueError("GBFMM precision must be 'fp64' or 'fp16x3'")
        self.precision = precision
        self.grids = list(grids)
        self.lmax = lmax
        self.quad = quad if quad is not None else GaussQuad(25, 25)
        axes = [a.c() for g in self.grids for a in g.axes]
        arr = (DageGrid1D * len(axes))(*axes)
        self._keep = (arr, self.grids, self.quad.c())
        h = ctypes.c_void_p()
        check(lib.dage_gbfmm_batch_create(len(self.grids), arr, maxlevel, lmax,
                                          ctypes.byref(self._keep[2]), PRECISIONS[precision],
                                          near_budget_bytes, ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                load().dage_gbfmm_batch_destroy(h)
            except Exception:
                pass
            self._h = None

    def set_energies(self, energies) -> None:
        """Per-density kernel: energy < 0 gives e^(-kappa r)/r, kappa = sqrt(-2 E);
        0 the Coulomb kernel."""
        e = np.ascontiguousarray(energies, dtype=np.float64)
        if e.size != len(self.grids):
            raise ValueError("one energy per density")
        check(load().dage_gbfmm_batch_set_energies(
            self._h, e.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))

    def set_bubbles(self, bubbles, factors, lmin: int = 0) -> None:
        """First pipeline stage: rho_i += factors[i] * bubbles, in place, before the
        operator (None removes it).  Keep the Bubbles object alive meanwhile."""
        if bubbles is None:
            check(load().dage_gbfmm_batch_set_bubbles(self._h, None, None, 0))
            self._bubbles = None
            return
        f = np.ascontiguousarray(factors, dtype=np.float64)
        if f.size != len(self.grids):
            raise ValueError("one factor per density")
        self._bubbles = (bubbles, f)
        check(load().dage_gbfmm_batch_set_bubbles(
            self._h, bubbles._h, f.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), lmin))

    def info(self):
        """(plans, near-field chunks, tile widths, nodes of the captured graph)."""
        npl, nch, nodes = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        t = (ctypes.c_int * 3)()
        check(load().dage_gbfmm_batch_info(self._h, ctypes.byref(npl), ctypes.byref(nch), t,
                                           ctypes.byref(nodes)))
        return npl.value, nch.value, tuple(t), nodes.value

    @property
    def last_time_ms(self) -> float:
        v = ctypes.c_float()
        check(load().dage_gbfmm_batch_last_time_ms(self._h, ctypes.byref(v)))
        return v.value

    def apply(self, rhos, outs, energy: bool = False, graph: bool = True):
        """outs[i] = GBFMM potential of rhos[i] (all host numpy or all device
        torch cubes); returns the per-density energies with energy=True."""
        n = len(self.grids)
        if len(rhos) != n or len(outs) != n:
            raise ValueError(f"need {n} input and output cubes")
        rp = (ctypes.c_void_p * n)()
        vp = (ctypes.c_void_p * n)()
        devs = set()
        for i, g in enumerate(self.grids):
            m = int(np.prod(g.shape))
            rp[i], d1 = _ptr(rhos[i], m)
            vp[i], d2 = _ptr(outs[i], m)
            devs.update((d1, d2))
        if len(devs) != 1:
            raise ValueError("cubes must all be host or all be device cubes")
        flags = (_capi.DAGE_DEVICE_PTRS if devs.pop() else 0) | (_capi.DAGE_ENERGY if energy else 0)
        if not graph:
            flags |= _capi.DAGE_NO_GRAPH
        e = np.zeros(n)
        check(load().dage_gbfmm_batch_apply(self._h, rp, vp, flags,
                                            e.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return e if energy else None

class Bubbles:
    """Atom-centred radial functions times real spherical harmonics
    (Bubbles, src/bubbles/bubbles.F90), uploaded once for GPU injection into
    cubes (Function3D_inject_bubbles, function3d.F90:1757-1787)."""

    def __init__(self, centers, radial_grids, f, lmax: int, k: int = 0):
        lib = load()
        c = np.ascontiguousarray(np.asarray(centers, dtype=np.float64).reshape(-1, 3))
        self.natom = len(c)
        self.lmax = lmax
        self._grids = list(radial_grids)
        arr = (DageGrid1D * self.natom)(*[gr.c() for gr in self._grids])
        ff = np.ascontiguousarray(np.concatenate([np.asarray(a, dtype=np.float64).reshape(-1) for a in f]))
        h = ctypes.c_void_p()
        dp = ctypes.POINTER(ctypes.c_double)
        check(lib.dage_bubbles_create(self.natom, c.ctypes.data_as(dp), arr, lmax, k,
                                      ff.ctypes.data_as(dp), ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                load().dage_bubbles_destroy(h)
            except Exception:
                pass
            self._h = None

    @classmethod
    def _wrap(cls, handle, like: "Bubbles") -> "Bubbles":
        obj = cls.__new__(cls)
        obj.natom = like.natom
        obj.lmax = like.lmax
        obj._grids = like._grids
        obj._h = handle
        return obj

    def coulomb_potential(self) -> "Bubbles":
        """The radial Coulomb potential of these bubbles as a bubble set of
        its own (Coulomb3D_evaluate_bubbles_potential, coulomb.F90:222-336),
        computed on the GPU."""
        h = ctypes.c_void_p()
        check(load().dage_bubbles_coulomb_potential(self._h, ctypes.byref(h)))
        return Bubbles._wrap(h, self)

    def helmholtz_potential(self, energy: float) -> "Bubbles":
        """The radial potential of these bubbles for the kernel
        e^(-kappa r)/r, kappa = sqrt(-2 energy) (Helmholtz3D_bubbles,
        helmholtz3d.F90:506-650), computed on the GPU."""
        h = ctypes.c_void_p()
        check(load().dage_bubbles_helmholtz_potential(self._h, float(energy), ctypes.byref(h)))
        return Bubbles._wrap(h, self)

    def integrate(self) -> float:
        """Integral of the bubbles over all space (Bubbles_integrate_all,
        bubbles.F90:3146-3240): 4 pi sum_A int r^(2+k) f_A,00 dr, on the GPU."""
        out = ctypes.c_double()
        check(load().dage_bubbles_integrate(self._h, ctypes.byref(out)))
        return out.value

    def radial_values(self):
        """Per atom, the ((lmax+1)^2, npoints) radial values (as given)."""
        sizes = [int(gr.ncell * (gr.nlip - 1) + 1) for gr in self._grids]
        N = (self.lmax + 1) ** 2
        flat = np.zeros(N * sum(sizes))
        check(load().dage_bubbles_get_f(self._h, flat.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        out, o = [], 0
        for npts in sizes:
            out.append(flat[o:o + N * npts].reshape(N, npts))
            o += N * npts
        return out

    def multiply(self, other: "Bubbles", complete: bool = False) -> "Bubbles":
        """Radial product with another bubble set on the same atoms and radial
        grids (BubblesMultiplier_multiply, bubbles.F90:3567-3690): lmax and k
        add.  ``complete`` also keeps the terms with L < |m1 - m2| that the
        reference's product table (harmonic.F90:914-926) leaves out."""
        h = ctypes.c_void_p()
        check(load().dage_bubbles_multiply(self._h, other._h,
                                           _capi.DAGE_PRODUCT_COMPLETE if complete else 0,
                                           ctypes.byref(h)))
        res = Bubbles._wrap(h, self)
        res.lmax = self.lmax + other.lmax
        return res

    __mul__ = multiply

    def contaminants(self, tmax: int = 2) -> np.ndarray:
        """Bubble contaminants (Bubbles_get_contaminants, bubbles.F90:2844-2910):
        (natom, ncart) array whose row B holds the partial derivatives
        d^kappa, |kappa| <= tmax (CartIter order), of the other atoms'
        bubbles at atom B, computed on the GPU."""
        nc = (tmax + 1) * (tmax + 2) * (tmax + 3) // 6
        out = np.zeros((self.natom, nc))
        check(load().dage_bubbles_contaminants(self._h, int(tmax),
                                               out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def make_taylor(self, bubble_contaminants=None, cube_contaminants=None, tmax: int = 2,
                    exact: bool = False) -> "Bubbles":
        """Taylor-series bubbles from contaminants (Bubbles_make_taylor,
        bubbles.F90:1435-1530); lmax = max(self.lmax, tmax).  ``exact`` uses
        the true Taylor series instead of the reference's |kappa|! and dvpos
        conventions."""
        nc = (tmax + 1) * (tmax + 2) * (tmax + 3) // 6
        dp = ctypes.POINTER(ctypes.c_double)

        def arr(a):
            if a is None:
                return None, None
            a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(self.natom, nc))
            return a, a.ctypes.data_as(dp)
        cb, pb = arr(bubble_contaminants)
        cc, pc = arr(cube_contaminants)
        h = ctypes.c_void_p()
        check(load().dage_bubbles_make_taylor(self._h, pb, pc, int(tmax),
                                              _capi.DAGE_TAYLOR_EXACT if exact else 0,
                                              ctypes.byref(h)))
        res = Bubbles._wrap(h, self)
        res.lmax = max(self.lmax, tmax)
        return res

    def taylor_series(self, grid: Grid3D | None = None, cube=None, tmax: int = 2,
                      ignore_bubbles: bool = False, exact: bool = False) -> "Bubbles":
        """Taylor-series contaminant bubbles of the function cube + self
        (Function3D_get_taylor_series_bubbles, function3d.F90:1332-1405): the
        contaminants of the other atoms' bubbles and of the cube (when given,
        host array or CUDA tensor) at every atom, turned into bubbles, all on
        the GPU."""
        flags = (_capi.DAGE_TAYLOR_EXACT if exact else 0) | \
            (_capi.DAGE_TAYLOR_IGNORE_BUBBLES if ignore_bubbles else 0)
        p, g = None, None
        if cube is not None:
            if grid is None:
                raise ValueError("a cube needs its grid")
            p, dev = _ptr(cube, int(np.prod(grid.shape)))
            g = grid.c()
            if dev:
                flags |= _capi.DAGE_DEVICE_PTRS
        h = ctypes.c_void_p()
        check(load().dage_bubbles_taylor(self._h, g, p, int(tmax), flags, ctypes.byref(h)))
        res = Bubbles._wrap(h, self)
        res.lmax = max(self.lmax, tmax)
        return res

    def multiply_taylor(self, other: "Bubbles", taylor_self: "Bubbles", taylor_other: "Bubbles",
                        complete: bool = False) -> "Bubbles":
        """Radial product with Taylor series (option (1) of
        BubblesMultiplier_multiply, bubbles.F90:3567-3640):
        (self + taylor_self)(other + taylor_other) - taylor_self taylor_other,
        each Taylor set cut at its bubbles' lmax; lmax and k add."""
        h = ctypes.c_void_p()
        check(load().dage_bubbles_multiply_taylor(self._h, other._h, taylor_self._h,
                                                  taylor_other._h,
                                                  _capi.DAGE_PRODUCT_COMPLETE if complete else 0,
                                                  ctypes.byref(h)))
        res = Bubbles._wrap(h, self)
        res.lmax = self.lmax + other.lmax
        return res

    def inject(self, grid: Grid3D, cube=None, lmin: int = 0, factor: float = 1.0):
        """cube += factor * bubbles at the grid points; returns the cube."""
        n = int(np.prod(grid.shape))
        if cube is None:
            cube = np.zeros(grid.shape, order="F")
        p, dev = _ptr(cube, n)
        g = grid.c()
        check(load().dage_bubbles_inject(self._h, g, lmin, float(factor), p,
                                         _capi.DAGE_DEVICE_PTRS if dev else 0))
        return cube


def cube_contaminants(grid: Grid3D, cube, centers, tmax: int = 2) -> np.ndarray:
    """Cube contaminants (Function3D_get_cube_contaminants,
    function3d.F90:1570-1624): (natom, ncart) partial derivatives of the
    cube's LIP interpolant at the centres, 0 outside the grid; the cube is a
    host array or a CUDA tensor."""
    c = np.ascontiguousarray(np.asarray(centers, dtype=np.float64).reshape(-1, 3))
    nc = (tmax + 1) * (tmax + 2) * (tmax + 3) // 6
    out = np.zeros((len(c), nc))
    p, dev = _ptr(cube, int(np.prod(grid.shape)))
    dp = ctypes.POINTER(ctypes.c_double)
    check(load().dage_cube_contaminants(grid.c(), p, len(c), c.ctypes.data_as(dp), int(tmax),
                                        _capi.DAGE_DEVICE_PTRS if dev else 0,
                                        out.ctypes.data_as(dp)))
    return out


def cart2sph_table(tmax: int, exact: bool = False):
    """The monomial -> harmonic table of the Taylor bubbles (host only):
    list of (CartIter position, lm, coefficient)."""
    lib = load()
    flags = _capi.DAGE_TAYLOR_EXACT if exact else 0
    n = ctypes.c_int()
    check(lib.dage_cart2sph_table(int(tmax), flags, 0, None, None, None, ctypes.byref(n)))
    ki = (ctypes.c_int * n.value)()
    lm = (ctypes.c_int * n.value)()
    c = (ctypes.c_double * n.value)()
    check(lib.dage_cart2sph_table(int(tmax), flags, n.value, ki, lm, c, ctypes.byref(n)))
    return [(ki[i], lm[i], c[i]) for i in range(n.value)]


def multiply(grid: Grid3D, cube1, cube2, bubbles1: Bubbles | None = None,
             bubbles2: Bubbles | None = None, result_bubbles: Bubbles | None = None, out=None):
    """Cube part of the product of two functions (cube + bubbles each), as
    Function3D_multiply (function3d.F90:1097-1409) forms it:
    out = (cube1 + bubbles1)(cube2 + bubbles2) - result_bubbles, in one GPU
    pass.  ``result_bubbles`` is normally ``bubbles1 * bubbles2``."""
    n = int(np.prod(grid.shape))
    if out is None:
        out = cube1.new_empty(cube1.shape) if hasattr(cube1, "is_cuda") else np.zeros(grid.shape, order="F")
    p1, dev1 = _ptr(cube1, n)
    p2, dev2 = _ptr(cube2, n)
    po, devo = _ptr(out, n)
    if not (dev1 == dev2 == devo):
        raise ValueError("cubes must all be host arrays or all CUDA tensors")
    h = lambda b: b._h if b is not None else None
    check(load().dage_function3d_multiply(grid.c(), p1, h(bubbles1), p2, h(bubbles2),
                                          h(result_bubbles), po,
                                          _capi.DAGE_DEVICE_PTRS if dev1 else 0))
    return out
