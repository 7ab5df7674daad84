"""The allocation-free FP64 apply (dage_op3d_apply_fp64_noalloc), called
through the C ABI, against the regular entry point (dage_op3d_apply without
the coda) on the same operator matrices -- twice in a row, since every call
reuses the library's one fixed scratch array.  It is for callers that cannot
allocate device memory around the call (a caching allocator or fixed pool
owns the free memory, or the loop must avoid the device-wide sync of
cudaFree).  Collected last so a stop-at-first-failure run has run the rest."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_matrices(op, axis):
    import torch

    T = op.matrix(axis)  # T(i_out, j_in, p), column-major
    Tdev = np.ascontiguousarray(np.transpose(T, (2, 0, 1)))  # [p][i_out][j_in]
    return torch.from_numpy(Tdev).cuda()


@pytest.mark.parametrize("axes", [((-2.4, 4, 0.2),) * 3,
                                  ((-3.0, 5, 0.2), (-3.6, 6, 0.2), (-2.4, 4, 0.2))])
def test_noalloc_matches_regular_apply(dage, oracle, axes):
    import torch

    lib = dage.load()
    g = dage.Grid3D(tuple(dage.Grid1D.equidistant(*a) for a in axes))
    go = oracle.Grid3D(tuple(oracle.Grid1D.equidistant(*a) for a in axes))
    rho = oracle.gauss_cube(go, [1.0, -0.5], [1.7, 3.1], [[0.1, -0.2, 0.0], [-0.4, 0.3, 0.2]])
    op = dage.Coulomb3D(g, quad=dage.GaussQuad(6, 6))
    nx, ny, nz = g.shape
    rd = torch.from_numpy(rho.reshape(-1, order="F").copy()).cuda()
    Vref = op.apply(rd, coda=False)
    T = [_device_matrices(op, d) for d in range(3)]
    _, w = op.quadrature()
    w = np.ascontiguousarray(w)
    dp = ctypes.POINTER(ctypes.c_double)
    for _ in range(2):
        V = torch.full((nx * ny * nz,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.dage_op3d_apply_fp64_noalloc(
            nx, ny, nz, nx, ny, nz, len(w), ctypes.c_void_p(T[0].data_ptr()),
            ctypes.c_void_p(T[1].data_ptr()), ctypes.c_void_p(T[2].data_ptr()),
            w.ctypes.data_as(dp), ctypes.c_void_p(rd.data_ptr()), ctypes.c_void_p(V.data_ptr()),
            None)
        assert rc == 0, lib.dage_last_error()
        torch.cuda.synchronize()
        ref = Vref.reshape(-1)
        assert torch.isfinite(V).all()
        assert (V - ref).abs().max().item() <= 1e-12 * ref.abs().max().item()


def test_noalloc_on_a_caller_stream(dage, oracle):
    """All stage launches go to the stream the caller passes: the result is
    complete once that stream (and nothing else) has been synchronised."""
    import torch

    lib = dage.load()
    axes = ((-3.0, 5, 0.2),) * 3
    g = dage.Grid3D(tuple(dage.Grid1D.equidistant(*a) for a in axes))
    go = oracle.Grid3D(tuple(oracle.Grid1D.equidistant(*a) for a in axes))
    rho = oracle.gauss_cube(go, [1.3], [2.2], [[0.2, -0.1, 0.3]])
    op = dage.Coulomb3D(g, quad=dage.GaussQuad(6, 6))
    nx, ny, nz = g.shape
    rd = torch.from_numpy(rho.reshape(-1, order="F").copy()).cuda()
    Vref = op.apply(rd, coda=False).reshape(-1)
    T = [_device_matrices(op, d) for d in range(3)]
    _, w = op.quadrature()
    w = np.ascontiguousarray(w)
    dp = ctypes.POINTER(ctypes.c_double)
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    V = torch.full((nx * ny * nz,), float("nan"), dtype=torch.float64, device="cuda")
    rc = lib.dage_op3d_apply_fp64_noalloc(
        nx, ny, nz, nx, ny, nz, len(w), ctypes.c_void_p(T[0].data_ptr()),
        ctypes.c_void_p(T[1].data_ptr()), ctypes.c_void_p(T[2].data_ptr()),
        w.ctypes.data_as(dp), ctypes.c_void_p(rd.data_ptr()), ctypes.c_void_p(V.data_ptr()),
        ctypes.c_void_p(s.cuda_stream))
    assert rc == 0, lib.dage_last_error()
    s.synchronize()
    with torch.cuda.stream(s):
        err = (V - Vref).abs().max().item()
    assert err <= 1e-12 * Vref.abs().max().item()


def test_noalloc_rejects_cubes_beyond_its_scratch(dage):
    import torch

    lib = dage.load()
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(x.data_ptr())
    w = (ctypes.c_double * 1)(1.0)
    rc = lib.dage_op3d_apply_fp64_noalloc(241, 241, 241, 241, 241, 241, 1, p, p, p, w, p, p, None)
    assert rc == -1
    assert b"scratch" in lib.dage_last_error()
