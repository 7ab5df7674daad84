"""GPU tests of the split-precision tensor-core operator (tcgen05, BF16 or
FP16 parts, FP32 accumulation) against the FP64 GPU operator and the oracle.

Bars: bf16x6 and fp16x3 <= 1e-6 max-norm relative potential and <= 1e-7
relative energy (the targets) on every case; bf16x3 <= 1e-5 / 1e-5 (two
BF16 parts carry ~16 bits, a 2^-18 relative representation error per
element: it meets the targets on some workloads, e.g. 481^3, but not on the
121^3 single-box configuration, 1.8e-6 / 1.3e-7, nor on the Helmholtz case,
4.2e-6)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BARS = {"bf16x6": (1e-6, 1e-7), "fp16x3": (1e-6, 1e-7), "bf16x3": (1e-5, 1e-5)}
TARGET = ("bf16x6", "fp16x3")  # the modes held to the targets everywhere


def _case(dage, oracle, axes, quad, ng=3, seed=0):
    g = dage.Grid3D(tuple(dage.Grid1D.equidistant(q, n, h) for (q, n, h) in axes))
    go = oracle.Grid3D(tuple(oracle.Grid1D.equidistant(q, n, h) for (q, n, h) in axes))
    rng = np.random.default_rng(seed)
    lo = np.array([a.points[0] for a in go.axes])
    hi = np.array([a.points[-1] for a in go.axes])
    c = lo + (hi - lo) * rng.uniform(0.3, 0.7, (ng, 3))
    rho = oracle.gauss_cube(go, rng.uniform(0.5, 2, ng), rng.uniform(0.5, 5, ng), c)
    return g, go, rho, dage.GaussQuad(*quad)


def _errs(V, V64, E, E64):
    return np.abs(V - V64).max() / np.abs(V64).max(), abs(E - E64) / abs(E64)


@pytest.mark.parametrize("prec", ["bf16x6", "fp16x3", "bf16x3"])
@pytest.mark.parametrize("axes,quad", [
    (((-2.4, 4, 0.2),) * 3, (2, 2, 0.0, 2.0, 1e3)),          # 25^3, one K block
    (((-3.0, 5, 0.2), (-3.6, 6, 0.2), (-2.4, 4, 0.2)), (6, 6, 0.0, 2.0, 1e3)),  # 31x37x25
    (((-6.0, 10, 0.2),) * 3, (8, 8, 0.0, 2.0, 1e3)),        # 61^3
])
def test_mixed_vs_fp64(dage, oracle, prec, axes, quad):
    g, go, rho, q = _case(dage, oracle, axes, quad)
    op64 = dage.Coulomb3D(g, quad=q)
    V64, E64 = op64.apply(rho, energy=True)
    op = dage.Coulomb3D(g, quad=q, precision=prec)
    V, E = op.apply(rho, energy=True)
    ev, ee = _errs(V, V64, E, E64)
    assert ev <= BARS[prec][0], ev
    assert ee <= BARS[prec][1], ee


@pytest.mark.parametrize("prec", ["bf16x6", "fp16x3", "bf16x3"])
def test_mixed_config1_121(dage, oracle, prec):
    """The single-box configuration (121^3, 2 Gaussians, 40 t-points): the
    target bars, 1e-6 potential and 1e-7 energy, for bf16x6 and fp16x3;
    bf16x3 misses them here (1.8e-6 / 1.3e-7) and is held to 3e-6 / 3e-7."""
    rng = np.random.default_rng(1)
    q = rng.uniform(0.5, 2, 2)
    a = rng.uniform(0.5, 4, 2)
    c = rng.uniform(-3, 3, (2, 3))
    g = dage.Grid3D.cube(-12.0, 20, 0.2)
    go = oracle.Grid3D.cube(-12.0, 20, 0.2)
    rho = oracle.gauss_cube(go, q, a, c)
    quad = dage.GaussQuad(20, 20, 0.0, 2.0, 1e3)
    V64, E64 = dage.Coulomb3D(g, quad=quad).apply(rho, energy=True)
    V, E = dage.Coulomb3D(g, quad=quad, precision=prec).apply(rho, energy=True)
    ev, ee = _errs(V, V64, E, E64)
    print(f"  {prec} at 121^3: potential {ev:.2e}, energy {ee:.2e}")
    bar = (1e-6, 1e-7) if prec in TARGET else (3e-6, 3e-7)
    assert ev <= bar[0] and ee <= bar[1], (ev, ee)


def test_mixed_repeatable_and_linear(dage, oracle):
    """Deterministic (bitwise repeatable) and linear in rho within the bar."""
    g, go, rho, q = _case(dage, oracle, ((-3.0, 5, 0.2),) * 3, (6, 6, 0.0, 2.0, 1e3))
    op = dage.Coulomb3D(g, quad=q, precision="bf16x6")
    V1 = op.apply(rho)
    V2 = op.apply(rho)
    np.testing.assert_array_equal(V1, V2)
    V3 = op.apply(np.asfortranarray(2.5 * rho))
    assert np.abs(V3 - 2.5 * V1).max() <= 2e-6 * np.abs(V3).max()


def test_mixed_helmholtz(dage, oracle):
    g, go, rho, q = _case(dage, oracle, ((-3.0, 5, 0.2),) * 3, (8, 8, 0.0, 2.0, 1e3))
    E = -0.5 * 1.2 ** 2
    V64 = dage.Helmholtz3D(dage.Coulomb3D(g, quad=q), E).apply(rho)
    for prec in ("bf16x6", "fp16x3", "bf16x3"):
        V = dage.Helmholtz3D(dage.Coulomb3D(g, quad=q, precision=prec), E).apply(rho)
        err = np.abs(V - V64).max() / np.abs(V64).max()
        print(f"  {prec} Helmholtz: potential {err:.2e}")
        assert err <= (1e-6 if prec in TARGET else 1e-5), (prec, err)


def test_mixed_device_pointers(dage, oracle):
    import torch

    g, go, rho, q = _case(dage, oracle, ((-2.4, 4, 0.2),) * 3, (4, 4, 0.0, 2.0, 1e3))
    op = dage.Coulomb3D(g, quad=q, precision="bf16x6")
    Vh = op.apply(rho)
    Vd = op.apply(torch.from_numpy(rho.reshape(-1, order="F").copy()).cuda())
    np.testing.assert_array_equal(Vd.cpu().numpy().reshape(-1), Vh.reshape(-1, order="F"))


def test_headline_workload_meets_the_bounds(dage):
    """The 481^3 workload that bench.py times (32 Gaussians, 64 t-points):
    every split-precision mode within 1e-6 max-norm relative potential and
    1e-7 relative energy of the FP64 GPU operator."""
    import torch

    import bench

    g = dage.Grid3D.cube(-0.5 * bench.N_CELL * 6 * bench.STEP, bench.N_CELL, bench.STEP)
    quad = dage.GaussQuad(bench.NLIN, bench.NLOG, 0.0, bench.TLIN, bench.TLOG)
    q, a, c = bench.gaussians()
    rho = bench.density_torch(bench.axis_points(), q, a, c, torch.device("cuda"))
    V64 = torch.empty_like(rho)
    _, E64 = dage.Coulomb3D(g, quad=quad).apply(rho, out=V64, energy=True)
    scale = V64.abs().max().item()
    for prec in ("bf16x3", "bf16x6", "fp16x3"):
        V = torch.empty_like(rho)
        _, E = dage.Coulomb3D(g, quad=quad, precision=prec).apply(rho, out=V, energy=True)
        err = (V - V64).abs().max().item() / scale
        print(f"  {prec} at 481^3: potential {err:.2e}, energy {abs(E - E64) / abs(E64):.2e}")
        assert err <= 1e-6, (prec, err)
        assert abs(E - E64) <= 1e-7 * abs(E64), (prec, abs(E - E64) / abs(E64))
