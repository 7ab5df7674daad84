"""GPU tests of the GBFMM near field in the fp16x3 split precision on the
tensor cores (grouped tcgen05 stages over all boxes, near_mixed.cu) against
the FP64 GBFMM on the same densities: single densities (Coulomb, Helmholtz,
adaptive mode, uneven and asymmetric box splits, both tile widths) and the
batch (uneven grid sizes, mixed Coulomb/Helmholtz kernels, graph replay).

Bars (the targets of the split precision): <= 1e-6 max-norm relative
potential and <= 1e-7 relative energy against the FP64 operator, whose own
parity with the oracle is tested in test_gbfmm_gpu.py / test_configs_gpu.py."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
QUAD = (10, 10, 0.0, 2.0, 1e3)
BAR_V, BAR_E = 1e-6, 1e-7


def _density(oracle, go, ng, seed):
    rng = np.random.default_rng(seed)
    lo = np.array([a.points[0] for a in go.axes])
    hi = np.array([a.points[-1] for a in go.axes])
    c = lo + (hi - lo) * rng.uniform(0.15, 0.85, (ng, 3))
    return oracle.gauss_cube(go, rng.uniform(-1, 2, ng), rng.uniform(0.3, 6, ng), c)


def _grids(dage, oracle, ncells, h=0.2):
    axes = [(-0.5 * n * 6 * h, n, h) for n in ncells]
    g = dage.Grid3D(tuple(dage.Grid1D.equidistant(q, n, hh) for (q, n, hh) in axes))
    go = oracle.Grid3D(tuple(oracle.Grid1D.equidistant(q, n, hh) for (q, n, hh) in axes))
    return g, go


def _errs(V, V64, E, E64):
    return np.abs(V - V64).max() / np.abs(V64).max(), abs(E - E64) / abs(E64)


@pytest.mark.parametrize("tile", ["64", "128"])
@pytest.mark.parametrize("ncells", [(10, 10, 10), (15, 15, 15), (10, 15, 20), (21, 14, 9)])
def test_mixed_gbfmm_matches_fp64(dage, oracle, monkeypatch, tile, ncells):
    monkeypatch.setenv("DAGE_NEAR16_TILE", tile)
    g, go = _grids(dage, oracle, ncells)
    rho = _density(oracle, go, 6, sum(ncells))
    q = dage.GaussQuad(*QUAD)
    V64, E64 = dage.GBFMMCoulomb3D(g, lmax=8, quad=q).apply(rho, energy=True)
    op = dage.GBFMMCoulomb3D(g, lmax=8, quad=q, precision="fp16x3")
    assert op.tiles == (int(tile),) * 3
    V, E = op.apply(rho, energy=True)
    ev, ee = _errs(V, V64, E, E64)
    print(f"{ncells} tile {tile}: potential {ev:.2e}, energy {ee:.2e}")
    assert ev <= BAR_V and ee <= BAR_E, (ev, ee)
    V2, E2 = op.apply(rho, energy=True)  # a second call reuses the set
    assert np.array_equal(V, V2) and E == E2


def test_mixed_gbfmm_helmholtz_and_adaptive(dage, oracle):
    g, go = _grids(dage, oracle, (15, 15, 15))
    rho = _density(oracle, go, 5, 11)
    q = dage.GaussQuad(*QUAD)
    h64 = dage.GBFMMHelmholtz3D(g, energy=-0.5, lmax=8, quad=q)
    h16 = dage.GBFMMHelmholtz3D(g, energy=-0.5, lmax=8, quad=q, precision="fp16x3")
    V64, E64 = h64.apply(rho, energy=True)
    V, E = h16.apply(rho, energy=True)
    ev, ee = _errs(V, V64, E, E64)
    print(f"helmholtz: potential {ev:.2e}, energy {ee:.2e}")
    assert ev <= BAR_V and ee <= BAR_E, (ev, ee)
    # back to the Coulomb kernel: the device weights follow set_energy
    h16.set_energy(0.0)
    V, E = h16.apply(rho, energy=True)
    Vc, Ec = dage.GBFMMCoulomb3D(g, lmax=8, quad=q).apply(rho, energy=True)
    ev, ee = _errs(V, Vc, E, Ec)
    assert ev <= BAR_V and ee <= BAR_E, (ev, ee)
    g3, go3 = _grids(dage, oracle, (16, 16, 16))
    rho3 = _density(oracle, go3, 5, 12)
    a64 = dage.GBFMMCoulomb3D(g3, lmax=8, maxlevel=3, quad=q, adaptive_mode=True)
    a16 = dage.GBFMMCoulomb3D(g3, lmax=8, maxlevel=3, quad=q, adaptive_mode=True,
                              precision="fp16x3")
    V64, E64 = a64.apply(rho3, energy=True)
    V, E = a16.apply(rho3, energy=True)
    ev, ee = _errs(V, V64, E, E64)
    print(f"adaptive maxlevel 3: potential {ev:.2e}, energy {ee:.2e}")
    assert ev <= BAR_V and ee <= BAR_E, (ev, ee)


def test_mixed_gbfmm_device_cubes(dage, oracle):
    import torch

    g, go = _grids(dage, oracle, (20, 20, 20))
    rho = _density(oracle, go, 8, 3)
    q = dage.GaussQuad(*QUAD)
    V64, E64 = dage.GBFMMCoulomb3D(g, lmax=12, quad=q).apply(rho, energy=True)
    op = dage.GBFMMCoulomb3D(g, lmax=12, quad=q, precision="fp16x3")
    rd = torch.from_numpy(rho.reshape(-1, order="F").copy()).cuda()
    V, E = op.apply(rd, energy=True)
    Vh = V.cpu().numpy().reshape(-1).reshape(go.shape, order="F")
    ev, ee = _errs(Vh, V64, E, E64)
    print(f"121^3 device cubes: potential {ev:.2e}, energy {ee:.2e}")
    assert ev <= BAR_V and ee <= BAR_E, (ev, ee)


def test_mixed_batch_matches_fp64(dage, oracle):
    grids, gos, rhos = [], [], []
    for i, ncell in enumerate((10, 15, 20, 10, 15, 12)):
        g, go = _grids(dage, oracle, (ncell,) * 3)
        grids.append(g)
        gos.append(go)
        rhos.append(np.asfortranarray(_density(oracle, go, 1 + i % 5, 40 + i)))
    q = dage.GaussQuad(*QUAD)
    energies = [0.0, -0.5, 0.0, -1.2, -0.5, 0.0]
    b64 = dage.GBFMMBatch(grids, lmax=8, quad=q)
    b64.set_energies(energies)
    out64 = [np.zeros(g.shape, order="F") for g in grids]
    E64 = b64.apply(rhos, out64, energy=True)
    # a small budget splits the densities of a plan over several sets
    b16 = dage.GBFMMBatch(grids, lmax=8, quad=q, precision="fp16x3",
                          near_budget_bytes=24 << 20)
    b16.set_energies(energies)
    for rep in range(2):  # capture, then replay
        out = [np.zeros(g.shape, order="F") for g in grids]
        E = b16.apply(rhos, out, energy=True)
        for i in range(len(grids)):
            ev, ee = _errs(out[i], out64[i], E[i], E64[i])
            print(f"batch {i} ({grids[i].shape[0]}^3, E={energies[i]}): {ev:.2e} {ee:.2e}")
            assert ev <= BAR_V and ee <= BAR_E, (i, ev, ee)
