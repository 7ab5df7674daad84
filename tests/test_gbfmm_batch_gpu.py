"""GPU tests of the batched GBFMM (many independent densities of uneven grid
sizes, one launch per pipeline stage, CUDA-graph replay) against the
single-density GBFMM apply, which the GBFMM tests check against the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

QUAD = (6, 6, 0.0, 2.0, 1e3)


def _densities(dage, oracle, ncells, step=0.2, seed=11):
    rng = np.random.default_rng(seed)
    grids, rhos = [], []
    for ncell in ncells:
        half = 0.5 * ncell * 6 * step
        grids.append(dage.Grid3D.cube(-half, ncell, step))
        go = oracle.Grid3D.cube(-half, ncell, step)
        ng = int(rng.integers(1, 9))
        q = rng.uniform(-1, 2, ng)
        a = rng.uniform(0.3, 6, ng)
        c = rng.uniform(-0.6 * half, 0.6 * half, (ng, 3))
        rhos.append(np.asfortranarray(oracle.gauss_cube(go, q, a, c)))
    return grids, rhos


def _single(dage, grid, rho, lmax):
    op = dage.GBFMMCoulomb3D(grid, lmax=lmax, quad=dage.GaussQuad(*QUAD))
    return op.apply(rho, energy=True)


@pytest.mark.parametrize("budget", [0, 1 << 20])  # 1 MiB: one density per near-field chunk
def test_batch_matches_single(dage, oracle, budget):
    ncells = [8, 10, 9, 8, 10]  # uneven box splits, shared plans for equal sizes
    lmax = 6
    grids, rhos = _densities(dage, oracle, ncells)
    batch = dage.GBFMMBatch(grids, lmax=lmax, quad=dage.GaussQuad(*QUAD),
                            near_budget_bytes=budget)
    outs = [np.zeros(g.shape, order="F") for g in grids]
    E = batch.apply(rhos, outs, energy=True)
    nplans, nchunks, tiles, _ = batch.info()
    assert nplans == 3
    assert (nchunks == 5) if budget else (nchunks == 1)
    assert set(tiles) <= {32, 64, 128}
    for g, rho, V, e in zip(grids, rhos, outs, E):
        V1, e1 = _single(dage, g, rho, lmax)
        assert np.abs(V - V1).max() <= 1e-13 * np.abs(V1).max()
        assert abs(e - e1) <= 1e-13 * abs(e1)


def test_batch_graph_replay_and_device_cubes(dage, oracle):
    import torch

    ncells = [8, 9, 8]
    lmax = 4
    grids, rhos = _densities(dage, oracle, ncells, seed=5)
    batch = dage.GBFMMBatch(grids, lmax=lmax, quad=dage.GaussQuad(*QUAD))
    dr = [torch.from_numpy(r.reshape(-1, order="F").copy()).cuda() for r in rhos]
    dv = [torch.empty_like(r) for r in dr]
    E1 = batch.apply(dr, dv, energy=True)  # capture + launch
    nodes = batch.info()[3]
    assert nodes > 0
    V1 = [v.clone() for v in dv]
    for r in dr:  # new values in the same cubes: the graph replays
        r.mul_(0.5)
    E2 = batch.apply(dr, dv, energy=True)
    assert batch.info()[3] == nodes
    for a, b in zip(V1, dv):
        assert torch.allclose(b, 0.5 * a, rtol=1e-14, atol=0)
    np.testing.assert_allclose(E2, 0.25 * E1, rtol=1e-13)
    # eager launch gives the same numbers
    dv2 = [torch.empty_like(r) for r in dr]
    E3 = batch.apply(dr, dv2, energy=True, graph=False)
    for a, b in zip(dv, dv2):
        assert torch.equal(a, b)
    np.testing.assert_array_equal(E2, E3)


def test_batch_helmholtz_energies(dage, oracle):
    ncells = [8, 9, 8, 9]
    lmax = 6
    energies = [-0.5, -1.1, 0.0, -0.5]  # two shared kernels, one Coulomb density
    grids, rhos = _densities(dage, oracle, ncells, seed=7)
    batch = dage.GBFMMBatch(grids, lmax=lmax, quad=dage.GaussQuad(*QUAD))
    batch.set_energies(energies)
    outs = [np.zeros(g.shape, order="F") for g in grids]
    E = batch.apply(rhos, outs, energy=True)
    for g, rho, V, e, en in zip(grids, rhos, outs, E, energies):
        op = (dage.GBFMMHelmholtz3D(g, en, lmax=lmax, quad=dage.GaussQuad(*QUAD)) if en < 0
              else dage.GBFMMCoulomb3D(g, lmax=lmax, quad=dage.GaussQuad(*QUAD)))
        V1, e1 = op.apply(rho, energy=True)
        assert np.abs(V - V1).max() <= 1e-13 * np.abs(V1).max()
        assert abs(e - e1) <= 1e-13 * abs(e1)


def test_batch_inject_stage(dage, oracle):
    """The optional first stage: rho_i += f_i * bubbles in place, then the operator,
    equal to an explicit injection followed by the single-density apply."""
    import torch

    ncells = [8, 9, 8]
    lmax = 4
    grids, rhos = _densities(dage, oracle, ncells, seed=7)
    h = oracle.log_radial_grid()
    rad = dage.Grid1D(0.0, 33, 7, 1, h)
    r = oracle.Grid1D(0.0, 33, 7, 1, h).points
    rng = np.random.default_rng(3)
    centers = rng.uniform(-1.5, 1.5, (3, 3))
    f = [np.stack([rng.uniform(0.5, 1.5) * r ** (1 if lm else 0) * np.exp(-2 * r)
                   for lm in range(4)]) for _ in range(3)]
    bub = dage.Bubbles(centers, [rad] * 3, f, 1)
    factors = [0.8, 0.0, -1.3]
    batch = dage.GBFMMBatch(grids, lmax=lmax, quad=dage.GaussQuad(*QUAD))
    batch.set_bubbles(bub, factors, lmin=0)
    dr = [torch.from_numpy(x.reshape(-1, order="F").copy()).cuda() for x in rhos]
    dv = [torch.empty_like(x) for x in dr]
    E = batch.apply(dr, dv, energy=True)
    for g, x, fac, r1, V, e in zip(grids, rhos, factors, dr, dv, E):
        ref = torch.from_numpy(x.reshape(-1, order="F").copy()).cuda()
        if fac:
            bub.inject(g, cube=ref, lmin=0, factor=fac)
        assert torch.equal(r1, ref)  # the stage ran in place on the input cube
        V1, e1 = _single(dage, g, ref.cpu().numpy().reshape(g.shape, order="F"), lmax)
        got = V.cpu().numpy().reshape(g.shape, order="F")
        assert np.abs(got - V1).max() <= 1e-13 * np.abs(V1).max()
        assert abs(e - e1) <= 1e-13 * abs(e1)
    # removing the stage: the cubes are left as they are
    batch.set_bubbles(None, None)
    before = [x.clone() for x in dr]
    batch.apply(dr, dv)
    for a, b in zip(before, dr):
        assert torch.equal(a, b)
