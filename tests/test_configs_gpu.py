"""GPU parity tests at the full sizes of the GBFMM configurations, against
the oracle directly:

- the FP64 GBFMM on the 241^3 grid (40 cells, step 0.2) in 4x4x4 boxes,
  lmax 12, 40 t-points, 16 Gaussians (alpha ~ U[0.3, 6], q ~ U[-1, 2],
  centres uniform inside the box);
- the batched GBFMM on one density of each grid size the batch workload
  draws from (61^3 .. 181^3, step 0.2, 1-8 Gaussians), every instance
  compared with the oracle's own GBFMM of that density.

Bars as in the other FP64 parity tests: the potential within max(1e-10,
10x the spread of the reference algorithm under +-1 ulp erf/exp, which only
the near-field matrices see), the energy within 1e-11 relative."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
QUAD = (20, 20, 0.0, 2.0, 1e3)
LMAX = 12


def _check(oracle, go, rho, V, E, energy=0.0):
    Vo, _, _, Vn = oracle.gbfmm_apply(go, rho, lmax=LMAX, quad=QUAD, return_parts=True,
                                      blas=True, energy=energy)
    Vn1 = oracle.gbfmm_near_field(go, rho, 2, QUAD, libm_1ulp=True, blas=True, energy=energy)
    scale = np.abs(Vo).max()
    spread = np.abs(Vn1 - Vn).max() / scale
    err = np.abs(V - Vo).max() / scale
    print(f"  {go.shape[0]}^3: potential {err:.2e} (libm spread {spread:.2e})")
    assert err <= max(1e-10, 10 * spread), (err, spread)
    Eo = oracle.integrate_cube(go, rho * Vo)
    assert abs(E - Eo) <= 1e-11 * abs(Eo), (E, Eo)


def test_gbfmm_241_sixteen_gaussians(dage, oracle):
    rng = np.random.default_rng(3)
    q, a = rng.uniform(-1, 2, 16), rng.uniform(0.3, 6, 16)
    c = rng.uniform(-24, 24, (16, 3))
    g = dage.Grid3D.cube(-24.0, 40, 0.2)
    go = oracle.Grid3D.cube(-24.0, 40, 0.2)
    rho = oracle.gauss_cube(go, q, a, c)
    op = dage.GBFMMCoulomb3D(g, lmax=LMAX, quad=dage.GaussQuad(*QUAD))
    V, E = op.apply(rho, energy=True)
    _check(oracle, go, rho, V, E)


def test_batch_every_grid_size_against_oracle(dage, oracle):
    rng = np.random.default_rng(5)
    grids, gos, rhos = [], [], []
    for ncell in (10, 15, 20, 25, 30):  # 61, 91, 121, 151, 181 points per axis
        half = 0.5 * ncell * 6 * 0.2
        grids.append(dage.Grid3D.cube(-half, ncell, 0.2))
        go = oracle.Grid3D.cube(-half, ncell, 0.2)
        ng = int(rng.integers(1, 9))
        q, a = rng.uniform(-1, 2, ng), rng.uniform(0.3, 6, ng)
        c = rng.uniform(-0.6 * half, 0.6 * half, (ng, 3))
        gos.append(go)
        rhos.append(np.asfortranarray(oracle.gauss_cube(go, q, a, c)))
    batch = dage.GBFMMBatch(grids, lmax=LMAX, quad=dage.GaussQuad(*QUAD))
    outs = [np.zeros(g.shape, order="F") for g in grids]
    E = batch.apply(rhos, outs, energy=True)
    for go, rho, V, e in zip(gos, rhos, outs, E):
        _check(oracle, go, rho, V, e)
