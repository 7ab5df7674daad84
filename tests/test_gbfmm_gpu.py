"""GPU tests of the FP64 GBFMM Coulomb operator against the oracle
(multipoles, M2L local expansions, L2P, full potential and energy)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(dage, oracle, ncell, step, ng=6, seed=3):
    half = 0.5 * ncell * 6 * step
    g = dage.Grid3D.cube(-half, ncell, step)
    go = oracle.Grid3D.cube(-half, ncell, step)
    rng = np.random.default_rng(seed)
    q = rng.uniform(-1, 2, ng)
    a = rng.uniform(0.8, 6, ng)
    c = rng.uniform(-0.7 * half, 0.7 * half, (ng, 3))
    return g, go, oracle.gauss_cube(go, q, a, c)


def _oracle_moments(oracle, go, rho, lmax):
    plan = oracle.GBFMMPlan(go, 2)
    N = (lmax + 1) ** 2
    Q = np.zeros((N, plan.nbox))
    for b in range(1, plan.nbox + 1):
        (x0, x1), (y0, y1), (z0, z1) = plan.points(b)
        subs = [oracle.subgrid(a, c0, c1) for a, (c0, c1) in zip(go.axes, plan.cells(b))]
        Q[:, b - 1] = oracle.box_multipoles(lmax, subs[0].points, subs[0].weights(), subs[1].points,
                                            subs[1].weights(), subs[2].points, subs[2].weights(),
                                            rho[x0:x1, y0:y1, z0:z1], plan.center(b))
    return plan, Q


@pytest.mark.parametrize("ncell", [16, 15])  # 15 cells: uneven box split
def test_multipoles_and_local_expansions(dage, oracle, ncell):
    lmax = 10
    g, go, rho = _setup(dage, oracle, ncell, 0.2)
    op = dage.GBFMMCoulomb3D(g, lmax=lmax, quad=dage.GaussQuad(6, 6))
    Qg = op.multipole_moments(rho)
    plan, Qo = _oracle_moments(oracle, go, rho, lmax)
    for b in range(plan.nbox):
        assert np.abs(Qg[:, b] - Qo[:, b]).max() <= 1e-12 * np.abs(Qo[:, b]).max() + 1e-300
    op.apply(rho)
    Lg = op.local_expansions()
    Lo = np.zeros_like(Lg)
    for i in range(1, plan.nbox + 1):
        ci = plan.center(i)
        for j in oracle.local_farfield(i, 2):
            Lo[:, i - 1] += oracle.interaction_matrix(lmax, plan.center(j) - ci) @ Qo[:, j - 1]
    assert np.abs(Lg - Lo).max() <= 1e-11 * np.abs(Lo).max()


@pytest.mark.parametrize("ncell,lmax", [(16, 12), (15, 8), (20, 12)])
def test_gbfmm_apply_matches_oracle(dage, oracle, ncell, lmax):
    g, go, rho = _setup(dage, oracle, ncell, 0.2)
    quad = (8, 8, 0.0, 2.0, 1e3)
    op = dage.GBFMMCoulomb3D(g, lmax=lmax, quad=dage.GaussQuad(*quad))
    assert set(op.tiles) <= {32, 64, 128}  # near-field tile widths from the autotuner
    V, E = op.apply(rho, energy=True)
    Vo = oracle.gbfmm_apply(go, rho, lmax=lmax, quad=quad)
    V1 = oracle.gbfmm_apply(go, rho, lmax=lmax, quad=quad, libm_1ulp=True)
    spread = np.abs(V1 - Vo).max() / np.abs(Vo).max()
    err = np.abs(V - Vo).max() / np.abs(Vo).max()
    assert err <= max(1e-10, 10 * spread), (err, spread)
    Eo = oracle.integrate_cube(go, rho * Vo)
    assert abs(E - Eo) <= 1e-11 * abs(Eo)


def test_evaluate_local_expansions(dage, oracle):
    g, go, rho = _setup(dage, oracle, 16, 0.2)
    lmax = 6
    op = dage.GBFMMCoulomb3D(g, lmax=lmax, quad=dage.GaussQuad(4, 4))
    rng = np.random.default_rng(7)
    L = rng.standard_normal(((lmax + 1) ** 2, 64))
    V = np.zeros(go.shape, order="F")
    op.evaluate_local_expansions(L, V)
    plan = oracle.GBFMMPlan(go, 2)
    Vo = np.zeros(go.shape, order="F")
    for b in range(1, 65):
        own = plan.owned(b)
        pts = [go.axes[d].points[own[d][0]:own[d][1]] for d in range(3)]
        sub = np.zeros([len(p) for p in pts], order="F")
        oracle.l2p(lmax, L[:, b - 1], plan.center(b), pts[0], pts[1], pts[2], sub)
        Vo[own[0][0]:own[0][1], own[1][0]:own[1][1], own[2][0]:own[2][1]] = sub
    assert np.abs(V - Vo).max() <= 1e-12 * np.abs(Vo).max()


def test_gbfmm_close_to_direct_operator(dage, oracle):
    """GBFMM against the single-box FP64 operator on the GPU (no coda):
    the multipole truncation error of lmax 12."""
    g, go, rho = _setup(dage, oracle, 20, 0.2, ng=8)
    quad = dage.GaussQuad(12, 12)
    V, E = dage.GBFMMCoulomb3D(g, lmax=12, quad=quad).apply(rho, energy=True)
    Vd, Ed = dage.Coulomb3D(g, quad=quad).apply(rho, energy=True, coda=False)
    assert np.abs(V - Vd).max() / np.abs(Vd).max() < 5e-3
    assert abs(E - Ed) / abs(Ed) < 1e-3


@pytest.mark.parametrize("lmax", [0, 1, 2, 7, 15])  # lane-task splits: 32, 16, 10, 4, 2 points a pass
def test_multipoles_every_lmax(dage, oracle, lmax):
    g, go, rho = _setup(dage, oracle, 8, 0.2, seed=lmax)
    op = dage.GBFMMCoulomb3D(g, lmax=lmax, quad=dage.GaussQuad(4, 4))
    Qg = op.multipole_moments(rho)
    plan, Qo = _oracle_moments(oracle, go, rho, lmax)
    for b in range(plan.nbox):
        assert np.abs(Qg[:, b] - Qo[:, b]).max() <= 1e-12 * np.abs(Qo[:, b]).max() + 1e-300


@pytest.mark.parametrize("ncell,lmax", [(16, 8), (18, 6)])  # 18 cells: uneven, nested levels
def test_multilevel_matches_oracle(dage, oracle, ncell, lmax):
    """Three levels (8^3 finest boxes): moments, local expansions after
    M2M -> M2L at levels 2 and 3 -> L2L, and the full potential and energy
    against the oracle's restatement of the reference's multi-level passes."""
    g, go, rho = _setup(dage, oracle, ncell, 0.2)
    quad = (6, 6, 0.0, 2.0, 1e3)
    op = dage.GBFMMCoulomb3D(g, lmax=lmax, maxlevel=3, quad=dage.GaussQuad(*quad))
    V, E = op.apply(rho, energy=True)
    Vo, qo, Lo, _ = oracle.gbfmm_apply(go, rho, lmax=lmax, maxlevel=3, quad=quad,
                                       return_parts=True)
    Qg = op.multipole_moments(rho)
    assert np.abs(Qg - qo).max() <= 1e-12 * np.abs(qo).max()
    op.apply(rho)
    Lg = op.local_expansions()
    assert np.abs(Lg - Lo).max() <= 1e-11 * np.abs(Lo).max()
    V1 = oracle.gbfmm_apply(go, rho, lmax=lmax, maxlevel=3, quad=quad, libm_1ulp=True)
    spread = np.abs(V1 - Vo).max() / np.abs(Vo).max()
    err = np.abs(V - Vo).max() / np.abs(Vo).max()
    assert err <= max(1e-10, 10 * spread), (err, spread)
    Eo = oracle.integrate_cube(go, rho * Vo)
    assert abs(E - Eo) <= 1e-11 * abs(Eo)


@pytest.mark.parametrize("ncell,lmax,maxlevel", [(16, 8, 2), (16, 8, 3), (18, 6, 3)])
def test_adaptive_matches_oracle(dage, oracle, ncell, lmax, maxlevel):
    """The adaptive mode (multipoles up to level 1, whole parent-level boxes
    in the far field) against the oracle's restatement: moments, local
    expansions, potential and energy."""
    g, go, rho = _setup(dage, oracle, ncell, 0.2)
    quad = (6, 6, 0.0, 2.0, 1e3)
    op = dage.GBFMMCoulomb3D(g, lmax=lmax, maxlevel=maxlevel, quad=dage.GaussQuad(*quad),
                             adaptive_mode=True)
    V, E = op.apply(rho, energy=True)
    Vo, qo, Lo, _ = oracle.gbfmm_apply(go, rho, lmax=lmax, maxlevel=maxlevel, quad=quad,
                                       return_parts=True, adaptive=True)
    Qg = op.multipole_moments(rho)
    assert np.abs(Qg - qo).max() <= 1e-12 * np.abs(qo).max()
    op.apply(rho)
    Lg = op.local_expansions()
    assert np.abs(Lg - Lo).max() <= 1e-11 * np.abs(Lo).max()
    V1 = oracle.gbfmm_apply(go, rho, lmax=lmax, maxlevel=maxlevel, quad=quad, libm_1ulp=True,
                            adaptive=True)
    spread = np.abs(V1 - Vo).max() / np.abs(Vo).max()
    err = np.abs(V - Vo).max() / np.abs(Vo).max()
    assert err <= max(1e-10, 10 * spread), (err, spread)
    Eo = oracle.integrate_cube(go, rho * Vo)
    assert abs(E - Eo) <= 1e-11 * abs(Eo)

