"""GPU tests of the GBFMM Helmholtz operator (kernel e^(-kappa r)/r) against
the oracle: Bessel multipoles, the Helmholtz multipole-to-local converter,
the full potential and energy, and against the direct Helmholtz cube
operator within the multipole truncation error."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(dage, oracle, ncell, step=0.2, ng=6, seed=3):
    half = 0.5 * ncell * 6 * step
    g = dage.Grid3D.cube(-half, ncell, step)
    go = oracle.Grid3D.cube(-half, ncell, step)
    rng = np.random.default_rng(seed)
    q = rng.uniform(-1, 2, ng)
    a = rng.uniform(0.8, 6, ng)
    c = rng.uniform(-0.7 * half, 0.7 * half, (ng, 3))
    return g, go, oracle.gauss_cube(go, q, a, c)


# 15 cells: uneven split (box point counts not a multiple of the moment
# kernel's chunk of z values, 32 / (32 // (lmax + 1))); lmax 0 has no
# lmax - 1 series, lmax 1 no downward recursion
@pytest.mark.parametrize("ncell,energy,lmax", [(16, -0.5, 8), (15, -1.2, 8), (15, -0.7, 0),
                                               (15, -0.9, 1), (15, -1.5, 15)])
def test_helmholtz_moments_and_local_expansions(dage, oracle, ncell, energy, lmax):
    kappa = np.sqrt(-2 * energy)
    g, go, rho = _setup(dage, oracle, ncell)
    op = dage.GBFMMHelmholtz3D(g, energy, lmax=lmax, quad=dage.GaussQuad(6, 6))
    Qg = op.multipole_moments(rho)
    plan = oracle.GBFMMPlan(go, 2)
    Qo = np.zeros_like(Qg)
    for b in range(1, plan.nbox + 1):
        (x0, x1), (y0, y1), (z0, z1) = plan.points(b)
        subs = [oracle.subgrid(a, c0, c1) for a, (c0, c1) in zip(go.axes, plan.cells(b))]
        Qo[:, b - 1] = oracle.helm_box_multipoles(lmax, kappa, subs[0].points, subs[0].weights(),
                                                  subs[1].points, subs[1].weights(),
                                                  subs[2].points, subs[2].weights(),
                                                  rho[x0:x1, y0:y1, z0:z1], plan.center(b))
    assert np.abs(Qg - Qo).max() <= 1e-12 * np.abs(Qo).max()
    op.apply(rho)
    Lg = op.local_expansions()
    Lo = np.zeros_like(Lg)
    for i in range(1, plan.nbox + 1):
        for j in oracle.local_farfield(i, 2):
            Lo[:, i - 1] += oracle.helm_m2l(lmax, kappa, Qo[:, j - 1], plan.center(j),
                                            plan.center(i))
    assert np.abs(Lg - Lo).max() <= 1e-11 * np.abs(Lo).max()


def test_helmholtz_apply_matches_oracle(dage, oracle):
    g, go, rho = _setup(dage, oracle, 16)
    quad, lmax, energy = (8, 8, 0.0, 2.0, 1e3), 8, -0.5
    op = dage.GBFMMHelmholtz3D(g, energy, lmax=lmax, quad=dage.GaussQuad(*quad))
    V, E = op.apply(rho, energy=True)
    Vo = oracle.gbfmm_apply(go, rho, lmax=lmax, quad=quad, energy=energy)
    V1 = oracle.gbfmm_apply(go, rho, lmax=lmax, quad=quad, energy=energy, libm_1ulp=True)
    spread = np.abs(V1 - Vo).max() / np.abs(Vo).max()
    err = np.abs(V - Vo).max() / np.abs(Vo).max()
    assert err <= max(1e-10, 10 * spread), (err, spread)
    Eo = oracle.integrate_cube(go, rho * Vo)
    assert abs(E - Eo) <= 1e-11 * abs(Eo)


def test_helmholtz_close_to_direct_operator_and_back_to_coulomb(dage, oracle):
    g, go, rho = _setup(dage, oracle, 20, ng=8)
    quad = dage.GaussQuad(12, 12)
    op = dage.GBFMMHelmholtz3D(g, -0.8, lmax=12, quad=quad)
    V, E = op.apply(rho, energy=True)
    direct = dage.Helmholtz3D(dage.Coulomb3D(g, quad=quad), -0.8)
    Vd, Ed = direct.apply(rho, energy=True, coda=False)
    assert np.abs(V - Vd).max() / np.abs(Vd).max() < 5e-3
    assert abs(E - Ed) / abs(Ed) < 1e-3
    op.set_energy(0.0)  # the Coulomb operator again
    Vc = op.apply(rho)
    V0 = dage.GBFMMCoulomb3D(g, lmax=12, quad=quad).apply(rho)
    assert np.abs(Vc - V0).max() <= 1e-14 * np.abs(V0).max()


@pytest.mark.parametrize("lmax,energy", [(0, -0.3), (1, -0.5), (8, -2.0), (15, -0.8)])
def test_helmholtz_l2p_matches_oracle(dage, oracle, lmax, energy):
    """Far field of given local expansions (the L2P alone) against the oracle."""
    kappa = np.sqrt(-2 * energy)
    g, go, rho = _setup(dage, oracle, 8)
    op = dage.GBFMMHelmholtz3D(g, energy, lmax=lmax, quad=dage.GaussQuad(4, 4))
    plan = oracle.GBFMMPlan(go, 2)
    L = np.random.default_rng(lmax).standard_normal(((lmax + 1) ** 2, plan.nbox))
    V = np.zeros(go.shape, order="F")
    op.evaluate_local_expansions(L, V)
    Vo = np.zeros(go.shape, order="F")
    for b in range(1, plan.nbox + 1):
        own = plan.owned(b)
        outs = [go.axes[d].points[own[d][0]:own[d][1]] for d in range(3)]
        far = np.zeros(tuple(len(o) for o in outs), order="F")
        oracle.helm_l2p(lmax, kappa, L[:, b - 1], plan.center(b), outs[0], outs[1], outs[2], far)
        Vo[tuple(slice(o0, o1) for o0, o1 in own)] = far
    assert np.abs(V - Vo).max() <= 1e-12 * np.abs(Vo).max()


@pytest.mark.parametrize("lmax,energy", [(8, -0.18), (12, -0.5), (15, -1.2)])
def test_helmholtz_l2p_plane_wave_identity(dage, oracle, lmax, energy):
    """The plane-wave expansion sum_l (2l+1) i_l(kappa r) P_l(cos theta) =
    e^(kappa z) (the identity behind tests/multipole_translation_test.F90
    first_bessel_test): with L_l0 = 4 pi / (8 kappa) and every other
    coefficient zero, the GPU's L2P is e^(kappa (z - c_z)) at every point of
    every box, up to the truncation at lmax (bounded with the oracle's i_l)."""
    kappa = np.sqrt(-2 * energy)
    g, go, rho = _setup(dage, oracle, 8)
    op = dage.GBFMMHelmholtz3D(g, energy, lmax=lmax, quad=dage.GaussQuad(4, 4))
    plan = oracle.GBFMMPlan(go, 2)
    L = np.zeros(((lmax + 1) ** 2, plan.nbox))
    for l in range(lmax + 1):
        L[l * (l + 1), :] = 4 * np.pi / (8 * kappa)
    V = np.zeros(go.shape, order="F")
    op.evaluate_local_expansions(L, V)
    Vx = np.zeros(go.shape, order="F")
    rmax = 0.0
    for b in range(1, plan.nbox + 1):
        own = plan.owned(b)
        c = plan.center(b)
        pts = [go.axes[d].points[own[d][0]:own[d][1]] - c[d] for d in range(3)]
        Vx[tuple(slice(o0, o1) for o0, o1 in own)] = np.exp(kappa * pts[2])[None, None, :]
        rmax = max(rmax, np.sqrt(sum(np.abs(p).max() ** 2 for p in pts)))
    lt = np.arange(lmax + 1, lmax + 30)
    tail = ((2 * lt + 1) * oracle.bessel_i(kappa * rmax, lmax + 29)[lmax + 1:]).sum()
    err = np.abs(V - Vx).max()
    assert err <= 2 * tail + 1e-13 * np.abs(Vx).max(), (err, tail)


# maxlevel 3 (8^3 boxes of 2 cells): the Helmholtz M2M of the reference's
# translator, M2L at levels 2 and 3 (adaptive: level-1 moments and whole
# parent-level sources) and the L2L the M2M implies; against the oracle's
# restatement (rotations by the reference's recursion, the product's by least
# squares)
@pytest.mark.parametrize("adaptive", [False, True])
def test_helmholtz_multilevel_matches_oracle(dage, oracle, adaptive):
    g, go, rho = _setup(dage, oracle, 16)
    quad, lmax, energy = (6, 6, 0.0, 2.0, 1e3), 6, -0.5
    op = dage.GBFMMHelmholtz3D(g, energy, lmax=lmax, maxlevel=3, quad=dage.GaussQuad(*quad),
                               adaptive_mode=adaptive)
    V, E = op.apply(rho, energy=True)
    Lg = op.local_expansions()
    Vo, _, Lo, Vn = oracle.gbfmm_apply(go, rho, lmax=lmax, maxlevel=3, quad=quad, energy=energy,
                                       adaptive=adaptive, return_parts=True)
    Vn1 = oracle.gbfmm_near_field(go, rho, 3, quad, libm_1ulp=True, energy=energy)
    scale = np.abs(Vo).max()
    spread = np.abs(Vn1 - Vn).max() / scale
    err = np.abs(V - Vo).max() / scale
    print(f"adaptive={adaptive}: L {np.abs(Lg - Lo).max() / np.abs(Lo).max():.2e}, "
          f"V {err:.2e} (spread {spread:.2e})")
    assert np.abs(Lg - Lo).max() <= 1e-11 * np.abs(Lo).max()
    assert err <= max(1e-10, 10 * spread), (err, spread)
    Eo = oracle.integrate_cube(go, rho * Vo)
    assert abs(E - Eo) <= 1e-11 * abs(Eo), (E, Eo)
    # and against the direct Helmholtz operator: the far field uses the exact
    # kernel, the direct operator this 12-point quadrature's approximation of
    # it, so the bar is the quadrature's (as for maxlevel 2 above)
    direct = dage.Helmholtz3D(dage.Coulomb3D(g, quad=dage.GaussQuad(*quad)), energy)
    Vd, _ = direct.apply(rho, energy=True, coda=False)
    assert np.abs(V - Vd).max() <= 5e-3 * np.abs(Vd).max()
