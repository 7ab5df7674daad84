"""GPU tests of the fused all-atoms bubbles -> cube injection against the
oracle's restatement of Bubbles_eval_pick (bubbles.F90:1904-1975)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bubbles(oracle, natom, lmax, seed=5, box=15.0, ncell=33):
    rng = np.random.default_rng(seed)
    centers = rng.uniform(-box / 2, box / 2, (natom, 3))
    h = oracle.log_radial_grid(ncell, 1e-5, 15.0)
    r = oracle.Grid1D(0.0, ncell, 7, 1, h).points
    f = []
    for _ in range(natom):
        fa = np.zeros(((lmax + 1) ** 2, len(r)))
        for l in range(lmax + 1):
            for m in range(-l, l + 1):
                fa[l * (l + 1) + m] = rng.uniform(-1, 1) * r ** l * np.exp(-rng.uniform(0.5, 3) * r)
        f.append(fa)
    return centers, [ncell] * natom, [h] * natom, f


@pytest.mark.parametrize("natom,lmax,lmin,k", [(1, 0, 0, 0), (3, 2, 0, 0), (4, 2, 1, 0),
                                               (2, 4, 0, 1), (20, 2, 0, 0)])
def test_inject_matches_oracle(dage, oracle, natom, lmax, lmin, k):
    centers, ncells, hs, f = _bubbles(oracle, natom, lmax)
    g = dage.Grid3D.cube(-9.0, 15, 0.2)
    go = oracle.Grid3D.cube(-9.0, 15, 0.2)
    rad = [dage.Grid1D(0.0, n, 7, 1, h) for n, h in zip(ncells, hs)]
    b = dage.Bubbles(centers, rad, f, lmax, k=k)
    base = np.asfortranarray(np.random.default_rng(1).standard_normal(go.shape))
    cube = b.inject(g, cube=base.copy(order="F"), lmin=lmin, factor=0.7)
    ref = oracle.bubbles_inject(centers, ncells, hs, lmax, f, go, lmin=lmin, k=k, factor=0.7,
                                cube=base.copy(order="F"))
    assert np.abs(cube - ref).max() <= 1e-12 * np.abs(ref - base).max()


def test_inject_device_cube_and_analytic(dage, oracle):
    import torch

    h = oracle.log_radial_grid()
    r = oracle.Grid1D(0.0, 33, 7, 1, h).points
    f = [np.exp(-r)[None, :]]
    g = dage.Grid3D.cube(-6.0, 10, 0.2)
    go = oracle.Grid3D.cube(-6.0, 10, 0.2)
    b = dage.Bubbles([[0.13, -0.21, 0.07]], [dage.Grid1D(0.0, 33, 7, 1, h)], f, 0)
    cube = torch.zeros(go.shape[::-1], dtype=torch.float64, device="cuda")
    b.inject(g, cube=cube)
    X, Y, Z = np.meshgrid(*(a.points for a in go.axes), indexing="ij")
    exact = np.exp(-np.sqrt((X - 0.13) ** 2 + (Y + 0.21) ** 2 + (Z - 0.07) ** 2))
    got = cube.cpu().numpy().reshape(-1).reshape(go.shape, order="F")
    assert np.abs(got - exact).max() < 1e-6  # LIP interpolation error on the log grid


@pytest.mark.parametrize("natom,lmax,k", [(1, 0, 0), (3, 2, 0), (2, 4, 1)])
def test_coulomb_potential_matches_oracle(dage, oracle, natom, lmax, k):
    """Radial Coulomb potential of every (atom, lm) function on the GPU against
    the oracle's restatement of Coulomb3D_evaluate_bubbles_potential."""
    centers, ncells, hs, f = _bubbles(oracle, natom, lmax)
    rad = [dage.Grid1D(0.0, n, 7, 1, h) for n, h in zip(ncells, hs)]
    b = dage.Bubbles(centers, rad, f, lmax, k=k)
    pot = b.coulomb_potential()
    got = pot.radial_values()
    for a in range(natom):
        ref = oracle.bubbles_coulomb_potential(ncells[a], hs[a], lmax, f[a], k=k)
        assert np.abs(got[a] - ref).max() <= 1e-12 * np.abs(ref).max()


def test_coulomb_potential_of_gaussian_injects_erf(dage, oracle):
    """A Gaussian monopole bubble -> potential bubble -> injected into a cube:
    pi^{3/2} erf(r)/r within the LIP interpolation error."""
    from scipy.special import erf

    h = oracle.log_radial_grid(60, 1e-4, 12.0)
    r = oracle.Grid1D(0.0, 60, 7, 1, h).points
    b = dage.Bubbles([[0.1, -0.2, 0.05]], [dage.Grid1D(0.0, 60, 7, 1, h)], [np.exp(-r ** 2)[None, :]], 0)
    pot = b.coulomb_potential()
    g = dage.Grid3D.cube(-4.0, 10, 0.2)
    go = oracle.Grid3D.cube(-4.0, 10, 0.2)
    cube = pot.inject(g)
    X, Y, Z = np.meshgrid(*(a.points for a in go.axes), indexing="ij")
    d = np.sqrt((X - 0.1) ** 2 + (Y + 0.2) ** 2 + (Z - 0.05) ** 2)
    exact = np.pi ** 1.5 * erf(d) / d
    inside = d < 11.5  # the radial grid (and so the bubble) ends at r = 12
    assert np.abs(cube - exact)[inside].max() <= 1e-6 * np.abs(exact).max()


@pytest.mark.parametrize("natom,lmax,k,energy", [(1, 0, 0, -0.125), (3, 2, 0, -0.5), (2, 4, 1, -2.0),
                                                 (1, 8, 0, -0.8)])
def test_helmholtz_potential_matches_oracle(dage, oracle, natom, lmax, k, energy):
    """Radial Helmholtz potential of every (atom, lm) function on the GPU
    against the oracle's restatement of Helmholtz3D_transform_bubbles_sub."""
    centers, ncells, hs, f = _bubbles(oracle, natom, lmax)
    rad = [dage.Grid1D(0.0, n, 7, 1, h) for n, h in zip(ncells, hs)]
    V = dage.Bubbles(centers, rad, f, lmax, k=k).helmholtz_potential(energy).radial_values()
    kappa = np.sqrt(-2 * energy)
    for a in range(natom):
        ref = oracle.bubbles_helmholtz_potential(ncells[a], hs[a], lmax, f[a], kappa, k=k)
        assert np.abs(V[a] - ref).max() <= 1e-12 * np.abs(ref).max()


def test_helmholtz_potential_of_gaussian(dage, oracle):
    """rho = e^-r^2 -> pi^1.5/(2r) e^(k^2/4) [e^-kr erfc(k/2 - r) - e^kr erfc(k/2 + r)]."""
    from scipy.special import erfc

    h = oracle.log_radial_grid(60, 1e-4, 12.0)
    r = oracle.Grid1D(0.0, 60, 7, 1, h).points
    kappa = 1.3
    b = dage.Bubbles([[0.0, 0.0, 0.0]], [dage.Grid1D(0.0, 60, 7, 1, h)], [np.exp(-r ** 2)[None, :]], 0)
    V = b.helmholtz_potential(-0.5 * kappa ** 2).radial_values()[0][0]
    rr = r[1:]
    exact = (np.pi ** 1.5 / (2 * rr) * np.exp(kappa ** 2 / 4)
             * (np.exp(-kappa * rr) * erfc(kappa / 2 - rr) - np.exp(kappa * rr) * erfc(kappa / 2 + rr)))
    sel = rr < 8.0
    assert np.abs(V[1:][sel] - exact[sel]).max() < 2e-8 * np.abs(exact).max()


def test_helmholtz_potential_needs_negative_energy(dage, oracle):
    h = oracle.log_radial_grid()
    r = oracle.Grid1D(0.0, 33, 7, 1, h).points
    b = dage.Bubbles([[0.0, 0.0, 0.0]], [dage.Grid1D(0.0, 33, 7, 1, h)], [np.exp(-r)[None, :]], 0)
    with pytest.raises(dage.DageError):
        b.helmholtz_potential(0.0)


def test_operate_on_cube_and_bubbles(dage, oracle):
    """operate_on: the cube operator on the cube part and the radial
    potential of the bubbles (Coulomb and Helmholtz)."""
    centers, ncells, hs, f = _bubbles(oracle, 2, 2)
    rad = [dage.Grid1D(0.0, n, 7, 1, h) for n, h in zip(ncells, hs)]
    b = dage.Bubbles(centers, rad, f, 2)
    g = dage.Grid3D.cube(-2.4, 4, 0.2)
    cube = np.asfortranarray(np.random.default_rng(2).standard_normal(tuple(a.n for a in g.axes)))
    op = dage.Coulomb3D(g, quad=dage.GaussQuad(4, 4))
    V, Vb = op.operate_on(cube, b)
    assert np.array_equal(V, op.apply(cube))
    for a in range(2):
        ref = oracle.bubbles_coulomb_potential(ncells[a], hs[a], 2, f[a])
        assert np.abs(Vb.radial_values()[a] - ref).max() <= 1e-12 * np.abs(ref).max()
    hop = dage.Helmholtz3D(op, -0.5)
    V2, Vb2 = hop.operate_on(cube, b)
    assert np.array_equal(V2, hop.apply(cube))
    ref = oracle.bubbles_helmholtz_potential(ncells[0], hs[0], 2, f[0], 1.0)
    assert np.abs(Vb2.radial_values()[0] - ref).max() <= 1e-12 * np.abs(ref).max()
