"""CPU tests of the oracle's restatement of the Taylor-series contaminant
bubbles (Bubbles_get_contaminants bubbles.F90:2844-2910,
Function3D_get_cube_contaminants function3d.F90:1570-1624, Bubbles_make_taylor
bubbles.F90:1435-1530, Cart2SphIter harmonic.F90:1096-1265), pinned by
mathematics the reference's own tests do not cover: the harmonic expansion
of monomials, derivatives of exactly interpolated polynomials, finite
differences of the bubbles, and the exact series reproducing x^kappa/kappa!;
and the host-only table of the library against the oracle's."""
import math

import numpy as np
import pytest


def test_cart_iter_order(oracle):
    # the order documented for CartIter/CartShellIter (cartiter.F90:114-146)
    assert oracle.cart_iter(2) == [(0, 0, 0), (0, 0, 1), (0, 0, 2), (0, 1, 0), (0, 1, 1), (0, 2, 0),
                                   (1, 0, 0), (1, 0, 1), (1, 1, 0), (2, 0, 0)]
    assert len(oracle.cart_iter(3)) == 20


def test_dvpos_offset(oracle):
    """dvpos's shell offset |dv|^2 is the true one up to |dv| = 2 and one
    short for the third shell."""
    for K in range(4):
        for dv in [k for k in oracle.cart_iter(K) if sum(k) == K]:
            true = K * (K + 1) * (K + 2) // 6 + oracle.dvpos_shell(dv)
            assert oracle.dvpos(dv) == (true if K <= 2 else true - 1)


def test_cart_to_sph_reproduces_monomials(oracle):
    """x^kappa = r^|kappa| sum_lm C Y_lm(x/r) at random points."""
    C = oracle.cart_to_sph(3)
    rng = np.random.default_rng(0)
    for p in rng.standard_normal((5, 3)):
        r = np.linalg.norm(p)
        Y = oracle.solid_harmonics(3, p / r)
        for kappa in oracle.cart_iter(3):
            K = sum(kappa)
            col = K * (K + 1) * (K + 2) // 6 + oracle.dvpos_shell(kappa) - 1
            lhs = p[0] ** kappa[0] * p[1] ** kappa[1] * p[2] ** kappa[2]
            assert abs(r ** K * (C[:, col] @ Y) - lhs) <= 1e-13


@pytest.mark.parametrize("exact", [False, True])
def test_library_table_matches_oracle(dage_host, oracle, exact):
    """dage_cart2sph_table (host only) against the oracle's Cart2SphIter."""
    C = oracle.cart_to_sph(3)
    kap = oracle.cart_iter(3)
    got = np.zeros((16, 20))
    for i, lm, c in dage_host.cart2sph_table(3, exact=exact):
        got[lm, i] += c
    for i, kappa in enumerate(kap):
        K = sum(kappa)
        col = (K * (K + 1) * (K + 2) // 6 + oracle.dvpos_shell(kappa) - 1) if exact \
            else oracle.dvpos(kappa) - 1
        assert np.abs(got[:, i] - C[:, col]).max() <= 1e-14


def _poly(p):
    x, y, z = p
    return 0.3 * x ** 2 * y - 1.1 * z ** 3 + x * y * z + 0.5 * y ** 2 - 2.0 * x + 0.7


def _poly_derivative(kappa, p):
    """d^kappa of _poly, differentiated symbolically."""
    import sympy as sp
    x, y, z = sp.symbols("x y z")
    e = 0.3 * x ** 2 * y - 1.1 * z ** 3 + x * y * z + 0.5 * y ** 2 - 2.0 * x + 0.7
    d = sp.diff(e, x, kappa[0], y, kappa[1], z, kappa[2])
    return float(d.subs({x: p[0], y: p[1], z: p[2]}))


def test_cube_contaminants_of_polynomial(oracle):
    """A polynomial of degree <= 6 per axis is interpolated exactly, so the
    cube contaminants are its derivatives; a centre outside gives 0."""
    go = oracle.Grid3D.cube(-2.0, 5, 0.15)
    ax = go.axes[0].points
    X, Y, Z = np.meshgrid(ax, ax, ax, indexing="ij")
    cube = np.asfortranarray(_poly((X, Y, Z)))
    cen = np.array([[0.11, -0.37, 0.52], [-1.0, 0.7, 0.2], [5.0, 0.0, 0.0]])
    got = oracle.cube_contaminants(go, cube, cen, 3)
    for B in range(2):
        for i, kappa in enumerate(oracle.cart_iter(3)):
            assert abs(got[B, i] - _poly_derivative(kappa, cen[B])) <= 1e-10
    assert np.all(got[2] == 0.0)


def _set(oracle, lmax, seed, natom=3, k=0):
    rng = np.random.default_rng(seed)
    centers = np.array([[0.1, -0.3, 0.2], [1.4, 0.9, -1.1], [-1.2, 1.0, 0.8]])[:natom]
    h = oracle.log_radial_grid(33, 1e-5, 15.0)
    g = oracle.Grid1D(0.0, 33, 7, 1, h)
    r = g.points
    f = []
    for _ in range(natom):
        fa = np.zeros(((lmax + 1) ** 2, len(r)))
        for l in range(lmax + 1):
            for m in range(-l, l + 1):
                fa[l * (l + 1) + m] = rng.uniform(-1, 1) * r ** l * np.exp(-rng.uniform(0.5, 2) * r)
        f.append(fa)
    return centers, g, h, f


def _stencil(oracle, centre, delta):
    """One 7-point LIP cell per axis centred on `centre`."""
    axes = tuple(oracle.Grid1D.equidistant(c - 3 * delta, 1, delta) for c in centre)
    return oracle.Grid3D(axes)


@pytest.mark.parametrize("lmax,k", [(2, 0), (1, 1)])
def test_bubble_contaminants_against_differences(oracle, lmax, k):
    """Contaminants at each atom against the derivatives of a degree-6 fit
    (the cube interpolant of a 7-point stencil) of the other atoms' bubbles."""
    centers, g, h, f = _set(oracle, lmax, 3)
    got = oracle.bubble_contaminants(centers, [g] * 3, lmax, f, k, 3)
    delta = 2e-3
    for B in range(3):
        others = [A for A in range(3) if A != B]
        st = _stencil(oracle, centers[B], delta)
        cube = oracle.bubbles_inject(centers[others], [33] * 2, [h] * 2, lmax,
                                     [f[A] for A in others], st, k=k)
        ref = oracle.cube_contaminants(st, cube, centers[B:B + 1], 3)[0]
        scale = np.abs(ref).max()
        for i, kappa in enumerate(oracle.cart_iter(3)):
            tol = (1e-9, 1e-7, 1e-5, 1e-3)[sum(kappa)] * scale
            assert abs(got[B, i] - ref[i]) <= tol, (B, kappa, got[B, i], ref[i])


def test_exact_taylor_reproduces_series(oracle):
    """With the exact conventions the Taylor bubble of an atom, injected near
    its centre (w = 1 there, r^|kappa| interpolated exactly), is
    sum_kappa c_kappa x^kappa / kappa!."""
    centers, g, h, _ = _set(oracle, 2, 4, natom=1)
    c = np.random.default_rng(9).standard_normal((1, 20))
    ft = oracle.make_taylor([g], 2, 0, c, None, 3, exact=True)
    st = _stencil(oracle, centers[0], 0.05)
    cube = oracle.bubbles_inject(centers, [33], [h], 3, ft, st)
    ax = [a.points - centers[0][d] for d, a in enumerate(st.axes)]
    X, Y, Z = np.meshgrid(*ax, indexing="ij")
    ref = np.zeros_like(X)
    for i, (a, b, cc) in enumerate(oracle.cart_iter(3)):
        ref += c[0, i] * X ** a * Y ** b * Z ** cc / (math.factorial(a) * math.factorial(b) *
                                                      math.factorial(cc))
    assert np.abs(cube - ref).max() <= 1e-12 * np.abs(ref).max()


def test_reference_taylor_conventions(oracle):
    """The reference conventions against the exact ones: the |kappa|! factor
    halves the mixed second-order terms, and up to order 2 the harmonic
    columns agree."""
    centers, g, h, _ = _set(oracle, 2, 4, natom=1)
    for i, kappa in enumerate(oracle.cart_iter(2)):
        c = np.zeros((1, 10))
        c[0, i] = 1.0
        ref = oracle.make_taylor([g], 2, 0, c, None, 2)[0]
        ex = oracle.make_taylor([g], 2, 0, c, None, 2, exact=True)[0]
        ratio = math.factorial(kappa[0]) * math.factorial(kappa[1]) * math.factorial(kappa[2]) / \
            math.factorial(sum(kappa))
        assert np.abs(ref - ratio * ex).max() <= 1e-15 * max(np.abs(ex).max(), 1e-300)
