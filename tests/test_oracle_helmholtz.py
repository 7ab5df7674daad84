"""CPU checks of the oracle's Helmholtz (Yukawa) far field: the modified
spherical Bessel functions against closed forms and their Wronskian, and the
multipole -> M2L -> L2P chain against the exact e^(-kappa R)/R of point
charges (it converges with lmax, which pins the rotation direction, the
coaxial recurrence and the normalisations of the reference's converter)."""
import numpy as np
import pytest


def test_bessel_closed_forms(oracle):
    for x in (1e-3, 0.3, 1.0, 4.0, 13.0):
        i = oracle.bessel_i(x, 12)
        k = oracle.bessel_k(x, 12)
        assert abs(i[0] - np.sinh(x) / x) <= 1e-14 * abs(i[0])
        if x >= 0.3:  # the closed form cancels for small x; the series does not
            assert abs(i[1] - (x * np.cosh(x) - np.sinh(x)) / x ** 2) <= 1e-12 * abs(i[1])
        assert abs(k[0] - 0.5 * np.pi * np.exp(-x) / x) <= 1e-15 * k[0]
        # Wronskian: i_l k_{l+1} + i_{l+1} k_l = pi / (2 x^2)
        for l in range(11):
            w = i[l] * k[l + 1] + i[l + 1] * k[l]
            assert abs(w - np.pi / (2 * x * x)) <= 1e-12 * np.pi / (2 * x * x)


@pytest.mark.parametrize("kappa", [0.5, 1.0, 2.0])
def test_far_field_converges_to_yukawa(oracle, kappa):
    ci, cj = np.array([6.0, 2.0, -3.0]), np.zeros(3)
    rng = np.random.default_rng(1)
    pts = [(cj + rng.uniform(-1, 1, 3), ci + rng.uniform(-1, 1, 3)) for _ in range(4)]
    prev = None
    for lmax in (6, 10, 12):
        err = 0.0
        for s, r in pts:
            one = np.ones(1)
            M = oracle.helm_box_multipoles(lmax, kappa, s[:1], one, s[1:2], one, s[2:], one,
                                           np.ones((1, 1, 1)), cj)
            L = oracle.helm_m2l(lmax, kappa, M, cj, ci)
            V = np.zeros((1, 1, 1), order="F")
            oracle.helm_l2p(lmax, kappa, L, ci, r[:1], r[1:2], r[2:], V)
            R = np.linalg.norm(r - s)
            err = max(err, abs(V[0, 0, 0] - np.exp(-kappa * R) / R) / (np.exp(-kappa * R) / R))
        if prev is not None:
            assert err < prev
        prev = err
    assert prev < {0.5: 1e-7, 1.0: 1e-6, 2.0: 1e-5}[kappa]


def test_m2l_is_linear_and_zero_free(oracle):
    rng = np.random.default_rng(2)
    N = 49
    M1, M2 = rng.standard_normal(N), rng.standard_normal(N)
    a, b = np.array([0.1, -0.2, 0.3]), np.array([-3.0, 4.0, 2.5])
    L1 = oracle.helm_m2l(6, 1.3, M1, a, b)
    L2 = oracle.helm_m2l(6, 1.3, M2, a, b)
    L12 = oracle.helm_m2l(6, 1.3, 2 * M1 - M2, a, b)
    assert np.allclose(L12, 2 * L1 - L2, rtol=1e-12, atol=1e-14 * np.abs(L1).max())


def test_reference_bessel_identities(oracle):
    """The identities tests/multipole_translation_test.F90 evaluates
    (first_bessel_test :567-603, potential_test :519-565; the reference
    prints them): sum (2l+1) i_l(z) = e^z, sum (-1)^l (2l+1) i_l(z) = e^-z on
    its radial points r_i = 0.005 * 1.5^i (kappa = 1, arguments up to 8, where
    lmax 40 truncates below 1e-15), and the Yukawa addition theorem
    (2 kappa / pi) sum (2l+1) i_l(kappa r_i) k_l(kappa r_j) = e^(-kappa (r_j - r_i)) / (r_j - r_i)
    for collinear points with r_i <= r_j / 2 (lmax 50)."""
    r = 0.005 * 1.5 ** np.arange(25)
    for z in r[r <= 8.0]:
        i = oracle.bessel_i(z, 40)
        l = np.arange(41)
        assert abs(((2 * l + 1) * i).sum() - np.exp(z)) <= 2e-15 * np.exp(z)
        assert abs(((-1.0) ** l * (2 * l + 1) * i).sum() - np.exp(-z)) <= 1e-15 * np.exp(z)
    kappa = 1.0
    pts = np.linspace(0.0, 1.0, 21)[1:]
    l = np.arange(51)
    for ri in pts:
        for rj in pts[pts >= 2 * ri]:
            s = ((2 * l + 1) * oracle.bessel_i(kappa * ri, 50) * oracle.bessel_k(kappa * rj, 50)).sum()
            exact = np.exp(-kappa * (rj - ri)) / (rj - ri)
            assert abs(2 * kappa / np.pi * s - exact) <= 1e-13 * exact, (ri, rj)


def _lattice_dirs():
    import itertools

    return [v for v in itertools.product(range(-3, 4), repeat=3) if max(abs(x) for x in v) >= 2]


def _orth_err(oracle, d, lmax, repaired):
    d = np.asarray(d, float) / np.linalg.norm(d)
    B = oracle.ref_real_rotation(np.arctan2(d[1], d[0]), np.arccos(d[2]), 0.0, lmax, repaired)
    return max(np.abs(b @ b.T - np.eye(len(b))).max() for b in B)


def test_reference_rotation_recursion_defects(oracle):
    """Two defects of the reference's rotation of real expansions
    (helmholtz_multipole_tools.F90:911-1200), restated as written: its
    sqrt(2.0) is a single-precision literal, so every rotation is orthogonal
    only to ~3e-8; and its eq. 68 step divides by l cos(beta) - m', which is
    0/0 where l cos(beta) is an integer -- e.g. the level-2 box displacement
    (2, 1, 2), cos(beta) = 2/3 -- where the result is no rotation at all."""
    rng = np.random.default_rng(0)
    generic = max(_orth_err(oracle, rng.standard_normal(3), 12, False) for _ in range(10))
    assert 1e-9 < generic < 1e-7
    assert _orth_err(oracle, (2, 1, 2), 12, False) > 0.1
    bad = [v for v in _lattice_dirs() if _orth_err(oracle, v, 12, False) > 1e-6]
    assert len(bad) == 16  # of the 316 level-2 far-field displacement directions


@pytest.mark.parametrize("lmax", [0, 1, 3, 8, 12, 15])
def test_repaired_rotation_matches_least_squares(oracle, lmax):
    """The oracle's M2L rotates with the reference's recursion, the two
    defects repaired (double sqrt 2; the eq. 68 rows from the explicit Wigner
    sum).  That rotation is orthogonal on every lattice direction, and the
    conversion equals the one built with an independent least-squares
    rotation (the method the library uses) to rounding."""
    rng = np.random.default_rng(lmax)
    assert max(_orth_err(oracle, v, lmax, True) for v in _lattice_dirs()) < 1e-13
    N = (lmax + 1) ** 2
    worst = 0.0
    cases = [(rng.uniform(-1, 1, 3), rng.uniform(-6, 6, 3)) for _ in range(4)]
    cases += [(np.zeros(3), 2.4 * np.asarray(v, float)) for v in _lattice_dirs()[::7]]
    for src, d in cases:
        M = rng.standard_normal(N)
        a = oracle.helm_m2l(lmax, 1.1, M, src, src + d)
        b = oracle.helm_m2l(lmax, 1.1, M, src, src + d, least_squares=True)
        worst = max(worst, np.abs(a - b).max() / np.abs(b).max())
    assert worst < 1e-13, worst


def test_helmholtz_m2m_matches_direct_moments(oracle):
    """The restated HelmholtzMultipoleTranslator moves point-charge moments
    from a child centre to a parent centre as a direct evaluation about the
    parent does (up to the lmax truncation)."""
    lmax, kappa = 8, 0.7
    rng = np.random.default_rng(0)
    pts, qs = rng.uniform(-0.5, 0.5, (20, 3)), rng.uniform(-1, 1, 20)
    cc, cp = np.array([0.3, -0.2, 0.4]), np.zeros(3)

    def moments(center):
        out = np.zeros((lmax + 1) ** 2)
        for p, q in zip(pts, qs):
            out += oracle.helm_box_multipoles(lmax, kappa, [p[0] + cc[0]], [q], [p[1] + cc[1]],
                                              [1.0], [p[2] + cc[2]], [1.0], np.ones((1, 1, 1)),
                                              center)
        return out

    qc, qp = moments(cc), moments(cp)
    qt = oracle.helm_m2m(lmax, kappa, qc, cc, cp)
    assert np.abs(qt - qp).max() <= 1e-10 * np.abs(qp).max()
    W = oracle.helm_matrix("m2m", lmax, kappa, cc, cp)
    assert np.abs(W @ qc - qt).max() <= 1e-14 * np.abs(qt).max()


def test_helmholtz_l2l_preserves_potential(oracle):
    """helm_l2l re-expands a local expansion about a child centre: its L2P at
    points of the child box equals the parent expansion's."""
    lmax, kappa = 8, 0.7
    rng = np.random.default_rng(1)
    cp, cc = np.zeros(3), np.array([0.3, -0.2, 0.4])
    Lp = rng.normal(size=(lmax + 1) ** 2) * np.repeat(0.3 ** np.arange(lmax + 1),
                                                       2 * np.arange(lmax + 1) + 1)
    Lc = oracle.helm_l2l(lmax, kappa, Lp, cp, cc)
    xs, ys, zs = (c + np.linspace(-0.2, 0.2, 3) for c in cc)
    V1, V2 = np.zeros((3, 3, 3), order="F"), np.zeros((3, 3, 3), order="F")
    oracle.helm_l2p(lmax, kappa, Lp, cp, xs, ys, zs, V1)
    oracle.helm_l2p(lmax, kappa, Lc, cc, xs, ys, zs, V2)
    assert np.abs(V1 - V2).max() <= 1e-12 * np.abs(V1).max()
