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
