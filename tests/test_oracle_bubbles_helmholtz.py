"""The oracle's restatement of the Helmholtz bubble potential
(helmholtz3d.F90:519-650) against the closed form for a Gaussian and its
kappa -> 0 limit (the Coulomb bubble potential)."""
import numpy as np
from scipy.special import erfc


def _grid(oracle, ncell=60, r1=12.0):
    h = oracle.log_radial_grid(ncell, 1e-4, r1)
    return h, oracle.Grid1D(0.0, ncell, 7, 1, h).points


def test_gaussian_yukawa_potential(oracle):
    """rho = e^-r^2: V(r) = pi^1.5/(2r) e^(k^2/4) [e^-kr erfc(k/2 - r) - e^kr erfc(k/2 + r)]."""
    h, r = _grid(oracle)
    for kappa in (0.5, 1.3):
        V = oracle.bubbles_helmholtz_potential(60, h, 0, np.exp(-r ** 2)[None, :], kappa)[0]
        rr = r[1:]
        exact = (np.pi ** 1.5 / (2 * rr) * np.exp(kappa ** 2 / 4)
                 * (np.exp(-kappa * rr) * erfc(kappa / 2 - rr)
                    - np.exp(kappa * rr) * erfc(kappa / 2 + rr)))
        sel = rr < 8.0
        assert np.abs(V[1:][sel] - exact[sel]).max() < 2e-8 * np.abs(exact).max()  # 4.8e-9 seen
        # r = 0: pi^1.5 e^(k^2/4) (2/sqrt(pi) e^(-k^2/4) - k erfc(k/2))
        v0 = np.pi ** 1.5 * np.exp(kappa ** 2 / 4) * (2 / np.sqrt(np.pi) * np.exp(-kappa ** 2 / 4)
                                                    - kappa * erfc(kappa / 2))
        assert abs(V[0] - v0) < 1e-8 * v0


def test_small_kappa_tends_to_coulomb(oracle):
    h, r = _grid(oracle, 40, 10.0)
    lmax = 2
    rng = np.random.default_rng(4)
    f = np.array([rng.uniform(-1, 1) * r ** l * np.exp(-rng.uniform(1, 2) * r ** 2)
                  for l in range(lmax + 1) for _ in range(2 * l + 1)])
    Vc = oracle.bubbles_coulomb_potential(40, h, lmax, f)
    Vh = oracle.bubbles_helmholtz_potential(40, h, lmax, f, 1e-6)
    # e^(-k d)/d = 1/d - k + O(k^2): the difference is O(kappa) (r = 0 left out:
    # the l = 0 inward integrand's value there is extrapolated in the Helmholtz form)
    assert np.abs(Vh[:, 1:] - Vc[:, 1:]).max() < 5e-6 * np.abs(Vc).max()
