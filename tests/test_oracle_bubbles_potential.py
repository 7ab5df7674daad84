"""The oracle's bubble radial Coulomb potential (coulomb.F90:222-336) against
closed forms: a Gaussian monopole and a Gaussian dipole shell."""
import numpy as np
from scipy.special import erf


def test_gaussian_monopole(oracle):
    h = oracle.log_radial_grid(60, 1e-4, 12.0)
    r = oracle.Grid1D(0.0, 60, 7, 1, h).points
    f = np.exp(-r ** 2)[None, :]
    V = oracle.bubbles_coulomb_potential(60, h, 0, f)[0]
    exact = np.pi ** 1.5 * np.where(r > 0, erf(r) / np.where(r > 0, r, 1), 2 / np.sqrt(np.pi))
    sel = r > 1e-3  # r^-1 times a vanishing integral at the origin
    assert np.abs(V[sel] - exact[sel]).max() <= 1e-8 * np.abs(exact).max()


def test_gaussian_dipole(oracle):
    """rho = r e^{-r^2} Y_10: V(r) = 4 pi/3 [r^-2 int_0^r s^4 e^{-s^2} ds
    + r int_r^inf s e^{-s^2} ds] (k = 0, l = 1), in closed form."""
    h = oracle.log_radial_grid(60, 1e-4, 12.0)
    r = oracle.Grid1D(0.0, 60, 7, 1, h).points
    f = np.zeros((4, r.size))
    f[2] = r * np.exp(-r ** 2)
    V = oracle.bubbles_coulomb_potential(60, h, 1, f)
    rr = r[r > 1e-2]
    inner = 3 * np.sqrt(np.pi) / 8 * erf(rr) - np.exp(-rr ** 2) * (rr ** 3 / 2 + 3 * rr / 4)
    outer = np.exp(-rr ** 2) / 2
    exact = 4 * np.pi / 3 * (inner / rr ** 2 + rr * outer)
    assert np.abs(V[2][r > 1e-2] - exact).max() <= 5e-8 * np.abs(exact).max()  # LIP quadrature
    assert np.abs(V[[0, 1, 3]]).max() == 0.0
