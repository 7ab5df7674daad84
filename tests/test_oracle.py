"""CPU tests of the oracle: pinned against the reference's known answers
(DAGE tests/gauss_test.F90) and checked for internal consistency."""
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _kat():
    with open(os.path.join(GOLD, "gauss_test_kat.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("case", _kat()["cases"], ids=lambda c: c["name"])
def test_gauss_test_selfint_kat(oracle, case):
    kat = _kat()
    qd = kat["quadrature"]
    g = oracle.Grid3D.gauss_default(case["q"], case["alpha"], case["centers"], step=case["step"],
                                    nlip=case["nlip"], thres=case["thres"],
                                    grid_type=kat["grid_type"])
    rho = oracle.gauss_cube(g, case["q"], case["alpha"], case["centers"])
    s = oracle.selfint(g, rho, quad=(qd["nlin"], qd["nlog"], qd["tstart"], qd["tlin"], qd["tlog"]),
                       coda=kat["coda"])
    # the reference asserts |value - golden| < TOL = 1e-14 (gauss_test.F90:57)
    assert abs(s - case["selfint"]) < kat["tolerance"]


@pytest.mark.parametrize("case", _kat()["cases"], ids=lambda c: c["name"])
def test_gauss_analytic_energy_kat(oracle, case):
    e = oracle.gauss_analytical_energy(case["q"], case["alpha"], case["centers"])
    assert abs(e - case["selfint_analytic"]) < 1e-14


def test_quadrature_properties(oracle):
    tp, tw = oracle.gauss_quad(10, 8, 0.0, 2.0, 1.0e3)
    assert np.all(np.diff(tp) > 0)
    assert abs(tw[:10].sum() - 2.0) < 1e-13          # Gauss rule integrates 1 on [0, 2]
    # log-mapped tail integrates dt exactly in log space: sum(w) ~ 998
    assert abs(tw[10:].sum() - 998.0) / 998.0 < 1e-6
    x, w = np.zeros(12), np.zeros(12)
    lib = oracle.lib()
    import ctypes
    lib.orc_gauleg(12, x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                   w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    xr, wr = np.polynomial.legendre.leggauss(12)
    np.testing.assert_allclose(x, xr, atol=1e-14)
    np.testing.assert_allclose(w, wr, atol=1e-14)


@pytest.mark.parametrize("nlip,gt", [(7, 1), (5, 1), (7, 2), (6, 2)])
def test_lip_basis_cardinal(oracle, nlip, gt):
    c, first, last = oracle.lip_coeffs(nlip, gt)
    if gt == 1:
        nodes = np.arange(nlip) - (nlip + 1) // 2 + 1
    else:
        nodes = None
    ints = oracle.lip_integrals(nlip, gt)
    assert abs(ints.sum() - (last - first)) < 1e-13
    if nodes is not None:
        vals = np.array([[np.polyval(c[j, :], x) for x in nodes] for j in range(nlip)])
        np.testing.assert_allclose(vals, np.eye(nlip), atol=1e-12)


def test_expo_integrals_vs_quadrature(oracle):
    """Closed forms (t >= 0.1) and the 12-point rule (t < 0.1) against a fine
    numerical integral of x^n exp(-t^2 (x-p)^2) over [-3, 3]."""
    xs, ws = np.polynomial.legendre.leggauss(200)
    x = 3.0 * xs
    w = 3.0 * ws
    for t in (0.05, 0.1, 0.3, 1.0, 2.5):
        for p in (-2.0, 0.0, 1.3, 4.0):
            v = oracle.expo_integrals(-3.0, 3.0, t, p, 7)
            ref = np.array([np.sum(w * x ** n * np.exp(-t * t * (x - p) ** 2)) for n in range(7)])
            scale = np.sum(w * np.abs(x) ** 6 * np.exp(-t * t * (x - p) ** 2)) + 1e-300
            np.testing.assert_allclose(v[::-1], ref, atol=2e-7 * scale)


def test_blas_contraction_matches_loops(oracle):
    g = oracle.Grid3D.cube(-1.8, 3, 0.2)
    tp, tw = oracle.gauss_quad(4, 4)
    T = oracle.coulomb_matrix(g.axes[0], g.axes[0].points, tp)
    rho = oracle.gauss_cube(g, [1.0], [1.5], [[0.1, 0.0, -0.1]])
    w = oracle.coulomb_weights(tw)
    V1 = oracle.transform_cube(T, T, T, w, rho, 0.01)
    V2 = oracle.transform_cube_blas(T, T, T, w, rho, 0.01)
    np.testing.assert_allclose(V1, V2, rtol=1e-12, atol=1e-14 * np.abs(V1).max())


def test_oracle_fixture_stable(oracle):
    with open(os.path.join(GOLD, "oracle_small.json")) as f:
        fx = json.load(f)
    gd = fx["grid"]
    g = oracle.Grid3D.cube(gd["qmin"], gd["ncell"], gd["step"], gd["nlip"])
    qd = fx["quadrature"]
    tp, tw = oracle.gauss_quad(qd["nlin"], qd["nlog"], qd["tstart"], qd["tlin"], qd["tlog"])
    np.testing.assert_array_equal(tp, fx["tp"])
    np.testing.assert_array_equal(tw, fx["tw"])
    T = oracle.coulomb_matrix(g.axes[0], g.axes[0].points, tp)
    np.testing.assert_array_equal(T[0, :, 0], fx["T_row0_p0"])


def test_potential_close_to_analytic(oracle):
    """V of a Gaussian density approaches sum q erf(sqrt(a) r)/r."""
    q, a, c = [1.0, 0.7], [1.2, 2.0], [[0.2, -0.1, 0.0], [-0.6, 0.4, 0.3]]
    g = oracle.Grid3D.cube(-6.0, 10, 0.2)
    rho = oracle.gauss_cube(g, q, a, c)
    V = oracle.coulomb_apply(g, rho, quad=(20, 20, 0.0, 2.0, 1.0e3))
    Va = oracle.gauss_pot_cube(g, q, a, c)
    assert np.abs(V - Va).max() / np.abs(Va).max() < 2e-4


def test_slater_analytic_energies_match_reference_goldens(oracle):
    """tests/slater_test.F90 TESTs 1-2: the analytic self-interaction of the
    Slater densities (SlaterGenerator%selfint -> slater_analytical_energy,
    analytical.F90:70-188) reproduces the reference's golden values to its
    tolerance 1e-14, and the restated densities carry unit charge per q."""
    kat = json.load(open(os.path.join(GOLD, "slater_test_kat.json")))
    for case in kat["cases"]:
        c = [s[0] for s in case["shells"]]
        q = [s[1] for s in case["shells"]]
        z = [s[2] for s in case["shells"]]
        E = oracle.slater_analytical_energy(q, z, c)
        assert abs(E - case["selfint_analytic"]) <= kat["tolerance"] * abs(case["selfint_analytic"])
    r = np.linspace(0.0, 40.0, 400001)
    for zeta in (1.0, 2.0, 3.0):
        rho = oracle.slater_dens(zeta, 0, r)
        assert abs(np.trapezoid(4 * np.pi * r * r * rho, r) - 1.0) < 1e-9
