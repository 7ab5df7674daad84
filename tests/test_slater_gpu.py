"""tests/slater_test.F90 TESTs 1-2 through the GPU path: the Slater
densities as bubbles (SlaterGenerator, slater_generator.F90:153-392, cube 0,
Gauss-Lobatto cube grid 8 bohr around the centres, Grid1D_init_radial radial
grids), their Coulomb potential (bubble radial potentials; the cube part is
the operator applied to a zero cube), and rho .dot. V as Function3D_dot_product
forms it (function3d.F90:1499-1528): the product of two cuspy functions with
Taylor-series bubbles (Function3D_multiply_bubbles, function3d.F90:1415-1466)
integrated over cube and bubbles.  Checked against the oracle's restatement
of the same steps and against the reference's numerical and analytic goldens
(tests/golden/slater_test_kat.json)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# (centres, nuclear charges, shells (atom, coefficient, exponent), step)
CASES = {
    1: ([[-0.8660254037844387, -0.5, 0.1], [0.8660254037844387, 0.5, 0.1]], [1.0, 1.0],
        [(0, 1.0, 1.0), (1, 1.0, 1.0)], 0.2),
    2: ([[1.0, 0.5, 1.5], [-1.5, 3.0, 0.5], [-0.5, -1.5, -1.0]], [1.0, 1.0, 2.0],
        [(0, 1.0, 1.0), (0, 1.0, 2.0), (1, 1.0, 1.0), (2, 1.0, 2.0), (2, 1.0, 1.0), (2, 2.0, 3.0)],
        0.4),
}


def _setup(oracle, case):
    centers, zs, shells, step = CASES[case]
    centers = np.asarray(centers)
    rad = [oracle.radial_grid_charge(z) for z in zs]
    f = []
    for a, g in enumerate(rad):
        fa = np.zeros((1, g.n))
        for atom, q, zeta in shells:
            if atom == a:
                fa[0] += q * oracle.slater_dens(zeta, 0, g.points)
        f.append(fa)
    axes = [oracle.Grid1D.spheres(centers[:, d], np.full(len(zs), 8.0), step, 7, 2) for d in range(3)]
    return centers, rad, f, oracle.Grid3D(tuple(axes))


def _oracle_selfint(oracle, centers, rad, f, go, taylor=True, tmax=2):
    V = [oracle.bubbles_coulomb_potential(g.ncell, g.cell_scales, 0, fa) for g, fa in zip(rad, f)]
    n = len(rad)
    if taylor:
        tr = oracle.make_taylor(rad, 0, 0, oracle.bubble_contaminants(centers, rad, 0, f, 0, tmax), None, tmax)
        tv = oracle.make_taylor(rad, 0, 0, oracle.bubble_contaminants(centers, rad, 0, V, 0, tmax), None, tmax)
        f12 = [oracle.bubbles_multiply_taylor(f[a], 0, tr[a], V[a], 0, tv[a]) for a in range(n)]
    else:
        f12 = [oracle.bubbles_multiply(f[a], 0, V[a], 0) for a in range(n)]
    mk = lambda ff: dict(centers=centers, ncells=[g.ncell for g in rad],
                         cell_scales=[g.cell_scales for g in rad], lmax=0, f=ff)
    zero = np.zeros(go.shape, order="F")
    cube = oracle.function3d_multiply(go, zero, zero, mk(f), mk(V), mk(f12))
    return oracle.integrate_cube(go, cube) + oracle.bubbles_integrate(rad, f12)


def _gpu_selfint(dage, centers, rad, f, go, taylor=True, tmax=2):
    g1 = lambda g: dage.Grid1D(g.qmin, g.ncell, g.nlip, g.grid_type, g.cell_scales)
    grid = dage.Grid3D(tuple(g1(a) for a in go.axes))
    rho = dage.Bubbles(centers, [g1(g) for g in rad], f, 0)
    V = rho.coulomb_potential()
    if taylor:
        br = rho.multiply_taylor(V, rho.taylor_series(tmax=tmax), V.taylor_series(tmax=tmax))
    else:
        br = rho.multiply(V)
    zero = np.zeros(go.shape, order="F")
    cube = dage.multiply(grid, zero, zero, rho, V, br)
    return dage.integrate(grid, cube) + br.integrate()


@pytest.mark.parametrize("case", [1, 2])
def test_slater_selfint_through_gpu(dage, oracle, case):
    cases = json.load(open(os.path.join(GOLD, "slater_test_kat.json")))["cases"]
    kat = {c["name"]: c for c in cases}["TEST%d" % case]
    centers, rad, f, go = _setup(oracle, case)
    E = _gpu_selfint(dage, centers, rad, f, go)
    Eo = _oracle_selfint(oracle, centers, rad, f, go)
    assert abs(E - Eo) <= 1e-11 * abs(Eo)
    # the reference's numerical golden (made by an earlier version of the
    # generator, whose bubbles this snapshot no longer builds): 5.5e-7 and
    # 3.0e-4 away; its own distance to the analytic value is 2.3e-6 and 3.3e-4
    gold, exact = kat["selfint_numerical"], kat["selfint_analytic"]
    assert abs(E - gold) <= (1e-6, 5e-4)[case - 1] * abs(gold)
    # the Taylor-series bubbles are what brings the energy there: the plain
    # bubble product misses the analytic value by 1.0e-4 and 4.6e-3
    Ep = _gpu_selfint(dage, centers, rad, f, go, taylor=False)
    assert abs(E - exact) < 0.2 * abs(Ep - exact)


def test_bubbles_integrate_matches_oracle(dage, oracle):
    centers, rad, f, go = _setup(oracle, 2)
    g1 = lambda g: dage.Grid1D(g.qmin, g.ncell, g.nlip, g.grid_type, g.cell_scales)
    rho = dage.Bubbles(centers, [g1(g) for g in rad], f, 0)
    assert abs(rho.integrate() - oracle.bubbles_integrate(rad, f)) <= 1e-13 * 7
    assert abs(rho.integrate() - 7.0) <= 1e-6  # unit charge per coefficient: 1+1+1+1+1+2
    rk = dage.Bubbles(centers, [g1(g) for g in rad], f, 0, k=1)
    assert abs(rk.integrate() - oracle.bubbles_integrate(rad, f, k=1)) <= 1e-13 * abs(rk.integrate())
