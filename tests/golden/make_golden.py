"""Writes tests/golden/*.json.

gauss_test_kat.json holds the known-answer values that the reference's own
test program asserts (tests/gauss_test.F90 of DAGE, TESTs 1-3), copied as
numbers together with the inputs that produce them.  Those goldens were made
with the quadrature defaults of their time: nlin=10, nlog=8, tlin=2,
tlog=500 (today's GaussQuad default tlog is 1000); with those parameters,
equidistant 7-point (TEST 3: 5-point) cells and the coda term included, the
CPU oracle reproduces them to the reference test's tolerance of 1e-14.

multipole_test_kat.json holds the golden errors of the reference's
multipole test (tests/multipole_test.F90, displaced_monopoles_test), which
pin the M2L interaction matrix and the M2M translation matrix.

slater_test_kat.json holds the values of the reference's Slater test
(tests/slater_test.F90, TESTs 1-2): the Slater s-densities (explicit and
parsed input), the analytic self-interaction energies that its
SlaterGenerator%selfint returns (slater_analytical_energy, analytical.F90),
and the numerical <rho|V rho> it asserts.  The numerical values came from a
version of SlaterGenerator whose bubbles constructor is commented out in
the reference snapshot (slater_generator.F90:264-284), with Taylor-series
cusp treatment in the product; they are recorded with that provenance.

oracle_small.json freezes oracle outputs for a small operator (matrices and
potential samples) so the GPU tests have committed fixtures to compare with.
Regenerate with:  python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import oracle as O  # noqa: E402

KAT = {
    "source": "DAGE tests/gauss_test.F90 (TEST 1 :70-96, TEST 2 :105-132, TEST 3 :139-162)",
    "quadrature": {"nlin": 10, "nlog": 8, "tstart": 0.0, "tlin": 2.0, "tlog": 500.0},
    "coda": True,
    "grid_type": 1,
    "tolerance": 1e-14,
    "cases": [
        {"name": "TEST1", "q": [1.0], "alpha": [1.0], "centers": [[0.0, 0.0, 0.0]],
         "step": 0.2, "thres": 1e-12, "nlip": 7,
         "selfint": 0.7979283927253593, "selfint_analytic": 0.7978845608028654},
        {"name": "TEST2", "q": [1.0, 1.0, 1.0, 1.0], "alpha": [3.0, 0.4, 2.0, 1.5],
         "centers": [[-7.0, 0.0, 0.0], [0.0, 4.0, 4.0], [4.0, -10.0, -2.0], [3.0, 6.0, -5.0]],
         "step": 0.2, "thres": 1e-12, "nlip": 7,
         "selfint": 4.9612607728784432, "selfint_analytic": 4.9612771741430324},
        {"name": "TEST3", "q": [1.0, -1.0], "alpha": [2.0, 4.0],
         "centers": [[-1.0, 0.0, 0.0], [1.0, 0.0, 0.0]],
         "step": 0.1, "thres": 1e-8, "nlip": 5,
         "selfint": 1.7252361611235862, "selfint_analytic": 1.7252391238773686},
    ],
}


MULTIPOLE_KAT = {
    "source": "DAGE tests/multipole_test.F90 displaced_monopoles_test (:185-300)",
    "note": "|qi . T(boxj - boxi) qj - 1/|ri - rj|| for unit monopoles at ri, rj "
            "translated to the box centres, truncated at l = 0..15",
    "rj": [-12.31523266, -2.77677722, -13.87351588],
    "ri": [-13.80289944, -12.66934534, -8.92620243],
    "boxj": [-10.625, -2.125, -14.875],
    "boxi": [-14.875, -10.625, -10.625],
    "err_ref": [6.4549767744542658e-003, 3.5239702059782635e-003, 3.6472898611333848e-005,
                3.5551144335181639e-004, 1.2985977061118203e-004, 3.0889425959704231e-005,
                1.8391214269969369e-006, 2.0053722605550828e-006, 1.0603102051365276e-006,
                2.9594595833681847e-007, 3.4396637579869882e-008, 1.2534625434823532e-008,
                9.0637385791181302e-009, 2.9670064183306977e-009, 4.8909977456990106e-010,
                6.3554106422003542e-011],
}


SLATER_KAT = {
    "source": "DAGE tests/slater_test.F90 (TEST 1 :70-101, TEST 2 :106-143)",
    "tolerance": 1e-14,
    "cases": [
        {"name": "TEST1", "step": 0.2,
         # centers of the shells, charge q, exponent zeta (l = m = 0)
         "shells": [[[-0.8660254037844387, -0.5, 0.1], 1.0, 1.0],
                    [[0.8660254037844387, 0.5, 0.1], 1.0, 1.0]],
         "selfint_numerical": 2.1019438083447435, "selfint_analytic": 2.1019485856493985},
        {"name": "TEST2", "step": 0.4,
         "shells": [[[1.0, 0.5, 1.5], 1.0, 1.0], [[1.0, 0.5, 1.5], 1.0, 2.0],
                    [[-1.5, 3.0, 0.5], 1.0, 1.0],
                    [[-0.5, -1.5, -1.0], 1.0, 2.0], [[-0.5, -1.5, -1.0], 1.0, 1.0],
                    [[-0.5, -1.5, -1.0], 2.0, 3.0]],
         "selfint_numerical": 31.8808479535843396, "selfint_analytic": 31.8912297114622483},
    ],
}


def small_fixture():
    g = O.Grid3D.cube(-2.4, 4, 0.2)  # 25 points per axis
    tp, tw = O.gauss_quad(6, 6, 0.0, 2.0, 1.0e3)
    T = O.coulomb_matrix(g.axes[0], g.axes[0].points, tp)
    q, a, c = [1.0, -0.5], [1.3, 2.2], [[0.3, -0.2, 0.1], [-0.4, 0.5, -0.3]]
    rho = O.gauss_cube(g, q, a, c)
    V = O.transform_cube(T, T, T, O.coulomb_weights(tw), rho, O.coda_of(1.0e3))
    idx = [(0, 0, 0), (12, 12, 12), (3, 17, 9), (24, 1, 20), (7, 7, 23)]
    return {
        "grid": {"qmin": -2.4, "ncell": 4, "step": 0.2, "nlip": 7},
        "quadrature": {"nlin": 6, "nlog": 6, "tstart": 0.0, "tlin": 2.0, "tlog": 1000.0},
        "tp": tp.tolist(), "tw": tw.tolist(),
        "T_diag": [float(T[i, i, p]) for p in range(len(tp)) for i in (0, 6, 12)],
        "T_row0_p0": T[0, :, 0].tolist(),
        "T_row12_plast": T[12, :, -1].tolist(),
        "gauss": {"q": q, "alpha": a, "centers": c},
        "V_samples": [[list(i), float(V[i])] for i in idx],
        "energy": O.integrate_cube(g, rho * V),
    }


if __name__ == "__main__":
    with open(os.path.join(HERE, "gauss_test_kat.json"), "w") as f:
        json.dump(KAT, f, indent=1)
    with open(os.path.join(HERE, "multipole_test_kat.json"), "w") as f:
        json.dump(MULTIPOLE_KAT, f, indent=1)
    with open(os.path.join(HERE, "slater_test_kat.json"), "w") as f:
        json.dump(SLATER_KAT, f, indent=1)
    with open(os.path.join(HERE, "oracle_small.json"), "w") as f:
        json.dump(small_fixture(), f, indent=1)
    print("wrote", HERE)
