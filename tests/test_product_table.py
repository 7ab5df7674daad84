"""The real-harmonic product table (YProduct, harmonic.F90:884-1089): the
oracle's restatement of the reference's Clebsch-Gordan formula, checked
against the product identity Y_a Y_b = sum C Y_LM at random directions, and
the library's host-built table (projection on the sphere) against it.  No
GPU is needed: the table is built on the host."""
import ctypes

import numpy as np
import pytest


def _lib_table(dage, lmax, result_lmax, complete=False):
    lib = dage.load()
    n = ctypes.c_int()
    flags = dage._capi.DAGE_PRODUCT_COMPLETE if complete else 0
    assert lib.dage_product_table(lmax, result_lmax, flags, 0, None, None, None, None,
                                  ctypes.byref(n)) == 0
    a = np.zeros(n.value, dtype=np.int32)
    b = np.zeros_like(a)
    lm = np.zeros_like(a)
    c = np.zeros(n.value)
    ip = ctypes.POINTER(ctypes.c_int)
    assert lib.dage_product_table(lmax, result_lmax, flags, n.value, a.ctypes.data_as(ip),
                                  b.ctypes.data_as(ip), lm.ctypes.data_as(ip),
                                  c.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                  ctypes.byref(n)) == 0
    table = {}
    for i in range(n.value):
        table.setdefault((int(a[i]), int(b[i])), {})[int(lm[i])] = c[i]
    return table


def _lm(i):
    l = int(np.sqrt(i))
    return l, i - l * (l + 1)


def test_documented_products(oracle):
    """s*s = s; px*px = 1/3 s - 1/3 dz2 + 1/sqrt(3) dx2-y2 (Racah-normalised)."""
    t = oracle.yproduct(2)
    assert t[(0, 0)] == [(0, 1.0)]
    d = dict(t[(3, 3)])
    assert abs(d[0] - 1 / 3) < 1e-15 and abs(d[6] + 1 / 3) < 1e-15
    assert abs(d[8] - 1 / np.sqrt(3)) < 1e-15


@pytest.mark.parametrize("lmax", [2, 4])
def test_oracle_table_is_the_product_expansion_where_complete(oracle, lmax):
    """Every pair the reference enumeration covers fully satisfies the
    identity; the others miss exactly the terms with L < |m1 - m2|."""
    T = oracle.yproduct(lmax)
    rng = np.random.default_rng(lmax)
    for _ in range(8):
        v = rng.standard_normal(3)
        v /= np.linalg.norm(v)
        Y = oracle.solid_harmonics(2 * lmax, v)
        for (a, b), terms in T.items():
            (l1, m1), (l2, m2) = _lm(a), _lm(b)
            rhs = sum(C * Y[LM] for LM, C in terms)
            if abs(m1 - m2) <= abs(l1 - l2) or m1 * m2 >= 0:
                assert abs(Y[a] * Y[b] - rhs) < 1e-13, (l1, m1, l2, m2)


@pytest.mark.parametrize("lmax", [1, 2, 3, 5])
def test_library_table_matches_oracle(dage_host, oracle, lmax):
    T = oracle.yproduct(lmax, 2 * lmax)
    G = _lib_table(dage_host, lmax, 2 * lmax)
    for (a, b), terms in T.items():
        ref = {LM: C for LM, C in terms if abs(C) > 1e-13}
        got = G.get((a, b), {})
        assert set(got) == set(ref), (a, b)
        for LM, C in ref.items():
            assert abs(got[LM] - C) < 1e-14, (a, b, LM)
    assert set(G) <= set(T)


@pytest.mark.parametrize("lmax", [2, 3])
def test_complete_table_satisfies_the_identity(dage_host, oracle, lmax):
    G = _lib_table(dage_host, lmax, 2 * lmax, complete=True)
    rng = np.random.default_rng(7)
    N = (lmax + 1) ** 2
    for _ in range(8):
        v = rng.standard_normal(3)
        v /= np.linalg.norm(v)
        Y = oracle.solid_harmonics(2 * lmax, v)
        for a in range(N):
            for b in range(a, N):
                rhs = sum(C * Y[LM] for LM, C in G.get((a, b), {}).items())
                assert abs(Y[a] * Y[b] - rhs) < 1e-13
