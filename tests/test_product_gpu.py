"""GPU tests of the density producer: the radial product of two bubble sets
(BubblesMultiplier_multiply, bubbles.F90:3567-3690) and the fused cube part
of Function3D_multiply (function3d.F90:1097-1409), against the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _set(oracle, centers, lmax, seed, ncell=33, rmax=15.0):
    rng = np.random.default_rng(seed)
    h = oracle.log_radial_grid(ncell, 1e-5, rmax)
    r = oracle.Grid1D(0.0, ncell, 7, 1, h).points
    f = []
    for _ in range(len(centers)):
        fa = np.zeros(((lmax + 1) ** 2, len(r)))
        for l in range(lmax + 1):
            for m in range(-l, l + 1):
                fa[l * (l + 1) + m] = rng.uniform(-1, 1) * r ** l * np.exp(-rng.uniform(0.5, 2) * r)
        f.append(fa)
    return dict(centers=np.asarray(centers, float), ncells=[ncell] * len(centers),
                cell_scales=[h] * len(centers), lmax=lmax, f=f)


def _gpu(dage, s, k=0):
    rad = [dage.Grid1D(0.0, n, 7, 1, h) for n, h in zip(s["ncells"], s["cell_scales"])]
    return dage.Bubbles(s["centers"], rad, s["f"], s["lmax"], k=k)


CENTERS = [[0.1, -0.3, 0.2], [1.4, 0.9, -1.1], [-1.2, 1.0, 0.8]]


@pytest.mark.parametrize("l1,l2,k1,k2", [(0, 0, 0, 0), (1, 2, 0, 1), (2, 2, 0, 0), (3, 2, 1, 1)])
def test_bubbles_multiply_matches_oracle(dage, oracle, l1, l2, k1, k2):
    s1 = _set(oracle, CENTERS, l1, 1)
    s2 = _set(oracle, CENTERS, l2, 2)
    p = _gpu(dage, s1, k1).multiply(_gpu(dage, s2, k2))
    assert p.lmax == l1 + l2
    got = p.radial_values()
    for a in range(len(CENTERS)):
        ref = oracle.bubbles_multiply(s1["f"][a], l1, s2["f"][a], l2)
        assert np.abs(got[a] - ref).max() <= 1e-14 * np.abs(ref).max()


def test_bubbles_product_carries_k(dage, oracle):
    """r^k1 f1 * r^k2 f2 injected equals the injection of the product set."""
    s1 = _set(oracle, CENTERS[:1], 1, 3)
    s2 = _set(oracle, CENTERS[:1], 1, 4)
    b1, b2 = _gpu(dage, s1, 1), _gpu(dage, s2, 1)
    g = dage.Grid3D.cube(-2.0, 4, 0.2)
    p = b1.multiply(b2, complete=True)
    prod = b1.inject(g) * b2.inject(g)
    inj = p.inject(g)
    assert np.abs(prod - inj).max() <= 2e-5 * np.abs(prod).max()  # LIP interpolation (3.7e-6)


@pytest.mark.parametrize("natom,l1,l2", [(1, 0, 0), (3, 1, 2), (3, 2, 2)])
def test_function_product_matches_oracle(dage, oracle, natom, l1, l2):
    g = dage.Grid3D.cube(-3.0, 6, 0.2)
    go = oracle.Grid3D.cube(-3.0, 6, 0.2)
    rng = np.random.default_rng(natom)
    c1 = np.asfortranarray(rng.standard_normal(go.shape))
    c2 = np.asfortranarray(rng.standard_normal(go.shape))
    s1 = _set(oracle, CENTERS[:natom], l1, 5)
    s2 = _set(oracle, CENTERS[:natom], l2, 6)
    b1, b2 = _gpu(dage, s1), _gpu(dage, s2)
    br = b1 * b2
    out = dage.multiply(g, c1, c2, b1, b2, br)
    sr = dict(s1, lmax=l1 + l2,
              f=[oracle.bubbles_multiply(s1["f"][a], l1, s2["f"][a], l2) for a in range(natom)])
    ref = oracle.function3d_multiply(go, c1, c2, s1, s2, sr)
    assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max()


def test_function_product_without_bubbles_and_on_device(dage, oracle):
    import torch

    g = dage.Grid3D.cube(-3.0, 5, 0.25)
    n = tuple(a.n for a in g.axes)
    c1 = torch.randn(n[::-1], dtype=torch.float64, device="cuda")
    c2 = torch.randn(n[::-1], dtype=torch.float64, device="cuda")
    want = c1 * c2
    dage.multiply(g, c1, c2, out=c1)  # in place
    torch.cuda.synchronize()
    assert torch.equal(c1, want)
    s1 = _set(oracle, CENTERS, 2, 8)
    b1 = _gpu(dage, s1)
    d2 = torch.randn(n[::-1], dtype=torch.float64, device="cuda")
    out = dage.multiply(g, d2, d2, b1, None, None)
    host = oracle.bubbles_inject(cube=np.zeros(n, order="F"), grid=oracle.Grid3D.cube(-3.0, 5, 0.25),
                                 **s1)
    d2h = d2.cpu().numpy().reshape(-1).reshape(n, order="F")
    ref = (d2h + host) * d2h
    got = out.cpu().numpy().reshape(-1).reshape(n, order="F")
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_complete_table_leaves_only_interpolation_error(dage, oracle):
    """One atom, no cubes: (B1)(B2) - B1*B2 is the LIP interpolation error
    with the complete product; the reference's term set leaves the
    L < |m1-m2| terms in the cube instead."""
    g = dage.Grid3D.cube(-2.5, 5, 0.2)
    n = tuple(a.n for a in g.axes)
    zero = np.zeros(n, order="F")
    s1 = _set(oracle, CENTERS[:1], 1, 9)
    s2 = _set(oracle, CENTERS[:1], 2, 10)
    b1, b2 = _gpu(dage, s1), _gpu(dage, s2)
    full = b1.inject(g) * b2.inject(g)
    rest_c = dage.multiply(g, zero, zero, b1, b2, b1.multiply(b2, complete=True))
    rest_r = dage.multiply(g, zero, zero, b1, b2, b1.multiply(b2))
    assert np.abs(rest_c).max() <= 1e-5 * np.abs(full).max()  # 6.1e-7 in the oracle
    assert np.abs(rest_r).max() > 5e-4 * np.abs(full).max()  # 1.7e-3 in the oracle
