"""GPU tests of the Taylor-series contaminant bubbles against the oracle's
restatement of Bubbles_get_contaminants (bubbles.F90:2844-2910),
Function3D_get_cube_contaminants (function3d.F90:1570-1624),
Bubbles_make_taylor (bubbles.F90:1435-1530) and option (1) of
BubblesMultiplier_multiply (bubbles.F90:3567-3640), and of the exact series
against the function it expands."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CENTERS = np.array([[0.1, -0.3, 0.2], [1.4, 0.9, -1.1], [-1.2, 1.0, 0.8], [9.0, -8.0, 7.5]])


def _set(oracle, lmax, seed, natom=3, rmax=15.0):
    rng = np.random.default_rng(seed)
    h = oracle.log_radial_grid(33, 1e-5, rmax)
    g = oracle.Grid1D(0.0, 33, 7, 1, h)
    r = g.points
    f = []
    for _ in range(natom):
        fa = np.zeros(((lmax + 1) ** 2, len(r)))
        for l in range(lmax + 1):
            for m in range(-l, l + 1):
                fa[l * (l + 1) + m] = rng.uniform(-1, 1) * r ** l * np.exp(-rng.uniform(0.5, 2) * r)
        f.append(fa)
    return CENTERS[:natom], g, h, f


def _gpu(dage, centers, h, f, lmax, k=0):
    rad = [dage.Grid1D(0.0, 33, 7, 1, h) for _ in range(len(centers))]
    return dage.Bubbles(centers, rad, f, lmax, k=k)


# (lmax, k, tmax, natom, rmax): the fourth atom lies beyond the others'
# radial grids when rmax = 12 (contributes and receives nothing there)
@pytest.mark.parametrize("lmax,k,tmax,natom,rmax", [(0, 0, 0, 2, 15.0), (2, 0, 2, 3, 15.0),
                                                    (1, 1, 3, 3, 15.0), (4, 0, 3, 4, 12.0),
                                                    (2, 0, 1, 4, 20.0)])
def test_bubble_contaminants_match_oracle(dage, oracle, lmax, k, tmax, natom, rmax):
    centers, g, h, f = _set(oracle, lmax, 11 + lmax, natom, rmax)
    b = _gpu(dage, centers, h, f, lmax, k)
    got = b.contaminants(tmax)
    ref = oracle.bubble_contaminants(centers, [g] * natom, lmax, f, k, tmax)
    assert got.shape == ref.shape
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    if rmax == 12.0:
        assert np.all(got[3] == 0.0)


@pytest.mark.parametrize("tmax,gtype", [(0, 1), (2, 1), (3, 1), (2, 2)])  # 2: Gauss-Lobatto cells
def test_cube_contaminants_match_oracle(dage, oracle, tmax, gtype):
    import torch

    g = dage.Grid3D.cube(-3.0, 6, 0.2, grid_type=gtype)
    go = oracle.Grid3D.cube(-3.0, 6, 0.2, grid_type=gtype)
    cube = np.asfortranarray(np.random.default_rng(tmax).standard_normal(go.shape))
    # inside, on a cell boundary, on the last point, outside
    cen = np.array([[0.13, -0.41, 0.57], [0.6, 1.8, -0.6], [4.2, 4.2, 4.2], [5.0, 0.0, 0.0]])
    ref = oracle.cube_contaminants(go, cube, cen, tmax)
    got = dage.cube_contaminants(g, cube, cen, tmax)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    assert np.all(got[3] == 0.0)
    dev = torch.from_numpy(cube.reshape(-1, order="F").copy()).cuda()
    assert np.array_equal(dage.cube_contaminants(g, dev, cen, tmax), got)


@pytest.mark.parametrize("lmax,k,tmax,exact", [(2, 0, 2, False), (1, 0, 3, False),
                                               (3, 1, 3, False), (2, 0, 3, True), (0, 0, 2, True)])
def test_make_taylor_matches_oracle(dage, oracle, lmax, k, tmax, exact):
    centers, g, h, f = _set(oracle, lmax, 21, 3)
    b = _gpu(dage, centers, h, f, lmax, k)
    nc = (tmax + 1) * (tmax + 2) * (tmax + 3) // 6
    rng = np.random.default_rng(5)
    cb, cc = rng.standard_normal((3, nc)), rng.standard_normal((3, nc))
    t = b.make_taylor(cb, cc, tmax, exact=exact)
    assert t.lmax == max(lmax, tmax)
    got = t.radial_values()
    ref = oracle.make_taylor([g] * 3, lmax, k, cb, cc, tmax, exact=exact)
    for a in range(3):
        assert got[a].shape == ref[a].shape
        assert np.abs(got[a] - ref[a]).max() <= 1e-13 * np.abs(ref[a]).max()


def test_taylor_series_matches_oracle(dage, oracle):
    """The combined call (contaminants kept on the GPU) against the oracle's
    three steps, the cube given as a host array and as a CUDA tensor, and
    without cube or bubbles."""
    import torch

    lmax, tmax = 2, 2
    centers, g, h, f = _set(oracle, lmax, 31, 3)
    b = _gpu(dage, centers, h, f, lmax)
    gr = dage.Grid3D.cube(-3.0, 6, 0.2)
    go = oracle.Grid3D.cube(-3.0, 6, 0.2)
    cube = np.asfortranarray(np.random.default_rng(2).standard_normal(go.shape))
    cb = oracle.bubble_contaminants(centers, [g] * 3, lmax, f, 0, tmax)
    cc = oracle.cube_contaminants(go, cube, centers, tmax)
    cases = [(dict(grid=gr, cube=cube), cb, cc),
             (dict(grid=gr, cube=torch.from_numpy(cube.reshape(-1, order="F").copy()).cuda()), cb, cc),
             (dict(), cb, None),
             (dict(grid=gr, cube=cube, ignore_bubbles=True), None, cc)]
    for kw, rb, rc in cases:
        got = b.taylor_series(tmax=tmax, **kw).radial_values()
        ref = oracle.make_taylor([g] * 3, lmax, 0, rb, rc, tmax)
        for a in range(3):
            assert np.abs(got[a] - ref[a]).max() <= 1e-12 * np.abs(ref[a]).max()


@pytest.mark.parametrize("l1,l2,tmax", [(1, 2, 2), (2, 2, 2), (0, 1, 2)])
def test_multiply_taylor_matches_oracle(dage, oracle, l1, l2, tmax):
    centers, g, h, f1 = _set(oracle, l1, 41, 3)
    _, _, _, f2 = _set(oracle, l2, 42, 3)
    b1, b2 = _gpu(dage, centers, h, f1, l1), _gpu(dage, centers, h, f2, l2)
    t1, t2 = b1.taylor_series(tmax=tmax), b2.taylor_series(tmax=tmax)
    p = b1.multiply_taylor(b2, t1, t2)
    assert p.lmax == l1 + l2
    got = p.radial_values()
    tv1, tv2 = t1.radial_values(), t2.radial_values()
    for a in range(3):
        ref = oracle.bubbles_multiply_taylor(f1[a], l1, tv1[a], f2[a], l2, tv2[a])
        assert np.abs(got[a] - ref).max() <= 1e-13 * np.abs(ref).max()


def test_function_product_with_taylor_bubbles(dage, oracle):
    """Function3D_multiply for two cuspy functions: result bubbles from the
    Taylor product, then the cube (c1 + B1)(c2 + B2) - B12."""
    lmax, tmax = 1, 2
    centers, g, h, f1 = _set(oracle, lmax, 51, 3)
    _, _, _, f2 = _set(oracle, lmax, 52, 3)
    gr = dage.Grid3D.cube(-3.0, 6, 0.2)
    go = oracle.Grid3D.cube(-3.0, 6, 0.2)
    rng = np.random.default_rng(3)
    c1 = np.asfortranarray(0.1 * rng.standard_normal(go.shape))
    c2 = np.asfortranarray(0.1 * rng.standard_normal(go.shape))
    b1, b2 = _gpu(dage, centers, h, f1, lmax), _gpu(dage, centers, h, f2, lmax)
    t1 = b1.taylor_series(gr, c1, tmax)
    t2 = b2.taylor_series(gr, c2, tmax)
    b12 = b1.multiply_taylor(b2, t1, t2)
    out = dage.multiply(gr, c1, c2, b1, b2, b12)
    tv1 = oracle.make_taylor([g] * 3, lmax, 0, oracle.bubble_contaminants(centers, [g] * 3, lmax, f1, 0, tmax),
                             oracle.cube_contaminants(go, c1, centers, tmax), tmax)
    tv2 = oracle.make_taylor([g] * 3, lmax, 0, oracle.bubble_contaminants(centers, [g] * 3, lmax, f2, 0, tmax),
                             oracle.cube_contaminants(go, c2, centers, tmax), tmax)
    f12 = [oracle.bubbles_multiply_taylor(f1[a], lmax, tv1[a], f2[a], lmax, tv2[a]) for a in range(3)]
    mk = lambda f, l: dict(centers=centers, ncells=[33] * 3, cell_scales=[h] * 3, lmax=l, f=f)
    ref = oracle.function3d_multiply(go, c1, c2, mk(f1, lmax), mk(f2, lmax), mk(f12, 2 * lmax))
    assert np.abs(out - ref).max() <= 1e-11 * np.abs(ref).max()


@pytest.mark.parametrize("tmax", [1, 2, 3])
def test_exact_series_converges_to_function(dage, oracle, tmax):
    """DAGE_TAYLOR_EXACT: around each atom B, the injected Taylor bubble of B
    equals the other atoms' bubbles up to O(|x|^(tmax+1)); halving the
    distance divides the error by about 2^(tmax+1)."""
    lmax = 2
    centers, g, h, f = _set(oracle, lmax, 61, 3)
    b = _gpu(dage, centers, h, f, lmax)
    t = b.taylor_series(tmax=tmax, exact=True)
    tv = t.radial_values()
    rad = dage.Grid1D(0.0, 33, 7, 1, h)
    for B in range(3):
        others = [A for A in range(3) if A != B]
        own = dage.Bubbles(centers[B:B + 1], [rad], [tv[B]], max(lmax, tmax))
        rest = dage.Bubbles(centers[others], [rad] * 2, [f[A] for A in others], lmax)
        errs = []
        for delta in (0.02, 0.01):
            axes = tuple(dage.Grid1D.equidistant(c - 3 * delta, 1, delta) for c in centers[B])
            st = dage.Grid3D(axes)
            errs.append(np.abs(own.inject(st) - rest.inject(st)).max())
        assert errs[1] < errs[0] / (2 ** (tmax + 1) / 1.6), (B, errs)


def test_taylor_refusals(dage, oracle):
    centers, g, h, f = _set(oracle, 1, 71, 2)
    b = _gpu(dage, centers, h, f, 1)
    with pytest.raises(dage.DageError):
        b.contaminants(4)
    same = _gpu(dage, np.array([centers[0], centers[0]]), h, f, 1)
    with pytest.raises(dage.DageError):
        same.contaminants(2)
    other = _gpu(dage, centers[::-1].copy(), h, f, 1)
    t = b.taylor_series(tmax=2)
    with pytest.raises(dage.DageError):
        b.multiply_taylor(other, t, t)


def test_single_atom_and_high_lmax(dage, oracle):
    """One atom has no other atoms to contaminate it (zero contaminants, and
    the Taylor bubbles of the bubbles alone vanish); lmax 6 bubbles with
    tmax 3 exercise the harmonic recursion on jets up to l = 6."""
    centers, g, h, f = _set(oracle, 2, 81, natom=1)
    b = _gpu(dage, centers, h, f, 2)
    assert np.all(b.contaminants(3) == 0.0)
    t = b.taylor_series(tmax=2)
    assert all(np.all(v == 0.0) for v in t.radial_values())
    centers, g, h, f = _set(oracle, 6, 82, natom=3)
    b = _gpu(dage, centers, h, f, 6)
    got = b.contaminants(3)
    ref = oracle.bubble_contaminants(centers, [g] * 3, 6, f, 0, 3)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_multiply_taylor_complete_table(dage, oracle):
    """DAGE_PRODUCT_COMPLETE in the Taylor product: the plain complete product
    plus the complete products with the Taylor sets (bilinearity)."""
    centers, g, h, f1 = _set(oracle, 2, 91, 3)
    _, _, _, f2 = _set(oracle, 1, 92, 3)
    b1, b2 = _gpu(dage, centers, h, f1, 2), _gpu(dage, centers, h, f2, 1)
    t1, t2 = b1.taylor_series(tmax=2), b2.taylor_series(tmax=2)
    p = b1.multiply_taylor(b2, t1, t2, complete=True).radial_values()
    q = b1.multiply(b2, complete=True).radial_values()
    tv1, tv2 = t1.radial_values(), t2.radial_values()
    c1 = dage.Bubbles(centers, [dage.Grid1D(0.0, 33, 7, 1, h)] * 3, [v[:9] for v in tv1], 2)
    c2 = dage.Bubbles(centers, [dage.Grid1D(0.0, 33, 7, 1, h)] * 3, [v[:4] for v in tv2], 1)
    r1 = b1.multiply(c2, complete=True).radial_values()
    r2 = c1.multiply(b2, complete=True).radial_values()
    for a in range(3):
        ref = q[a] + r1[a] + r2[a]
        assert np.abs(p[a] - ref).max() <= 1e-13 * np.abs(ref).max()
