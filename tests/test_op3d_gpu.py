"""GPU parity tests of the FP64 cube operator (the drop-in) against the CPU
oracle, through the C ABI.

Bars (all max-norm relative unless said otherwise):
- the contraction, coda and energy given the same operator matrices:
  <= 1e-12 (the GPU arithmetic itself);
- the operator matrices: within 10x the spread the reference algorithm shows
  when erf/exp move by +-1 ulp (the oracle's libm_1ulp build) -- the
  reference's closed-form integrals cancel heavily for t*h just above 0.1,
  so no other libm can reproduce their last bits;
- the potential end to end: <= max(1e-10, 10x that same libm spread);
- energies: <= 1e-12 relative, and the reference's own known answers
  (tests/gauss_test.F90) to 1e-13 absolute."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL_FP64 = 1e-10


def _grids(dage, oracle, qmin, ncell, step, nlip=7, gt=1):
    return (dage.Grid3D.cube(qmin, ncell, step, nlip, gt), oracle.Grid3D.cube(qmin, ncell, step, nlip, gt))


def _relmax(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def _check_apply(oracle, op, go, rho, quad, V, E, coda=True):
    """V, E from the GPU operator `op` against the oracle."""
    tp, tw = oracle.gauss_quad(*quad)
    w = oracle.coulomb_weights(tw)
    c = oracle.coda_of(quad[4]) if coda else 0.0
    # 1. the GPU arithmetic: same matrices through the oracle's contraction
    Tg = [op.matrix(d) for d in range(3)]
    Vg = oracle.transform_cube(*Tg, w, rho, c)
    assert _relmax(V, Vg) <= 1e-12
    Eg = oracle.integrate_cube(go, rho * Vg)
    assert abs(E - Eg) <= 1e-12 * abs(Eg)
    # 2. end to end against the oracle, within the reference's libm spread
    To = oracle.coulomb_operator_matrices(go, go, tp)
    T1 = oracle.coulomb_operator_matrices(go, go, tp, libm_1ulp=True)
    Vo = oracle.transform_cube(*To, w, rho, c)
    V1 = oracle.transform_cube(*T1, w, rho, c)
    spread = _relmax(V1, Vo)
    assert _relmax(V, Vo) <= max(1e-10, 10 * spread), (_relmax(V, Vo), spread)
    Eo = oracle.integrate_cube(go, rho * Vo)
    assert abs(E - Eo) <= 1e-12 * abs(Eo)
    return Vo


def test_quadrature_matches_oracle(dage, oracle):
    g, _ = _grids(dage, oracle, -2.4, 4, 0.2)
    for q in [(10, 8, 0.0, 2.0, 1e3), (32, 32, 0.0, 2.0, 1e3), (20, 16, 0.0, 2.0, 500.0), (7, 0, 0.0, 3.0, 10.0)]:
        op = dage.Coulomb3D(g, quad=dage.GaussQuad(*q))
        tp, w = op.quadrature()
        tpo, two = oracle.gauss_quad(*q)
        np.testing.assert_allclose(tp, tpo, rtol=1e-14)
        np.testing.assert_allclose(w, oracle.coulomb_weights(two), rtol=1e-13)


@pytest.mark.parametrize("ncell,step,nlip,gt", [(4, 0.2, 7, 1), (20, 0.2, 7, 1), (6, 0.1, 5, 1),
                                                (5, 0.3, 7, 2), (3, 0.15, 6, 2)])
def test_matrices_match_oracle(dage, oracle, ncell, step, nlip, gt):
    qmin = -0.5 * ncell * (nlip - 1) * step
    g, go = _grids(dage, oracle, qmin, ncell, step, nlip, gt)
    quad = (16, 16, 0.0, 2.0, 1e3)
    op = dage.Coulomb3D(g, quad=dage.GaussQuad(*quad))
    tp, _ = oracle.gauss_quad(*quad)
    T = op.matrix(0)
    To = oracle.coulomb_matrix(go.axes[0], go.axes[0].points, tp)
    T1 = oracle.coulomb_matrix(go.axes[0], go.axes[0].points, tp, libm_1ulp=True)
    env = oracle.matrix_noise_envelope(To, T1)
    for p in range(T.shape[2]):
        tol = 10 * env[:, :, p] + 1e-13 * np.abs(To[:, :, p]).max()
        assert np.all(np.abs(T[:, :, p] - To[:, :, p]) <= tol), p
    # the 12-point Gauss rule branch (t*h < 0.1) has no cancellation: there
    # the GPU agrees to 1e-12 of the slice maximum
    for p in range(T.shape[2]):
        if tp[p] * step < 0.1:
            assert np.abs(T[:, :, p] - To[:, :, p]).max() <= 1e-12 * np.abs(To[:, :, p]).max(), p


def test_matrices_distinct_grids(dage, oracle):
    """Input and output grids differ (the GBFMM near-field situation)."""
    gi = dage.Grid3D.cube(-1.2, 2, 0.2)
    go_ = dage.Grid3D((dage.Grid1D.equidistant(-2.4, 4, 0.2), dage.Grid1D.equidistant(-1.2, 2, 0.2),
                       dage.Grid1D.equidistant(0.0, 3, 0.1)))
    quad = (8, 8, 0.0, 2.0, 1e3)
    op = dage.Coulomb3D(gi, go_, quad=dage.GaussQuad(*quad))
    oi = oracle.Grid3D.cube(-1.2, 2, 0.2)
    tp, tw = oracle.gauss_quad(*quad)
    pts = [np.asarray(oracle.Grid1D.equidistant(-2.4, 4, 0.2).points),
           np.asarray(oracle.Grid1D.equidistant(-1.2, 2, 0.2).points),
           np.asarray(oracle.Grid1D.equidistant(0.0, 3, 0.1).points)]
    Ts = [oracle.coulomb_matrix(oi.axes[d], pts[d], tp) for d in range(3)]
    Tg = []
    for d in range(3):
        T = op.matrix(d)
        assert T.shape == Ts[d].shape
        T1 = oracle.coulomb_matrix(oi.axes[d], pts[d], tp, libm_1ulp=True)
        env = oracle.matrix_noise_envelope(Ts[d], T1)
        assert np.all(np.abs(T - Ts[d]) <= 10 * env + 1e-13 * np.abs(Ts[d]).max())
        Tg.append(T)
    rho = oracle.gauss_cube(oi, [1.0], [2.0], [[0.1, -0.1, 0.05]])
    V = op.apply(np.asfortranarray(rho))
    Vo = oracle.transform_cube(*Tg, oracle.coulomb_weights(tw), rho, 0.0)
    assert _relmax(V, Vo) <= 1e-12


@pytest.mark.parametrize("ncell,step,quad", [(4, 0.2, (6, 6, 0.0, 2.0, 1e3)),
                                             (9, 0.2, (10, 8, 0.0, 2.0, 500.0)),
                                             (7, 0.1, (12, 10, 0.0, 2.0, 1e3))])
def test_apply_fp64_matches_oracle(dage, oracle, ncell, step, quad):
    qmin = -3.0 * ncell * step
    g, go = _grids(dage, oracle, qmin, ncell, step)
    rng = np.random.default_rng(ncell)
    q = rng.uniform(0.5, 2, 3)
    a = rng.uniform(0.5, 4, 3)
    c = rng.uniform(-1, 1, (3, 3))
    rho = oracle.gauss_cube(go, q, a, c)
    op = dage.Coulomb3D(g, quad=dage.GaussQuad(*quad))
    V, E = op.apply(rho, energy=True)
    _check_apply(oracle, op, go, rho, quad, V, E)


def test_committed_fixture(dage):
    with open(os.path.join(GOLD, "oracle_small.json")) as f:
        fx = json.load(f)
    gd, qd = fx["grid"], fx["quadrature"]
    g = dage.Grid3D.cube(gd["qmin"], gd["ncell"], gd["step"], gd["nlip"])
    op = dage.Coulomb3D(g, quad=dage.GaussQuad(qd["nlin"], qd["nlog"], qd["tstart"], qd["tlin"], qd["tlog"]))
    T = op.matrix(0)
    np.testing.assert_allclose(T[0, :, 0], fx["T_row0_p0"], rtol=1e-12, atol=1e-13 * np.abs(T[0, :, 0]).max())
    pts = g.axes[0].coordinates()
    gs = fx["gauss"]
    X, Y, Z = np.meshgrid(pts, pts, pts, indexing="ij")
    rho = np.zeros(X.shape)
    for q, a, c in zip(gs["q"], gs["alpha"], gs["centers"]):
        rho += q * (a / np.pi) ** 1.5 * np.exp(-a * ((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2))
    V, E = op.apply(np.asfortranarray(rho), energy=True)
    for idx, val in fx["V_samples"]:
        assert abs(V[tuple(idx)] - val) <= 1e-10 * abs(val)
    assert abs(E - fx["energy"]) <= 1e-10 * abs(fx["energy"])


def _kat():
    with open(os.path.join(GOLD, "gauss_test_kat.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("case", _kat()["cases"], ids=lambda c: c["name"])
def test_gauss_test_kat_on_gpu(dage, oracle, case):
    """The reference's own known answers, through the GPU operator."""
    kat = _kat()
    qd = kat["quadrature"]
    og = oracle.Grid3D.gauss_default(case["q"], case["alpha"], case["centers"], step=case["step"],
                                     nlip=case["nlip"], thres=case["thres"])
    g = dage.Grid3D(tuple(dage.Grid1D(a.qmin, a.ncell, a.nlip, 1, a.cell_scales) for a in og.axes))
    rho = oracle.gauss_cube(og, case["q"], case["alpha"], case["centers"])
    op = dage.Coulomb3D(g, quad=dage.GaussQuad(qd["nlin"], qd["nlog"], qd["tstart"], qd["tlin"], qd["tlog"]))
    V, E = op.apply(rho, energy=True)
    assert abs(E - case["selfint"]) < 1e-13
    assert abs(dage.integrate(g, rho, V) - E) < 1e-14


def test_device_and_host_pointers_agree(dage, oracle):
    import torch

    g, go = _grids(dage, oracle, -3.6, 6, 0.2)
    rho = oracle.gauss_cube(go, [1.0, -0.3], [1.0, 3.0], [[0, 0, 0], [0.4, 0.2, -0.3]])
    op = dage.Coulomb3D(g, quad=dage.GaussQuad(8, 8))
    Vh, Eh = op.apply(rho, energy=True)
    rd = torch.from_numpy(rho.reshape(-1, order="F").copy()).cuda()
    Vd, Ed = op.apply(rd, energy=True)
    np.testing.assert_array_equal(Vd.cpu().numpy().reshape(-1), Vh.reshape(-1, order="F"))
    assert Ed == Eh
    # accumulate: V += op(rho)
    V2 = op.apply(rd, out=Vd.clone(), accumulate=True)
    ref = 2 * Vd.cpu().numpy().reshape(-1)
    got = V2.cpu().numpy().reshape(-1)
    assert np.abs(got - ref).max() <= 1e-14 * np.abs(ref).max()


def test_helmholtz_matches_oracle(dage, oracle):
    g, go = _grids(dage, oracle, -3.0, 5, 0.2)
    quad = (12, 12, 0.0, 2.0, 1e3)
    rho = oracle.gauss_cube(go, [1.0], [2.0], [[0.1, 0.2, -0.1]])
    cop = dage.Coulomb3D(g, quad=dage.GaussQuad(*quad))
    kappa = 1.3
    E = -0.5 * kappa ** 2
    hop = dage.Helmholtz3D(cop, E)
    V = hop.apply(rho)
    tp, tw = oracle.gauss_quad(*quad)
    T = cop.matrix(0)
    Vo = oracle.transform_cube(T, T, T, oracle.helmholtz_weights(tp, tw, E), rho, oracle.coda_of(1e3))
    assert _relmax(V, Vo) <= 1e-12
    To = oracle.coulomb_matrix(go.axes[0], go.axes[0].points, tp)
    Vr = oracle.transform_cube(To, To, To, oracle.helmholtz_weights(tp, tw, E), rho, oracle.coda_of(1e3))
    assert _relmax(V, Vr) <= TOL_FP64
    # the energy is reset to 0 afterwards (helmholtz3d.F90:479)
    np.testing.assert_allclose(cop.weights, oracle.coulomb_weights(tw), rtol=1e-13)


def test_config1_121_cube(dage, oracle):
    """121^3, 2 seeded Gaussians, 40 t-points on [0, 1e3]: FP64 GPU vs oracle
    (<= 1e-10) and vs the analytic potential."""
    g, go = _grids(dage, oracle, -12.0, 20, 0.2)
    rng = np.random.default_rng(1)
    q = rng.uniform(0.5, 2, 2)
    a = rng.uniform(0.5, 4, 2)
    c = rng.uniform(-3, 3, (2, 3))
    rho = oracle.gauss_cube(go, q, a, c)
    quad = (20, 20, 0.0, 2.0, 1e3)
    op = dage.Coulomb3D(g, quad=dage.GaussQuad(*quad))
    V, E = op.apply(rho, energy=True)
    _check_apply(oracle, op, go, rho, quad, V, E)
    Va = oracle.gauss_pot_cube(go, q, a, c)
    assert _relmax(V, Va) < 1e-3  # discretisation + quadrature error, reported not pinned


def test_invalid_arguments_raise(dage):
    g = dage.Grid3D.cube(-1.2, 2, 0.2)
    with pytest.raises(ValueError):
        dage.Coulomb3D(g, precision="fp8")
    with pytest.raises(dage.DageError):
        dage.Coulomb3D(g, quad=dage.GaussQuad(0, 0))
    with pytest.raises(dage.DageError):
        dage.Coulomb3D(dage.Grid3D.cube(-1.2, 2, 0.2, nlip=9))
    op = dage.Coulomb3D(g, quad=dage.GaussQuad(4, 4))
    with pytest.raises(dage.DageError):
        op.set_transformation_weights(np.ones(3))
    with pytest.raises(ValueError):
        op.apply(np.zeros((3, 3, 3), order="F"))


@pytest.mark.parametrize("prec", ["fp64", "fp16x3"])
def test_pipelined_host_batch_matches_single_applies(dage, oracle, prec):
    """Host cubes through the batched call's copy/compute pipeline: seven
    densities on one operator (both staging slots reused three times), from
    pinned and from pageable memory, equal to one apply each, bit for bit."""
    import torch

    g = dage.Grid3D.cube(-3.6, 6, 0.2)
    go = oracle.Grid3D.cube(-3.6, 6, 0.2)
    op = dage.Coulomb3D(g, quad=dage.GaussQuad(8, 8), precision=prec)
    rng = np.random.default_rng(5)
    rhos = [oracle.gauss_cube(go, rng.uniform(0.5, 2, 2), rng.uniform(0.5, 4, 2),
                              rng.uniform(-1, 1, (2, 3))) for _ in range(7)]
    want = [op.apply(r, energy=True) for r in rhos]
    n = go.shape[0]

    def pinned(a):
        t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
        t.copy_(torch.from_numpy(a.reshape(-1, order="F").copy()))
        return t.numpy().reshape(n, n, n).T

    for host in ("pinned", "pageable"):
        ins = [pinned(r) if host == "pinned" else r for r in rhos]
        outs = [pinned(np.zeros(go.shape, order="F")) if host == "pinned"
                else np.zeros(go.shape, order="F") for _ in rhos]
        E = dage.apply_batched([op] * 7, ins, outs, energy=True)
        for (Vw, Ew), V, e in zip(want, outs, E):
            assert np.array_equal(np.asarray(V), Vw) and e == Ew, host


def test_apply_batched_matches_single_applies(dage, oracle):
    """Several densities through two operators (FP64 and split precision) in
    one batched call, device and host cubes, equal to one apply each."""
    import torch

    g = dage.Grid3D.cube(-3.0, 5, 0.2)
    go = oracle.Grid3D.cube(-3.0, 5, 0.2)
    quad = dage.GaussQuad(6, 6)
    op64 = dage.Coulomb3D(g, quad=quad)
    opmx = dage.Coulomb3D(g, quad=quad, precision="bf16x6")
    rng = np.random.default_rng(11)
    rhos = [oracle.gauss_cube(go, rng.uniform(0.5, 2, 2), rng.uniform(0.5, 4, 2),
                              rng.uniform(-1, 1, (2, 3))) for _ in range(4)]
    ops = [op64, opmx, op64, opmx]
    want = [op.apply(r, energy=True) for op, r in zip(ops, rhos)]
    outs = [np.zeros(go.shape, order="F") for _ in rhos]
    E = dage.apply_batched(ops, rhos, outs, energy=True)
    for (Vw, Ew), V, e in zip(want, outs, E):
        assert np.array_equal(V, Vw) and e == Ew
    drho = [torch.from_numpy(r.reshape(-1, order="F").copy()).cuda() for r in rhos]
    dout = [torch.empty_like(r) for r in drho]
    E2 = dage.apply_batched(ops, drho, dout, energy=True)
    for (Vw, Ew), V, e in zip(want, dout, E2):
        assert np.array_equal(V.cpu().numpy(), Vw.reshape(-1, order="F")) and e == Ew
