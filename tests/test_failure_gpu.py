"""Failure detection without a GPU fault: the tensor-core kernel's bounded
mbarrier waits are made to run out (a 1-cycle budget), the apply reports
DAGE_E_TIMEOUT, and the context stays usable for the next call."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_wait_timeout_reports_and_recovers(dage, oracle):
    lib = dage.load()
    g = dage.Grid3D.cube(-2.4, 4, 0.2)
    go = oracle.Grid3D.cube(-2.4, 4, 0.2)
    rho = oracle.gauss_cube(go, [1.0], [2.0], [[0.1, 0.0, -0.1]])
    op = dage.Coulomb3D(g, quad=dage.GaussQuad(2, 2), precision="bf16x3")
    V_ok = op.apply(rho)
    try:
        assert lib.dage_set_wait_limit(1) == 0
        with pytest.raises(dage.DageError) as ei:
            op.apply(rho)
        assert ei.value.code == -5
    finally:
        assert lib.dage_set_wait_limit(2_000_000_000) == 0
    np.testing.assert_array_equal(op.apply(rho), V_ok)


def test_bad_arguments_are_errors_not_crashes(dage):
    g = dage.Grid3D.cube(-1.2, 2, 0.2)
    op = dage.Coulomb3D(g, quad=dage.GaussQuad(2, 2))
    lib = dage.load()
    assert lib.dage_op3d_apply(op._h, None, None, 0, None) == -1
    assert lib.dage_gbfmm_create(g.c(), 7, 12, None, 0, None) == -1
