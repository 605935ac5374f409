"""Factor-model rewrite (gb_factor_detect / gb_factor_expand, host code, no GPU):
a lifted factor-model QP becomes the engine's diagonal-plus-low-rank form."""
import os

import numpy as np
import pytest

from ganit_v2_b200 import workloads as W

from oracle.oracle import REF_INSTANCES as REF_ROOT, REF_MISSING  # noqa: E402


@pytest.fixture(scope="module")
def gb():
    from ganit_v2_b200 import build

    build.build()
    import ganit_v2_b200 as gb

    return gb


def test_lifted_portfolio_recovers_the_factor_form(gb):
    lifted = W.portfolio_qp(300, 8, seed=5, lifted=True)
    direct = W.portfolio_qp(300, 8, seed=5)
    ff = gb.FactorForm(lifted)
    red = ff.lp
    assert ff.factors == 8 and (red.m, red.n) == (1, 300)
    np.testing.assert_allclose(red.F @ red.F.T, direct.F @ direct.F.T, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(red.D, direct.D, rtol=1e-15)
    np.testing.assert_allclose(red.c, direct.c, rtol=1e-15)
    np.testing.assert_array_equal(red.A.to_scipy().toarray(), np.ones((1, 300)))
    assert red.Q is None and red.obj_const == 0.0


def test_expand_restores_factors_and_row_duals(gb):
    lifted = W.portfolio_qp(200, 5, seed=6, lifted=True)
    ff = gb.FactorForm(lifted)
    rng = np.random.default_rng(0)
    x = rng.random(ff.lp.n)
    y = rng.standard_normal(ff.lp.m)
    xf, yf = ff.expand(x, y)
    A = lifted.A.to_scipy().tocsr()
    np.testing.assert_allclose(xf[:200], x)
    f = xf[200:]
    np.testing.assert_allclose(A[1:] @ xf, 0.0, atol=1e-12)          # f - F'x = 0 holds
    q = lifted.Q.to_scipy().diagonal()[200:]
    np.testing.assert_allclose(yf[1:], q * f)                         # stationarity of f: q f - y = 0
    assert yf[0] == y[0]


@pytest.mark.parametrize("name", ["port_tiny.mps", "port_small.mps"])
def test_reference_portfolio_files_are_detected(gb, name):
    path = os.path.join(REF_ROOT, "qp", name)
    if not os.path.exists(path):
        pytest.skip(REF_MISSING)
    lp = gb.read_mps(path)
    ff = gb.FactorForm(lp)
    assert ff.factors > 0 and ff.lp.n == lp.n - ff.factors and ff.lp.m == lp.m - ff.factors


def test_problems_without_the_structure_are_rejected(gb):
    from ganit_v2_b200.lp import Csr

    lp = W.random_feasible_lp(30, 60, 4, seed=1)
    with pytest.raises(gb.GanitError, match="no CSR Hessian"):
        gb.FactorForm(lp)
    lifted = W.portfolio_qp(50, 3, seed=2, lifted=True)
    Q = lifted.Q.to_scipy().tolil()
    Q[0, 1] = Q[1, 0] = 0.1
    lifted.Q = Csr.from_scipy(Q.tocsr())
    with pytest.raises(gb.GanitError, match="not diagonal"):
        gb.FactorForm(lifted)
