"""Seeded workload generators: shapes, feasibility by construction, and the
sizes the benchmark configurations are quoted at."""
import numpy as np
import pytest

from ganit_v2_b200 import workloads as W


def test_random_feasible_lp_is_feasible_by_construction():
    lp = W.random_feasible_lp(300, 700, 6, seed=4)
    x0 = lp.meta["x0"]
    ax = lp.A.to_scipy() @ x0
    assert np.all(ax >= lp.lo - 1e-9) and np.all(ax <= lp.hi + 1e-9)
    assert np.all(x0 >= lp.l) and np.all(x0 <= lp.u)
    cols = np.diff(lp.A.transpose().ptr)
    assert np.all(cols == 6)  # distinct rows per column
    assert np.sum(np.isfinite(lp.lo)) == 150


def test_random_lp_is_deterministic():
    a = W.random_feasible_lp(100, 250, 4, seed=9)
    b = W.random_feasible_lp(100, 250, 4, seed=9)
    assert np.array_equal(a.A.val, b.A.val) and np.array_equal(a.c, b.c)


@pytest.mark.slow
def test_blending_sizes_match_the_quoted_configuration():
    lp = W.blending_lp()  # 60 crudes, 16 products, 5 specs, 365 periods
    assert (lp.m, lp.n, lp.A.nnz) == (57305, 405880, 2886344)


def test_blending_small_structure():
    lp = W.blending_lp(4, 3, 2, 5, seed=2)
    assert lp.m == (1 + 4 + 3 + 6) * 5 and lp.n == (4 * (2 + 3) + 2 * 3) * 5
    assert np.all(lp.l == 0) and np.all(lp.u > 0)


def test_portfolio_forms_agree_on_objective():
    dp = W.portfolio_qp(200, 4, seed=3)
    li = W.portfolio_qp(200, 4, seed=3, lifted=True)
    x = np.full(200, 1.0 / 200)
    f = dp.F.T @ x
    xl = np.concatenate([x, f])
    assert abs(dp.objective(x) - li.objective(xl)) < 1e-12


def test_batch_sizes():
    lps = W.lp_batch(16, seed=100)
    ms = [lp.m for lp in lps]
    assert all(50 <= m <= 4000 for m in ms)
    assert all(lp.n == round(2.5 * lp.m) for lp in lps)
    k = np.diff(lps[0].A.transpose().ptr)
    assert k.min() >= 4 and k.max() <= 12


def test_infeasible_lp_has_contradicting_rows():
    lp = W.infeasible_lp(50, 120, seed=1)
    A = lp.A.to_scipy()
    r1, r2 = A.getrow(lp.m - 2).toarray(), A.getrow(lp.m - 1).toarray()
    assert np.array_equal(r1, r2)
    assert lp.hi[-2] < lp.lo[-1]
