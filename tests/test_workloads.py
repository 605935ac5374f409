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


def test_nondegenerate_lp_has_a_strictly_complementary_unique_vertex():
    lp = W.nondegenerate_lp(80, 200, 6, seed=3)
    A = lp.A.to_scipy().tocsr()
    x0, y0, interior, tight = (lp.meta[k] for k in ("x0", "y0", "interior", "tight"))
    ax = A @ x0
    # primal feasibility; tight rows hold with equality, the others with slack >= 0.1
    assert np.all(x0 >= lp.l) and np.all(x0 <= lp.u)
    assert np.allclose(ax[tight], lp.hi[tight], atol=1e-9)
    assert np.all(lp.hi[~tight] - ax[~tight] >= 0.1 - 1e-12)
    eq = np.isfinite(lp.lo)
    assert np.allclose(ax[eq], lp.lo[eq], atol=1e-9)
    # dual: y <= -0.1 on tight <= rows, 0 on slack rows; reduced costs strictly signed at bounds
    assert np.all(y0[~eq & tight] <= -0.1) and np.all(y0[~tight] == 0.0)
    d = lp.c - A.T @ y0
    assert np.allclose(d[interior], 0.0, atol=1e-9)
    at_l = ~interior & (x0 == 0.0)
    at_u = ~interior & (x0 == 10.0)
    assert np.all(d[at_l] >= 0.1 - 1e-9) and np.all(d[at_u] <= -0.1 + 1e-9)
    # square nonsingular basis
    B = A[np.flatnonzero(tight)][:, np.flatnonzero(interior)].toarray()
    assert B.shape[0] == B.shape[1] and np.linalg.matrix_rank(B) == B.shape[0]


def test_diff_batch_is_deterministic_and_conditioned():
    a = W.diff_batch(3, 50, 100, 5, seed=10, max_cond=1e4)
    b = W.diff_batch(3, 50, 100, 5, seed=10, max_cond=1e4)
    for x, y in zip(a, b):
        assert np.array_equal(x.A.val, y.A.val) and np.array_equal(x.c, y.c)
    for lp in a:
        A = lp.A.to_scipy().tocsr()
        B = A[np.flatnonzero(lp.meta["tight"])][:, np.flatnonzero(lp.meta["interior"])].toarray()
        assert np.linalg.cond(B, 1) <= 1e4 * 1.0001


def test_unbounded_lp_has_an_improving_recession_ray():
    lp = W.unbounded_lp(60, 150, 5, seed=2)
    A = lp.A.to_scipy().tocsr()
    d, x0 = lp.meta["ray"], lp.meta["x0"]
    assert np.allclose(A @ d, 0.0) and lp.c @ d < 0
    assert np.all(d[np.isfinite(lp.l)] >= 0) and np.all(d[np.isfinite(lp.u)] == 0)
    ax = A @ x0
    assert np.all(ax <= lp.hi + 1e-9) and np.all(ax[np.isfinite(lp.lo)] >= lp.lo[np.isfinite(lp.lo)] - 1e-9)
