"""Warm start (gb_problem_set_start / gb_batch_set_start), an extension: the
reference's PDHG always starts from the projection of 0.  Started from its
own solution a solve certifies within a few checks and returns the same
point; instances without a start are bit-identical to a cold solve; the
default start comes back when the start is dropped."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gb():
    from ganit_v2_b200 import build

    build.build()
    import ganit_v2_b200 as gb

    return gb


def test_problem_started_at_its_solution(gb):
    from ganit_v2_b200 import workloads

    lp = workloads.random_feasible_lp(300, 700, seed=5)
    opt = gb.Options(tol=1e-6, precision=gb.Precision.Double)
    P = gb.Problem(lp, opt)
    cold = P.solve(opt)
    assert cold.status == gb.Status.Optimal
    P.set_start(cold.x, cold.y)
    warm = P.solve(opt)
    assert warm.status == gb.Status.Optimal
    assert warm.iterations <= max(2 * opt.check_every, cold.iterations // 4)
    assert abs(warm.pobj - cold.pobj) <= 1e-5 * (1 + abs(cold.pobj))
    # x outside the bounds is projected: the start is still accepted
    P.set_start(cold.x + 10.0, cold.y)
    assert P.solve(opt).status == gb.Status.Optimal
    P.set_start()  # back to the default start: the cold run again, bit for bit
    again = P.solve(opt)
    assert again.iterations == cold.iterations
    np.testing.assert_array_equal(again.x, cold.x)
    with pytest.raises(gb.GanitError, match="infinite"):
        P.set_start(np.full(lp.n, np.inf), None)


def test_batch_start_touches_only_its_instance(gb):
    from ganit_v2_b200 import workloads

    lps = [workloads.random_feasible_lp(200 + 50 * k, 500 + 80 * k, seed=40 + k) for k in range(4)]
    opt = gb.Options(tol=1e-6, precision=gb.Precision.Mixed)
    B = gb.BatchSolver(lps, opt)
    cold = B.solve(opt)
    B.set_start(2, cold[2].x, cold[2].y)
    warm = B.solve(opt)
    for k in (0, 1, 3):
        assert warm[k].iterations == cold[k].iterations
        np.testing.assert_array_equal(warm[k].x, cold[k].x)
        np.testing.assert_array_equal(warm[k].y, cold[k].y)
    assert warm[2].status == gb.Status.Optimal and warm[2].iterations < cold[2].iterations
    # a primal-only start (NULL y) is allowed
    B.clear_start()
    B.set_start(1, cold[1].x, None)
    assert B.solve(opt)[1].status == gb.Status.Optimal
    B.clear_start()
    again = B.solve(opt)
    assert [r.iterations for r in again] == [r.iterations for r in cold]


def test_strong_branching_from_the_node_point(gb, oracle_built):
    """Children started from the node's (x, y) reach the same child values as
    cold children, in fewer iterations."""
    from ganit_v2_b200 import workloads

    if not oracle_built.ref_available():
        pytest.skip("reference dual simplex not built")
    lp = workloads.milp_node(n=400, knapsacks=20, up_blocked=0, down_blocked=0, seed=12)
    r = oracle_built.ref_dual_simplex(lp)
    x, y, z = r["x"], r["y"], r["objective"]
    cands = gb.most_fractional(x, gb.fractional(x, lp.is_int), 8)
    opt = gb.Options(tol=1e-7, precision=gb.Precision.Double)
    cold = gb.strong_branch(lp, x, cands, z, opt=opt)
    warm = gb.strong_branch(lp, x, cands, z, opt=opt, y=y)
    ref = oracle_built.strong_branch_reference(lp, x, cands, z)
    fin = np.isfinite(ref["z"])
    assert (np.isfinite(warm.z) == fin).all()
    np.testing.assert_allclose(warm.z[fin], ref["z"][fin], rtol=1e-5, atol=1e-5)
    assert (warm.cert[fin] <= ref["z"][fin] + 1e-12 * (1 + np.abs(ref["z"][fin]))).all()
    assert warm.iterations.sum() < cold.iterations.sum()
