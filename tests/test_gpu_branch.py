"""Batched strong branching (gb_strong_branch) on the GPU against the
reference's dual simplex (oracle/_ref) solving every child LP exactly, and
against the reference's branching rule (src/mip.cpp:727-783) restated in the
oracle.  The certified child bounds are checked against the EXACT rational
value of the Lagrangian bound at the same duals: never above it (rigour),
and within a few ulps of it."""
from dataclasses import replace

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-7


@pytest.fixture(scope="module")
def gb():
    from ganit_v2_b200 import build

    build.build()
    import ganit_v2_b200 as gb

    return gb


@pytest.fixture(scope="module")
def opt(gb):
    return gb.Options(tol=TOL, precision=gb.Precision.Double)


@pytest.fixture(scope="module")
def node(oracle_built):
    from ganit_v2_b200 import workloads

    if not oracle_built.ref_available():
        pytest.skip("reference dual simplex not built")

    lp = workloads.milp_node(both_blocked=1)
    r = oracle_built.ref_dual_simplex(lp)
    assert r["status"] == 0
    return lp, r["x"], r["objective"]


def _close(a, b, rel):
    return abs(a - b) <= rel * (1.0 + abs(b))


def test_children_match_the_dual_simplex(gb, oracle_built, node, opt):
    lp, x, z = node
    planted = set(np.concatenate([lp.meta["up_blocked"], lp.meta["down_blocked"], lp.meta["both_blocked"]]))
    frac = [j for j in gb.fractional(x, lp.is_int) if j not in planted]
    cands = gb.most_fractional(x, frac, 8)
    assert len(cands) >= 4
    sb = gb.strong_branch(lp, x, cands, z, opt=opt)
    ref = oracle_built.strong_branch_reference(lp, x, cands, z)
    assert sb.children_solved == 2 * len(cands)
    for t in range(len(cands)):
        for d in range(2):
            zr = ref["z"][t, d]
            if np.isinf(zr):
                assert np.isinf(sb.z[t, d]) and sb.status[t, d] == gb.Status.PrimalInfeasible
                continue
            assert sb.status[t, d] == gb.Status.Optimal
            assert _close(sb.z[t, d], zr, 1e-5), (t, d, sb.z[t, d], zr)
            # a certified bound never exceeds the child's optimum, and with
            # accurate duals it is close to it
            assert sb.cert[t, d] <= zr + 1e-12 * (1.0 + abs(zr))
            assert sb.cert[t, d] >= zr - 1e-4 * (1.0 + abs(zr))
    np.testing.assert_allclose(sb.score, ref["score"], rtol=1e-3, atol=1e-9)
    assert sb.action == ref["action"] == gb.BRANCH_VAR
    # the chosen column is the reference's unless the two best scores tie
    top = np.sort(ref["score"])[-2:]
    if top[1] > top[0] * (1 + 1e-3):
        assert sb.var == ref["var"]
    t = list(cands).index(sb.var)
    np.testing.assert_array_equal(sb.est, sb.z[t])
    np.testing.assert_array_equal(sb.cert_choice, sb.cert[t])


def test_certified_bounds_are_exact_lower_bounds(gb, oracle_built, node, opt):
    """The device bound at the duals of each child against the rational value
    of the same bound: the same batch solved through BatchSolver (the engine
    is deterministic) gives those duals."""
    lp, x, z = node
    cands = gb.most_fractional(x, gb.fractional(x, lp.is_int), 6)
    sb = gb.strong_branch(lp, x, cands, z, opt=opt)
    children = []
    for j in cands:
        v = float(x[j])
        for lo, hi in ((lp.l[j], np.floor(v)), (np.ceil(v), lp.u[j])):
            l, u = lp.l.copy(), lp.u.copy()
            l[j], u[j] = lo, hi
            children.append((int(j), lo, hi, replace(lp, l=l, u=u, meta={})))
    res = gb.BatchSolver([c[3] for c in children], opt).solve(opt)
    checked = 0
    for s, (j, lo, hi, child) in enumerate(children):
        t, d = divmod(s, 2)
        assert res[s].status == sb.status[t, d]
        if res[s].status == gb.Status.PrimalInfeasible:
            continue
        exact = oracle_built.lagrangian_bound_exact(lp, res[s].y, j, lo, hi)
        cert = sb.cert[t, d]
        if exact == -np.inf:
            assert cert == -np.inf
            continue
        assert np.isfinite(cert)
        assert cert <= exact, (s, cert, float(exact))
        assert float(exact) - cert <= 1e-12 * (1.0 + abs(float(exact))), (s, cert, float(exact))
        checked += 1
    assert checked >= 6


def test_infeasible_sides_decide_like_select_branch(gb, oracle_built, node, opt):
    lp, x, z = node
    regular = gb.most_fractional(x, [j for j in gb.fractional(x, lp.is_int) if j < 120], 3)
    up = int(lp.meta["up_blocked"][0])
    down = int(lp.meta["down_blocked"][0])
    both = int(lp.meta["both_blocked"][0])
    # up child infeasible: keep the down side, x_j <= floor(x_j)
    sb = gb.strong_branch(lp, x, np.r_[regular, up], z, opt=opt)
    assert (sb.action, sb.var, sb.lo, sb.hi) == (gb.BRANCH_TIGHTEN, up, lp.l[up], np.floor(x[up]))
    assert np.isinf(sb.z[-1, 1]) and sb.status[-1, 1] == gb.Status.PrimalInfeasible
    assert np.isfinite(sb.z[-1, 0])
    # down child infeasible: keep the up side
    sb = gb.strong_branch(lp, x, [down, up], z, opt=opt)
    assert (sb.action, sb.var, sb.lo, sb.hi) == (gb.BRANCH_TIGHTEN, down, np.ceil(x[down]), lp.u[down])
    # both infeasible: the node is
    sb = gb.strong_branch(lp, x, np.r_[regular, both], z, opt=opt)
    assert (sb.action, sb.var) == (gb.BRANCH_NODE_INFEASIBLE, both)
    for c in ([*regular, up], [down, up], [*regular, both]):
        ref = oracle_built.strong_branch_reference(lp, x, c, z)
        got = gb.strong_branch(lp, x, c, z, opt=opt)
        assert (got.action, got.var) == (ref["action"], ref["var"])


def test_crossing_bounds_need_no_solve(gb, node, opt):
    """A child whose branched bounds cross is infeasible without a solve."""
    lp, x, z = node
    j = int(gb.most_fractional(x, gb.fractional(x, lp.is_int), 1)[0])
    l = lp.l.copy()
    l[j] = np.floor(x[j]) + 0.25 if x[j] - np.floor(x[j]) > 0.25 else np.floor(x[j])
    lp2 = replace(lp, l=l, meta={})
    sb = gb.strong_branch(lp2, x, [j], z, opt=opt)
    if l[j] > np.floor(x[j]):
        assert sb.children_solved == 1
        assert sb.status[0, 0] == gb.Status.PrimalInfeasible and sb.iterations[0, 0] == 0
        assert (sb.action, sb.lo, sb.hi) == (gb.BRANCH_TIGHTEN, np.ceil(x[j]), lp.u[j])


def test_cutoff_prunes_like_the_reference(gb, oracle_built, node, opt):
    """A finite cutoff between the children's optima: a child is pruned
    (z = +inf) exactly where the reference's rule prunes it -- its optimum
    reaches the cutoff (the dual simplex returns Cutoff, src/mip.cpp:755) --
    and the decision is the oracle's."""
    lp, x, z = node
    planted = set(np.concatenate([lp.meta["up_blocked"], lp.meta["down_blocked"], lp.meta["both_blocked"]]))
    cands = gb.most_fractional(x, [j for j in gb.fractional(x, lp.is_int) if j not in planted], 6)
    free = oracle_built.strong_branch_reference(lp, x, cands, z)
    finite = np.sort(free["z"][np.isfinite(free["z"])])
    # a cutoff halfway between two distinct optima, so no child sits within the tolerance of it
    gaps = np.diff(finite)
    i = int(np.argmax(gaps[len(gaps) // 4:])) + len(gaps) // 4
    cutoff = float(0.5 * (finite[i] + finite[i + 1]))
    assert gaps[i] > 1e-4 * (1 + abs(cutoff))
    ref = oracle_built.strong_branch_reference(lp, x, cands, z, cutoff=cutoff)
    cut = gb.strong_branch(lp, x, cands, z, cutoff=cutoff, opt=opt)
    pruned = np.isinf(ref["z"]) & np.isfinite(free["z"])
    assert pruned.any()
    np.testing.assert_array_equal(np.isinf(cut.z), np.isinf(ref["z"]))
    fin = np.isfinite(ref["z"])
    np.testing.assert_allclose(cut.z[fin], ref["z"][fin], rtol=1e-5, atol=1e-5)
    assert cut.action == ref["action"]
    if ref["action"] != gb.BRANCH_VAR:
        assert cut.var == ref["var"]


def test_maximisation_is_branched_in_minimisation_form(gb, oracle_built, node, opt):
    lp, x, z = node
    mx = replace(lp, c=-lp.c, maximize=True, meta=lp.meta)
    cands = gb.most_fractional(x, [j for j in gb.fractional(x, lp.is_int) if j < 120], 4)
    a = gb.strong_branch(lp, x, cands, z, opt=opt)
    b = gb.strong_branch(mx, x, cands, z, opt=opt)
    np.testing.assert_array_equal(a.z, b.z)
    np.testing.assert_array_equal(a.cert, b.cert)
    assert (a.action, a.var) == (b.action, b.var)
