"""Strong branching host logic (no GPU): argument checks of gb_strong_branch
(all made before any device work), the candidate helpers against the
reference's rules (Mip::fractional, src/mip.cpp:256-263; the expert order of
src/mip.cpp:709-714), and the oracle's restatement of the branching rule on
the planted MILP node (dual simplex children, src/mip.cpp:727-783)."""
from dataclasses import replace

import numpy as np
import pytest


@pytest.fixture(scope="module")
def gb():
    from ganit_v2_b200 import build

    build.build()
    import ganit_v2_b200 as gb

    return gb


@pytest.fixture(scope="module")
def simplex(oracle_built):
    if not oracle_built.ref_available():
        pytest.skip("reference dual simplex not built")
    return oracle_built


@pytest.fixture(scope="module")
def node():
    from ganit_v2_b200 import workloads

    return workloads.milp_node(both_blocked=1)


def test_fractional_follows_the_reference_rule(gb):
    x = np.array([0.0, 0.5, 1.0000001, 2.9999999, 3.2, -0.5, 7.0, 0.999999])
    is_int = np.array([1, 1, 1, 1, 1, 1, 0, 1], dtype=bool)
    expect = [j for j in range(len(x)) if is_int[j] and 1e-6 < x[j] - np.floor(x[j]) < 1 - 1e-6]
    np.testing.assert_array_equal(gb.fractional(x, is_int), expect)
    # most fractional first, stable among equals
    np.testing.assert_array_equal(gb.most_fractional(x, [1, 4, 5, 7], 3), [1, 5, 4])


@pytest.mark.parametrize("case,msg", [
    ("integral", "integral"),
    ("range", "out of range"),
    ("nan_cutoff", "NaN"),
    ("inf_x", "not finite"),
])
def test_arguments_are_checked_before_device_work(gb, node, case, msg):
    lp = node
    x = np.full(lp.n, 0.5)
    cand, cutoff = [0], np.inf
    if case == "integral":
        x[0] = 1.0
    elif case == "range":
        cand = [lp.n]
    elif case == "nan_cutoff":
        cutoff = np.nan
    elif case == "inf_x":
        x[0] = np.inf
    with pytest.raises(gb.GanitError, match=msg) as e:
        gb.strong_branch(lp, x, cand, 0.0, cutoff=cutoff)
    assert e.value.code == -1


def test_hessian_is_unsupported(gb, node):
    lp = node
    F = np.ones((lp.n, 1))
    qp = replace(lp, F=F, D=np.ones(lp.n), meta={})
    with pytest.raises(gb.GanitError) as e:
        gb.strong_branch(qp, np.full(lp.n, 0.5), [0], 0.0)
    assert e.value.code == -5


def test_planted_node_structure(simplex, node):
    """The generator plants what the GPU tests rely on: fractional knapsack
    columns whose children are feasible, columns with an infeasible up child,
    an infeasible down child, or both."""
    lp = node
    r = simplex.ref_dual_simplex(lp)
    assert r["status"] == 0
    x, z = r["x"], r["objective"]
    up, down, both = (int(lp.meta[k][0]) for k in ("up_blocked", "down_blocked", "both_blocked"))
    np.testing.assert_allclose(x[[up, down, both]], [0.6, 0.4, 0.6], atol=1e-9)
    frac = [j for j in range(120) if 1e-6 < x[j] - np.floor(x[j]) < 1 - 1e-6]
    assert len(frac) >= 4
    ref = simplex.strong_branch_reference(lp, x, frac, z)
    assert ref["action"] == 0 and np.isfinite(ref["z"]).all()
    assert (ref["z"] >= z - 1e-9).all()  # children never beat their parent
    ref = simplex.strong_branch_reference(lp, x, [frac[0], up], z)
    assert (ref["action"], ref["var"], ref["lo"], ref["hi"]) == (-1, up, 0.0, 0.0)
    ref = simplex.strong_branch_reference(lp, x, [down], z)
    assert (ref["action"], ref["var"], ref["lo"], ref["hi"]) == (-1, down, 1.0, 1.0)
    ref = simplex.strong_branch_reference(lp, x, [both], z)
    assert (ref["action"], ref["var"]) == (-2, both)


def test_exact_bound_at_the_simplex_duals_is_the_optimum(simplex, node):
    """With the dual simplex's optimal duals the Lagrangian bound of a child
    equals the child's optimum (strong duality), exactly up to the simplex's
    own rounding -- a check of the oracle's bound restatement."""
    lp = node
    x = simplex.ref_dual_simplex(lp)["x"]
    j = [j for j in range(120) if 1e-6 < x[j] - np.floor(x[j]) < 1 - 1e-6][0]
    for lo, hi in ((lp.l[j], np.floor(x[j])), (np.ceil(x[j]), lp.u[j])):
        l, u = lp.l.copy(), lp.u.copy()
        l[j], u[j] = lo, hi
        r = simplex.ref_dual_simplex(replace(lp, l=l, u=u, meta={}))
        b = simplex.lagrangian_bound_exact(lp, r["y"], j, lo, hi)
        assert abs(float(b) - r["objective"]) <= 1e-9 * (1 + abs(r["objective"]))


@pytest.mark.parametrize("name", ["p0548", "lseu", "egout", "bell5"])
def test_oracle_rule_matches_the_reference_loop_on_mip_files(simplex, gb, name):
    """The oracle's restatement of the strong-branching loop (cold dual simplex
    per child) against the reference's own loop (src/mip.cpp:738-760: warm
    dual simplex from the node basis, here without an iteration limit) on the
    LP relaxations of the reference's MIP instance files: the same child
    optimum on every side, the same infeasible sides."""
    import os

    from oracle.oracle import REF_INSTANCES, REF_MISSING

    path = os.path.join(REF_INSTANCES, "mip", f"{name}.mps")
    if not os.path.exists(path):
        pytest.skip(REF_MISSING)
    lp = gb.read_mps(path)
    assert lp.is_int is not None and not lp.maximize
    root = simplex.ref_dual_simplex(lp)
    assert root["status"] == 0
    x, z = root["x"], root["objective"]
    cands = gb.most_fractional(x, gb.fractional(x, lp.is_int), 6)
    if len(cands) == 0:
        pytest.skip("integral relaxation")
    mine = simplex.strong_branch_reference(lp, x, cands, z)
    ref = simplex.ref_strong_branch(lp, x, cands, iter_limit=-1)
    assert abs(ref["z_node"] - z) <= 1e-9 * (1 + abs(z))
    inf_mine, inf_ref = ~np.isfinite(mine["z"]), ~np.isfinite(ref["z"])
    np.testing.assert_array_equal(inf_mine, inf_ref)
    fin = ~inf_mine
    np.testing.assert_allclose(mine["z"][fin], ref["z"][fin], rtol=1e-9, atol=1e-9)
