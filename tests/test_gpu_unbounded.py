"""Unboundedness (dual infeasibility) certificate -- an extension: the
reference has no such test and runs to its iteration or time limit on an
unbounded LP (README.md:197).  With Options.detect_unbounded the engine stops
with DUAL_INFEASIBLE when the primal ray x - x_r lowers the objective and
violates its recession conditions by at most infeas_tol relative to that
decrease.  Off (the default) it keeps the reference's behaviour; on, it never
changes a verdict on the reference's own fixtures."""
import json
import os

import pytest

from ganit_v2_b200 import workloads as W
from tests.golden.make_golden import load_lp

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("prec", ["double", "mixed"])
@pytest.mark.parametrize("seed", [2, 3])
def test_unbounded_lp_is_certified(prec, seed):
    import ganit_v2_b200 as gb

    lp = W.unbounded_lp(120, 300, 5, seed=seed)
    P = {"double": gb.Precision.Double, "mixed": gb.Precision.Mixed}[prec]
    r = gb.solve_pdhg_gpu(lp, gb.Options(precision=P, detect_unbounded=True, max_iter=200_000))
    assert r.status_name == "DUAL_INFEASIBLE"


def test_without_detection_the_reference_behaviour_is_kept(oracle_built):
    import ganit_v2_b200 as gb

    lp = W.unbounded_lp(120, 300, 5, seed=2)
    r = gb.solve_pdhg_gpu(lp, gb.Options(precision=gb.Precision.Double, max_iter=4096))
    o = oracle_built.solve(lp, precision="double", max_iter=4096)
    assert r.status_name == o.status == "ITERATION_LIMIT"
    assert r.iterations == o.iterations


def test_detection_changes_no_verdict_on_the_reference_fixtures():
    import ganit_v2_b200 as gb

    gold = json.load(open(os.path.join(GOLD, "golden.json")))
    for name, entry in sorted(gold["synthetic"].items()):
        lp, _ = load_lp(os.path.join(GOLD, name + ".npz"))
        tol = entry["options"].get("tol", 1e-4)
        r = gb.solve_pdhg_gpu(lp, gb.Options(tol=tol, precision=gb.Precision.Double, detect_unbounded=True))
        assert r.status_name == entry["results"]["double"]["status"], name


def test_batch_mixes_unbounded_and_bounded_instances(oracle_built):
    import ganit_v2_b200 as gb

    lps = [W.unbounded_lp(80, 200, 5, seed=5)] + W.lp_batch(4, seed=70, m_min=30, m_max=200) + \
          [W.infeasible_lp(60, 150, seed=3)]
    with gb.BatchSolver(lps) as bs:
        res = bs.solve(gb.Options(precision=gb.Precision.Mixed, detect_unbounded=True, max_iter=200_000))
    assert res[0].status_name == "DUAL_INFEASIBLE"
    for lp, r in zip(lps[1:], res[1:]):
        assert r.status_name == oracle_built.solve(lp, precision="mixed").status
