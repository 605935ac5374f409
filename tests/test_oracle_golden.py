"""The C oracle reproduces the reference's own results (golden fixtures made by
tests/golden/make_golden.py from ganit::solve_pdhg_cpu at OMP_NUM_THREADS=1).

The restatement is single-threaded and FMA-free, so it must agree with the
reference bit for bit: same status, iteration and restart counts, and the
same solution vectors."""
import json
import os

import numpy as np
import pytest

from tests.golden.make_golden import PRECISIONS, instance_path, load_lp, lp_digest

GOLD = os.path.join(os.path.dirname(__file__), "golden")
with open(os.path.join(GOLD, "golden.json")) as f:
    GOLDEN = json.load(f)


@pytest.mark.parametrize("inst", sorted(GOLDEN["reference_instances"]))
def test_instance_fixture_is_the_reference_reader_output(inst):
    """tests/golden/instances/*.npz hold exactly what the reference's MPS
    reader (src/mps.cpp) parsed from its instance files: the digest recorded
    when the reference solved them."""
    lp, _ = load_lp(instance_path(inst))
    assert lp_digest(lp) == GOLDEN["reference_instances"][inst]["digest"]


@pytest.mark.parametrize("name", sorted(GOLDEN["synthetic"]))
@pytest.mark.parametrize("prec", PRECISIONS)
def test_oracle_matches_reference_fixture(oracle_built, name, prec):
    O = oracle_built
    lp, arr = load_lp(os.path.join(GOLD, name + ".npz"))
    entry = GOLDEN["synthetic"][name]
    assert lp_digest(lp) == entry["digest"]
    g = entry["results"][prec]
    r = O.solve(lp, precision=prec, **entry["options"])
    assert r.status == g["status"]
    assert r.iterations == g["iterations"]
    assert r.fp32_iterations == g["fp32_iterations"]
    assert r.l2_iterations == g["l2_iterations"]
    assert r.restarts == g["restarts"]
    for k in ("pobj", "dobj", "rel_p", "rel_d", "rel_gap"):
        assert getattr(r, k) == g[k], k
    np.testing.assert_array_equal(r.x, arr[f"x_{prec}"])
    np.testing.assert_array_equal(r.y, arr[f"y_{prec}"])


from oracle.oracle import REF_INSTANCES as REF_ROOT, REF_MISSING  # noqa: E402


@pytest.mark.skipif(not os.path.isdir(REF_ROOT), reason=REF_MISSING)
@pytest.mark.parametrize("inst", sorted(GOLDEN["reference_instances"]))
def test_oracle_on_reference_instances(oracle_built, inst):
    O = oracle_built
    entry = GOLDEN["reference_instances"][inst]
    if entry["results"]["double"]["iterations"] > 1_000_000:
        pytest.skip("millions of iterations (minutes on one core): the fixture itself is the reference's result")
    if not O.ref_available():
        O.build(ref=True)
    lp = O.ref_read_mps(os.path.join(REF_ROOT, inst + ".mps"))
    assert lp_digest(lp) == entry["digest"]
    for prec, g in entry["results"].items():
        r = O.solve(lp, precision=prec)
        assert (r.status, r.iterations, r.restarts) == (g["status"], g["iterations"], g["restarts"])
        assert r.pobj == g["pobj"] and r.dobj == g["dobj"]
        assert float(np.sum(r.x)) == g["x_sum"]


def test_published_verdicts_pinned():
    """Published reference numbers: bgetam is PRIMAL_INFEASIBLE after 4736
    iterations (results.csv:2) and afiro's objective is -464.78 (README.md:83)."""
    ri = GOLDEN["reference_instances"]
    assert ri["bgetam"]["results"]["double"]["status"] == "PRIMAL_INFEASIBLE"
    assert ri["bgetam"]["results"]["double"]["iterations"] == 4736
    assert abs(ri["afiro"]["results"]["double"]["pobj"] + 464.7853) / 464.7853 < 1e-4
    # port_tiny: README.md:98 reports -0.1370938992 at a tighter tolerance; at 1e-4 agreement is 1e-4 relative
    assert abs(ri["qp/port_tiny"]["results"]["double"]["pobj"] + 0.1370938992) / 0.137 < 1e-4


def test_oracle_scaling_matches_its_own_solver(oracle_built):
    """ora_scale exposes the scaled problem (scaling.cpp:36-155) used by the
    solver; sanity: Ruiz + PC leave every row/col inf-norm near 1."""
    O = oracle_built
    lp, _ = load_lp(os.path.join(GOLD, "rand_small.npz"))
    s = O.scale(lp)
    A = lp.A.to_scipy().copy()
    A.data = s["a_val"]
    rmax = abs(A).max(axis=1).toarray().ravel()
    assert np.all(rmax > 0.05) and np.all(rmax < 20)
    assert s["norm_a"] > 0 and s["bscale"] > 1 and s["cscale"] > 1
