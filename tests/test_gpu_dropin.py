"""Drop-in check of the Backend boundary: the reference's own, unmodified
run_pdhg (src/pdhg_impl.hpp) instantiated with B200Backend<M,V>
(include/ganit_b200_backend.hpp) instead of CudaBackend, driving the B200
kernels through the gb_backend_* C ABI.  Built by oracle/Makefile (target
dropin) from the reference sources; it ships with the repository's built
files.

Same driver, same scaling, same decisions: the FP64 trajectory matches the
reference CPU run (same verdict, iterations within one check), mixed precision
within the solution-level bar of tests/test_gpu_solve.py."""
import json
import os

import pytest

from tests.golden.make_golden import load_lp

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
with open(os.path.join(GOLD, "golden.json")) as f:
    GOLDEN = json.load(f)

CASES = ["rand_small", "rand_free", "infeasible", "blend_small", "port_lifted_small", "rand_max", "rand_cfg0"]


@pytest.fixture(scope="module")
def dropin():
    from oracle import oracle as O

    if not O.dropin_available():
        pytest.skip("oracle/_ref/libganit_dropin.so not built (needs the reference sources at build time)")
    return O


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("prec", ["double", "mixed"])
def test_reference_driver_on_b200_backend(dropin, name, prec):
    lp, _ = load_lp(os.path.join(GOLD, name + ".npz"))
    entry = GOLDEN["synthetic"][name]
    g = entry["results"][prec]
    tol = entry["options"].get("tol", 1e-4)
    r = dropin.dropin_solve(lp, precision=prec, **entry["options"])
    assert r.status == g["status"]
    if g["status"] == "OPTIMAL":
        assert max(r.rel_p, r.rel_d, r.rel_gap) <= tol * 1.0000001
        assert abs(r.pobj - g["pobj"]) <= 10 * tol * (1 + abs(g["pobj"]))
    if prec == "double":
        assert abs(r.iterations - g["iterations"]) <= 64
