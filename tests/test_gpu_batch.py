"""Batched solving (gb_batch_*): every instance of a batch behaves as if solved
alone -- same verdict as the reference CPU PDHG (the oracle), FP64-certified
KKT within tol, objective within 10 * tol, and at FP64 the per-instance
iteration count within two checks of the oracle's."""
import os

import numpy as np
import pytest

from ganit_v2_b200 import workloads as W
from tests.golden.make_golden import load_lp

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def mixed_batch():
    lps = W.lp_batch(10, seed=500, m_min=30, m_max=400)
    for name in ("rand_small", "infeasible", "rand_max", "rand_free", "blend_small"):
        lps.append(load_lp(os.path.join(GOLD, name + ".npz"))[0])
    return lps


@pytest.fixture(scope="module")
def batch():
    return mixed_batch()


@pytest.mark.parametrize("prec", ["double", "mixed"])
def test_batch_matches_oracle_per_instance(batch, oracle_built, prec):
    import ganit_v2_b200 as gb

    P = {"double": gb.Precision.Double, "mixed": gb.Precision.Mixed}[prec]
    with gb.BatchSolver(batch) as bs:
        res = bs.solve(gb.Options(precision=P))
        for i, (lp, r) in enumerate(zip(batch, res)):
            o = oracle_built.solve(lp, precision=prec)
            assert r.status_name == o.status, (i, lp.name)
            if o.status == "OPTIMAL":
                assert max(r.rel_primal, r.rel_dual, r.rel_gap) <= 1e-4 * 1.0000001, (i, lp.name)
                assert abs(r.pobj - o.pobj) <= 1e-3 * (1 + abs(o.pobj)), (i, lp.name, r.pobj, o.pobj)
            if prec == "double":
                assert abs(r.iterations - o.iterations) <= 128, (i, lp.name, r.iterations, o.iterations)
            x, y = r.x, r.y
            assert x.shape == (lp.n,) and y.shape == (lp.m,) and np.all(np.isfinite(x))


def test_batch_instance_equals_single_solve(batch):
    """An instance inside a batch follows the same trajectory as alone."""
    import ganit_v2_b200 as gb

    with gb.BatchSolver(batch) as bs:
        res = bs.solve(gb.Options(precision=gb.Precision.Double))
    for i in (0, 3, len(batch) - 1):
        single = gb.solve_pdhg_gpu(batch[i], gb.Options(precision=gb.Precision.Double))
        assert single.status == res[i].status
        assert abs(single.iterations - res[i].iterations) <= 64
        assert abs(single.pobj - res[i].pobj) <= 1e-6 * (1 + abs(single.pobj))


def test_batch_schedule_report(batch):
    import ganit_v2_b200 as gb

    with gb.BatchSolver(batch[:4]) as bs:
        s = bs.schedule()
    assert s["threads"] == 256 and s["blocks_per_sm"] >= 1
    assert len(s["groups_A"]) == 4 and all(g in (1, 2, 4, 8, 16, 32) for g in s["groups_A"])


def test_autotuned_schedules_keep_every_result(batch):
    """The autotuner only re-cuts row blocks: verdicts stay those of the oracle,
    every result stays certified, and the tuned iteration is not slower."""
    import ganit_v2_b200 as gb

    opt = gb.Options(precision=gb.Precision.Mixed)
    with gb.BatchSolver(batch) as bs:
        before = bs.solve(opt)
        t = bs.autotune(iters=10)
        assert all(256 <= b <= 2048 for b in t["block_nnz"].tolist() + t["block_nnz_f64"].tolist())
        assert set(t["max_rows"].tolist()) <= {256, 128, 64, 32}
        assert t["ms_per_iter_tuned"] <= 1.05 * t["ms_per_iter_default"]
        assert t["ms_per_iter_tuned_f64"] <= 1.05 * t["ms_per_iter_default_f64"]
        after = bs.solve(opt)
        for i, (a, b) in enumerate(zip(before, after)):
            assert a.status == b.status, i
            if b.status_name == "OPTIMAL":
                assert max(b.rel_primal, b.rel_dual, b.rel_gap) <= 1e-4 * 1.0000001
                assert abs(a.pobj - b.pobj) <= 1e-3 * (1 + abs(a.pobj))
        k = bs.time_kernels(0, 20)
        assert k["ms_primal"] > 0 and k["ms_dual"] > 0 and k["bytes_per_iter"] > 0


def test_batch_with_bf16_phase_certifies_every_instance(batch, oracle_built):
    import ganit_v2_b200 as gb

    with gb.BatchSolver(batch) as bs:
        res = bs.solve(gb.Options(precision=gb.Precision.MixedBf16))
        for i, (lp, r) in enumerate(zip(batch, res)):
            o = oracle_built.solve(lp, precision="mixed")
            assert r.status_name == o.status, (i, lp.name)
            if o.status == "OPTIMAL":
                assert max(r.rel_primal, r.rel_dual, r.rel_gap) <= 1e-4 * 1.0000001
                assert abs(r.pobj - o.pobj) <= 1e-3 * (1 + abs(o.pobj))
        k = bs.time_kernels(3, 10)
        assert k["ms_primal"] > 0 and k["bytes_per_iter"] > 0


def test_streamed_batch_is_bit_identical_to_a_cached_one():
    """A batch whose FP32 iteration exceeds the L2 (the 512-LP batch, 207 MB)
    runs the iteration kernels' variant that streams idx / val without L1
    allocation; its first 48 instances, batched alone (well inside the L2),
    run the default loads.  Loads change nothing but caching, and instances
    of a batch never share a row block or a reduction, so every instance
    gives the same bits either way."""
    import ganit_v2_b200 as gb

    lps = W.lp_batch(512, seed=1000)
    opt = gb.Options(precision=gb.Precision.Mixed)
    with gb.BatchSolver(lps, opt) as bs:
        big = bs.solve(opt)
    with gb.BatchSolver(lps[:48], opt) as bs:
        small = bs.solve(opt)
    assert all(r.status_name == "OPTIMAL" for r in big)
    for i in range(48):
        assert big[i].iterations == small[i].iterations, i
        np.testing.assert_array_equal(big[i].x, small[i].x)
        np.testing.assert_array_equal(big[i].y, small[i].y)
