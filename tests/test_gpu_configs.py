"""Parity at the benchmark configurations' full sizes, against the reference
CPU PDHG run on the same seeded data (tests/golden/configs.json, written by
make_configs.py; each workload's digest is checked first, so the data here is
the data the reference solved).

* blending LP, 60 x 16 x 5 x 365 (m 57,305, n 405,880, nnz 2,886,344):
  double and mixed -- same verdict, certified, objective within 10 * tol,
  iterations within two checks at double and at mixed;
* the 512-LP batch, every instance (double: verdict, objective, iterations
  within two checks; mixed: verdict and objective);
* the 100,000 x 50 portfolio QP through the diagonal-plus-low-rank kernel
  against the reference solving the lifted form (solution level: the
  trajectories differ); its budget row (100,000 nonzeros) runs through the
  SpMV's chunked long-row path;
* the SpMV pair on rows of 4,097 and 20,000 nonzeros (chunked) and of 1,500
  (one CTA per row) against NumPy."""
import json
import os

import numpy as np
import pytest

from ganit_v2_b200 import workloads as W
from tests.golden.make_golden import lp_digest
from tests.test_gpu_solve import check_against

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
with open(os.path.join(GOLD, "configs.json")) as f:
    CONFIGS = json.load(f)


@pytest.fixture(scope="module")
def gb():
    import ganit_v2_b200 as gb

    gb.load_library()
    return gb


@pytest.mark.parametrize("prec", ["double", "mixed"])
def test_blending_lp_full_size(gb, prec):
    lp = W.blending_lp()
    ref = CONFIGS["blending"]
    assert lp_digest(lp) == ref["digest"]
    P = {"double": gb.Precision.Double, "mixed": gb.Precision.Mixed}[prec]
    r = gb.solve_pdhg_gpu(lp, gb.Options(precision=P))
    g = ref["results"][prec]
    check_against(r, g, 1e-4, prec)
    assert abs(r.iterations - g["iterations"]) <= 128, (r.iterations, g["iterations"])


@pytest.fixture(scope="module")
def batch512():
    lps = W.lp_batch(512, seed=1000)
    ref = CONFIGS["batch512"]["instances"]
    assert len(ref) == len(lps)
    for lp, g in zip(lps, ref):
        assert lp_digest(lp) == g["digest"], lp.name
    return lps, ref


@pytest.mark.parametrize("prec", ["double", "mixed"])
def test_batch512_every_instance(gb, batch512, prec):
    lps, ref = batch512
    P = {"double": gb.Precision.Double, "mixed": gb.Precision.Mixed}[prec]
    with gb.BatchSolver(lps, gb.Options(precision=P)) as bs:
        res = bs.solve(gb.Options(precision=P))
    bad = []
    for i, (r, g) in enumerate(zip(res, ref)):
        ok = r.status_name == g["status"]
        if ok and g["status"] == "OPTIMAL":
            ok = max(r.rel_primal, r.rel_dual, r.rel_gap) <= 1e-4 * 1.0000001
            # objective within 10 tol of the reference's, relative to |pobj| -- and, where c'x is a
            # cancellation of much larger terms, to tol times their size: a relative KKT of 1e-4
            # fixes the objective only to about that (instance 170: terms sum to 2874 for an
            # objective of 1.007; the reference itself gives 1.0055 at 1e-4 and 1.0067 at 1e-9)
            scale = 10 * 1e-4 * (1 + abs(g["pobj"])) + 1e-4 * float(np.sum(np.abs(lps[i].c * r.x)))
            ok = ok and abs(r.pobj - g["pobj"]) <= scale
        if ok and prec == "double":
            ok = abs(r.iterations - g["iterations"]) <= 128
        if not ok:
            bad.append((i, r.status_name, g["status"], r.pobj, g["pobj"], r.iterations, g["iterations"]))
    assert not bad, bad[:10]


@pytest.mark.parametrize("prec", ["double", "mixed"])
def test_portfolio_qp_full_size(gb, prec):
    lp = W.portfolio_qp(100_000, 50, seed=7)
    ref = CONFIGS["portfolio"]
    assert lp_digest(W.portfolio_qp(100_000, 50, seed=7, lifted=True)) == ref["digest"]
    P = {"double": gb.Precision.Double, "mixed": gb.Precision.Mixed}[prec]
    r = gb.solve_pdhg_gpu(lp, gb.Options(precision=P))
    g = ref["results"]["double"]
    assert r.status_name == g["status"] == "OPTIMAL"
    assert max(r.rel_primal, r.rel_dual, r.rel_gap) <= 1e-4 * 1.0000001
    assert abs(r.pobj - g["pobj"]) <= 1e-3 * (1 + abs(g["pobj"])), (r.pobj, g["pobj"])
    x = r.x
    assert abs(x.sum() - 1.0) <= 1e-3 and x.min() >= 0.0 and x.max() <= 0.05
    obj = x @ (lp.F @ (lp.F.T @ x)) + x @ (lp.D * x) + lp.c @ x
    assert abs(obj - r.pobj) <= 1e-6 * (1 + abs(obj))


def _long_row_matrix():
    """400 x 30,000: rows 0 / 1 / 2 with 20,000 / 4,097 / 1,500 nonzeros, the
    rest 3..12; column 7 with 350 nonzeros."""
    import scipy.sparse as sp

    rng = np.random.default_rng(3)
    m, n = 400, 30_000
    R, C = [], []
    for i, k in enumerate([20_000, 4_097, 1_500]):
        R.append(np.full(k, i))
        C.append(rng.choice(n, k, replace=False))
    for i in range(3, m):
        k = int(rng.integers(3, 13))
        R.append(np.full(k, i))
        C.append(rng.choice(n, k, replace=False))
    R.append(np.arange(3, 353))
    C.append(np.full(350, 7))
    r, c = np.concatenate(R), np.concatenate(C)
    A = sp.coo_matrix((rng.standard_normal(r.size), (r, c)), shape=(m, n)).tocsr()
    A.sum_duplicates()
    return A


@pytest.mark.parametrize("mat,vec", [("f64", "f64"), ("f32", "f32")])
def test_spmv_long_rows(gb, mat, vec):
    from ganit_v2_b200.lp import Csr

    As = _long_row_matrix()
    A = Csr.from_scipy(As)
    lens = np.diff(A.ptr)
    assert lens.max() == 20_000 and (lens == 4_097).any() and (lens == 1_500).any()
    m, n = A.rows, A.cols
    one_n, one_m = np.ones(n), np.ones(m)
    scaled = dict(A=A, AT=A.transpose(), c=one_n, l=-one_n, u=one_n, lo=-one_m, hi=one_m, Rres=one_m, Cres=one_n)
    be = gb.Backend(scaled, mat, vec)
    rng = np.random.default_rng(9)
    x, y = rng.standard_normal(n), rng.standard_normal(m)
    Am = As.copy()
    if vec == "f32":
        x = x.astype(np.float32).astype(np.float64)
        y = y.astype(np.float32).astype(np.float64)
    if mat == "f32":
        Am.data = Am.data.astype(np.float32).astype(np.float64)
    rt = 1e-13 if vec == "f64" else 2e-6
    ax, aty = be.zeros(m), be.zeros(n)
    for _ in range(2):  # twice: the chunk counters re-arm themselves
        be.spmv_A(be.from_host(x), ax)
        be.spmv_AT(be.from_host(y), aty)
        scale_a = float(np.max(abs(Am) @ np.abs(x)))
        scale_t = float(np.max(abs(Am.T) @ np.abs(y)))
        np.testing.assert_allclose(ax.to_host(), Am @ x, rtol=rt, atol=rt * scale_a)
        np.testing.assert_allclose(aty.to_host(), Am.T @ y, rtol=rt, atol=rt * scale_t)
