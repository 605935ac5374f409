"""The differentiable layer at the size of its benchmark workload: 256
nondegenerate LPs of m=500, n=1000, 10 nonzeros per column
(workloads.diff_batch), mixed precision to 1e-6, K=200 tail iterations
checkpointed every R=20, loss L = w.x* + v.y*.

* every instance is OPTIMAL and FP64-certified at 1e-6, was polished, and its
  implicit completion converged (no instance left with NaN gradients);
* on the first 16 instances the gradients match the basis sensitivities of
  the reference dual simplex's optimal basis (tests/golden/diff_bases.npz,
  written by make_diff_bases.py): dL/dc = B^-1 v_D on the basic columns,
  dL/db = B^-T w_F on the active rows, dL/dA = -(dL/db) x^T - y (dL/dc)^T, to
  1e-4 relative."""
import os

import numpy as np
import pytest

from ganit_v2_b200 import DiffSolver, Options, Precision, workloads as W
from tests.golden.make_golden import lp_digest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-4


@pytest.fixture(scope="module")
def run():
    lps = W.diff_batch(256)
    opt = Options(tol=1e-6, precision=Precision.Mixed)
    ds = DiffSolver(lps, opt, tail_iters=200, ckpt_every=20)
    rng = np.random.default_rng(3)
    w = rng.standard_normal(int(ds.n_off[-1]))
    v = rng.standard_normal(int(ds.m_off[-1]))
    res, x, y = ds.forward(opt)
    g = ds.backward(w, v)
    infos = [ds.info(i) for i in range(len(lps))]
    yield lps, ds, res, g, infos, w, v
    ds.close()


def test_every_instance_certified_polished_and_completed(run):
    lps, ds, res, g, infos, _, _ = run
    bad = [(i, r.status_name, r.rel_primal, r.rel_gap, inf["polished"], inf["implicit_converged"])
           for i, (r, inf) in enumerate(zip(res, infos))
           if not (r.status_name == "OPTIMAL" and max(r.rel_primal, r.rel_dual, r.rel_gap) <= 1e-6 * 1.0000001
                   and inf["polished"] and inf["implicit_converged"])]
    assert not bad, bad[:8]
    for k in ("c", "lo", "hi", "a_val"):
        assert np.all(np.isfinite(g[k])), k


def test_gradients_match_reference_basis_sensitivities(run):
    lps, ds, res, g, infos, w, v = run
    ref = np.load(os.path.join(GOLD, "diff_bases.npz"))
    errs = []
    for i in range(len(ref["heads"])):
        lp = lps[i]
        assert lp_digest(lp) == str(ref["digests"][i])
        head = ref["heads"][i]
        basic = np.sort(head[head < lp.n])
        active = np.ones(lp.m, dtype=bool)
        active[head[head >= lp.n] - lp.n] = False
        x, y = ref["x"][i], ref["y"][i]
        A = lp.A.to_scipy().tocsr()
        B = A[np.flatnonzero(active)][:, basic].toarray()
        n0, n1 = int(ds.n_off[i]), int(ds.n_off[i + 1])
        m0, m1 = int(ds.m_off[i]), int(ds.m_off[i + 1])
        z0, z1 = int(ds.nnz_off[i]), int(ds.nnz_off[i + 1])
        p = np.zeros(lp.m)
        q = np.zeros(lp.n)
        p[active] = np.linalg.solve(B.T, w[n0:n1][basic])
        q[basic] = np.linalg.solve(B, v[m0:m1][active])
        rows = np.repeat(np.arange(lp.m), np.diff(lp.A.ptr))
        da = -(p[rows] * x[lp.A.idx] + y[rows] * q[lp.A.idx])
        rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))  # noqa: E731
        e = (rel(g["c"][n0:n1], q), rel(g["lo"][m0:m1] + g["hi"][m0:m1], p), rel(g["a_val"][z0:z1], da))
        errs.append(e)
        assert abs(res[i].pobj - ref["objective"][i]) <= 1e-6 * (1 + abs(ref["objective"][i]))
    assert max(max(e) for e in errs) <= TOL, errs
