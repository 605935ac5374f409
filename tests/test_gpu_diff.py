"""Differentiable batched LP layer (gb_diff_*).

Three checks, on LPs whose optimum is a nondegenerate vertex
(workloads.nondegenerate_lp), loss L = w.x* + v.y*:

* truncated gradient (implicit completion off) against central differences
  (h = 1e-4, FP64) of the K-step tail map started at the library's own tail
  start point, evaluated by the oracle's plain FP64 PDHG iterations;
* full gradient against basis sensitivities of the reference dual simplex:
  dL/dc = B^-1 v_R on basic columns, dL/db = B^-T w_B on active rows,
  dL/dA = -(dL/db) x^T - y (dL/dc)^T on the pattern;
* full gradient against central differences (h = 1e-4) of the exact
  solution map, re-solved by the dual simplex.

Relative tolerance 1e-4 throughout.  By default the tail starts from the
polished vertex; without polishing the adjoint still gives dL/dc and dL/db of
the vertex, while dL/dA = -(p x^T + y q^T) inherits the PDHG point's error.
The torch.autograd.Function wrapper is checked to return the same gradients.
"""
import numpy as np
import pytest

from ganit_v2_b200 import DiffSolver, Options, Precision, workloads as W
from ganit_v2_b200.lp import Csr

pytestmark = pytest.mark.gpu

SHAPE = (60, 150, 6)
SEEDS = (0, 1, 2)
TOL = 1e-4


@pytest.fixture(scope="module")
def lps():
    return [W.nondegenerate_lp(*SHAPE, seed=s, max_cond=2e4) for s in SEEDS]


@pytest.fixture(scope="module")
def loss(lps):
    rng = np.random.default_rng(7)
    return rng.standard_normal(sum(lp.n for lp in lps)), rng.standard_normal(sum(lp.m for lp in lps))


def _slices(lps):
    n = np.concatenate([[0], np.cumsum([lp.n for lp in lps])])
    m = np.concatenate([[0], np.cumsum([lp.m for lp in lps])])
    z = np.concatenate([[0], np.cumsum([lp.A.nnz for lp in lps])])
    return [(slice(n[i], n[i + 1]), slice(m[i], m[i + 1]), slice(z[i], z[i + 1])) for i in range(len(lps))]


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def _rows(lp):
    return np.repeat(np.arange(lp.m), np.diff(lp.A.ptr))


def _basis(lp, O):
    """Active rows, basic columns, x, y of the optimal vertex (dual simplex when the
    reference build is present, else the generator's construction)."""
    if O.ref_available():
        ds = O.ref_dual_simplex(lp)
        assert ds["status"] == 0
        head = ds["head"]
        basic = np.sort(head[head < lp.n])
        active = np.ones(lp.m, dtype=bool)
        active[head[head >= lp.n] - lp.n] = False
        assert np.array_equal(basic, np.flatnonzero(lp.meta["interior"]))
        return active, basic, ds["x"], ds["y"]
    return lp.meta["tight"], np.flatnonzero(lp.meta["interior"]), lp.meta["x0"], lp.meta["y0"]


def _basis_sensitivities(lp, w, v, O):
    active, basic, x, y = _basis(lp, O)
    A = lp.A.to_scipy().tocsr()
    B = A[np.flatnonzero(active)][:, basic].toarray()
    p = np.zeros(lp.m)
    q = np.zeros(lp.n)
    p[active] = np.linalg.solve(B.T, w[basic])
    q[basic] = np.linalg.solve(B, v[active])
    rows = _rows(lp)
    da = -(p[rows] * x[lp.A.idx] + y[rows] * q[lp.A.idx])
    return q, p, da


def _direction(lp, rng):
    """Random data direction; equality rows move lo and hi together."""
    dc = rng.standard_normal(lp.n)
    db = rng.standard_normal(lp.m)
    dlo = np.where(np.isfinite(lp.lo), db, 0.0)
    dhi = np.where(np.isfinite(lp.hi), db, 0.0)
    da = rng.standard_normal(lp.A.nnz)
    return dc, dlo, dhi, da


def _dot(g, d):
    dc, dlo, dhi, da = d
    return g["c"] @ dc + g["lo"] @ dlo + g["hi"] @ dhi + g["a_val"] @ da


def _perturbed(lp, d, h):
    from ganit_v2_b200.lp import LP

    dc, dlo, dhi, da = d
    lo = np.where(np.isfinite(lp.lo), lp.lo + h * dlo, lp.lo)
    hi = np.where(np.isfinite(lp.hi), lp.hi + h * dhi, lp.hi)
    return LP(Csr(lp.m, lp.n, lp.A.ptr, lp.A.idx, lp.A.val + h * da), lp.c + h * dc, lp.l, lp.u, lo, hi)


@pytest.fixture(scope="module")
def full(lps, loss):
    w, v = loss
    ds = DiffSolver(lps, Options(tol=1e-8, precision=Precision.Double), tail_iters=200, ckpt_every=20,
                    implicit_iters=20000, implicit_tol=1e-12)
    res, x, y = ds.forward(Options(tol=1e-8, precision=Precision.Double))
    g = ds.backward(w, v)
    yield ds, res, x, y, g
    ds.close()


def test_forward_reaches_the_vertex(lps, full):
    ds, res, x, y, _ = full
    for i, (lp, r, (sn, sm, _)) in enumerate(zip(lps, res, _slices(lps))):
        assert r.status_name == "OPTIMAL"
        assert max(r.rel_primal, r.rel_dual, r.rel_gap) <= 1e-8 * 1.0000001
        assert ds.info(i)["polished"] == 1
        assert _rel(x[sn], lp.meta["x0"]) < 1e-9
        assert _rel(y[sm], lp.meta["y0"]) < 1e-9


def test_masks_and_implicit_solve(lps, full):
    ds = full[0]
    for i, lp in enumerate(lps):
        inf = ds.info(i)
        assert inf["tail_iterations"] == 200 and inf["checkpoint_every"] == 20
        assert inf["free_cols"] == int(lp.meta["interior"].sum())
        assert inf["active_rows"] == int(lp.meta["tight"].sum())
        assert inf["implicit_converged"] == 1 and inf["implicit_residual"] <= 1e-12


def test_gradients_match_basis_sensitivities(lps, loss, full, oracle_built):
    w, v = loss
    g = full[4]
    for lp, (sn, sm, sz) in zip(lps, _slices(lps)):
        q, p, da = _basis_sensitivities(lp, w[sn], v[sm], oracle_built)
        assert _rel(g["c"][sn], q) < TOL
        assert _rel(g["lo"][sm] + g["hi"][sm], p) < TOL
        assert _rel(g["a_val"][sz], da) < TOL


def test_gradients_match_central_differences_of_the_solution(lps, loss, full, oracle_built):
    if not oracle_built.ref_available():
        pytest.skip("reference dual simplex not built")
    w, v = loss
    g = full[4]
    rng = np.random.default_rng(11)
    h = 1e-4
    for lp, (sn, sm, sz) in zip(lps, _slices(lps)):
        gi = {"c": g["c"][sn], "lo": g["lo"][sm], "hi": g["hi"][sm], "a_val": g["a_val"][sz]}
        for _ in range(3):
            d = _direction(lp, rng)
            vals = []
            for s in (1.0, -1.0):
                r = oracle_built.ref_dual_simplex(_perturbed(lp, d, s * h))
                assert r["status"] == 0
                vals.append(w[sn] @ r["x"] + v[sm] @ r["y"])
            fd = (vals[0] - vals[1]) / (2 * h)
            assert abs(_dot(gi, d) - fd) <= TOL * max(abs(fd), 1e-8)


def test_adjoint_without_polishing(lps, loss, oracle_built):
    """dL/dc and dL/db depend only on the active set; dL/dA is evaluated at the
    (unpolished) PDHG point, whose distance to the vertex bounds its error."""
    w, v = loss
    opt = Options(tol=1e-8, precision=Precision.Double)
    with DiffSolver(lps, opt, tail_iters=200, ckpt_every=20, implicit_tol=1e-12, polish=False) as ds:
        res, x, _ = ds.forward(opt)
        g = ds.backward(w, v)
        assert all(ds.info(i)["polished"] == 0 for i in range(len(lps)))
    for lp, (sn, sm, sz) in zip(lps, _slices(lps)):
        q, p, da = _basis_sensitivities(lp, w[sn], v[sm], oracle_built)
        assert _rel(g["c"][sn], q) < TOL
        assert _rel(g["lo"][sm] + g["hi"][sm], p) < TOL
        assert _rel(g["a_val"][sz], da) < max(TOL, 20 * _rel(x[sn], lp.meta["x0"]))


def test_truncated_gradient_is_the_derivative_of_the_tail_map(lps, loss, oracle_built):
    """Implicit completion off: the exact gradient of z_0 -> z_K with z_0 fixed."""
    w, v = loss
    K, R = 40, 10
    opt = Options(tol=1e-8, precision=Precision.Double)
    with DiffSolver(lps, opt, tail_iters=K, ckpt_every=R, implicit_iters=0) as ds:
        ds.forward(opt)
        g = ds.backward(w, v)
        x0, y0 = ds.tail_start()
        infos = [ds.info(i) for i in range(len(lps))]
    rng = np.random.default_rng(5)
    h = 1e-4
    for i, (lp, (sn, sm, sz)) in enumerate(zip(lps, _slices(lps))):
        sc = oracle_built.scale(lp)
        R_, C_, bs, cs = sc["R"], sc["C"], sc["bscale"], sc["cscale"]
        rows = _rows(lp)

        def tail_loss(p):
            As = Csr(lp.m, lp.n, lp.A.ptr, lp.A.idx, p.A.val * R_[rows] * C_[lp.A.idx])
            AT = Csr.from_scipy(As.to_scipy().T.tocsr())
            x, y = oracle_built.plain_iterations(As, AT, p.c * C_ / cs, p.l / C_ / bs, p.u / C_ / bs, p.lo * R_ / bs,
                                                 p.hi * R_ / bs, infos[i]["tau"], infos[i]["sigma"], K, x0[sn],
                                                 y0[sm])
            return w[sn] @ (x * C_ * bs) + v[sm] @ (y * R_ * cs)

        gi = {"c": g["c"][sn], "lo": g["lo"][sm], "hi": g["hi"][sm], "a_val": g["a_val"][sz]}
        for _ in range(3):
            d = _direction(lp, rng)
            fd = (tail_loss(_perturbed(lp, d, h)) - tail_loss(_perturbed(lp, d, -h))) / (2 * h)
            assert abs(_dot(gi, d) - fd) <= TOL * max(abs(fd), 1e-8)


def test_torch_layer_matches_diff_solver(lps, loss, full):
    torch = pytest.importorskip("torch")
    from ganit_v2_b200.diff import LPLayer

    w, v = loss
    layer = LPLayer(lps, Options(tol=1e-8, precision=Precision.Double), tail_iters=200, ckpt_every=20,
                    implicit_iters=20000, implicit_tol=1e-12)
    c, lo, hi, a = (t.clone().requires_grad_(True) for t in layer.template_parameters())
    x, y = layer(c, lo, hi, a)
    (torch.from_numpy(w) @ x + torch.from_numpy(v) @ y).backward()
    g = full[4]
    np.testing.assert_allclose(c.grad.numpy(), g["c"], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(lo.grad.numpy(), g["lo"], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(hi.grad.numpy(), g["hi"], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(a.grad.numpy(), g["a_val"], rtol=1e-9, atol=1e-12)
    assert all(r.status_name == "OPTIMAL" for r in layer.last_results)
