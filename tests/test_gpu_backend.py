"""Backend-concept operations (gb_backend_* / gb_vec_*) against NumPy on the
scaled problem the oracle produces (src/scaling.cpp:36-155).

FP64 elementwise steps are bit-exact (the library is built without FMA
contraction, as the reference's scalar loops are); FP64 SpMV agrees to
1e-13 relative; FP32 levels to single-precision rounding; reductions are
FP64 and agree to 1e-12 relative."""
import os

import numpy as np
import pytest

from tests.golden.make_golden import load_lp

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def scaled(oracle_built):
    lp, _ = load_lp(os.path.join(GOLD, "rand_free.npz"))
    s = oracle_built.scale(lp)
    from ganit_v2_b200.lp import Csr

    A = Csr(lp.m, lp.n, lp.A.ptr, lp.A.idx, s["a_val"])
    return dict(A=A, AT=A.transpose(), c=s["c"], l=s["l"], u=s["u"], lo=s["lo"], hi=s["hi"], Rres=s["Rres"],
                Cres=s["Cres"])


@pytest.mark.parametrize("mat,vec", [("f64", "f64"), ("f32", "f64"), ("f32", "f32")])
def test_backend_ops(scaled, mat, vec):
    import ganit_v2_b200 as gb

    be = gb.Backend(scaled, mat, vec)
    rng = np.random.default_rng(0)
    A = scaled["A"].to_scipy()
    m, n = A.shape
    x = rng.standard_normal(n)
    y = rng.standard_normal(m)
    if vec == "f32":
        x = x.astype(np.float32).astype(np.float64)
        y = y.astype(np.float32).astype(np.float64)
    Am = A.copy()
    if mat == "f32":
        Am.data = Am.data.astype(np.float32).astype(np.float64)
    rt = 1e-13 if vec == "f64" else 2e-6
    dx, dy = be.from_host(x), be.from_host(y)
    ax, aty = be.zeros(m), be.zeros(n)
    be.spmv_A(dx, ax)
    be.spmv_AT(dy, aty)
    np.testing.assert_allclose(ax.to_host(), Am @ x, rtol=rt, atol=rt * float(np.max(np.abs(Am) @ np.abs(x))))
    np.testing.assert_allclose(aty.to_host(), Am.T @ y, rtol=rt, atol=rt * float(np.max(np.abs(Am.T) @ np.abs(y))))

    # primal / dual step (backend_cpu.cpp:67-92)
    aty_h = aty.to_host()
    tau, sigma = 0.37, 1.9
    xn, xbar, sumx = be.zeros(n), be.zeros(n), be.from_host(np.ones(n))
    be.primal_step(dx, aty, None, tau, xn, xbar, sumx)
    c, l, u = scaled["c"], scaled["l"], scaled["u"]
    if vec == "f32":
        f = np.float32
        v = (x.astype(f) - f(tau) * (c.astype(f) - aty_h.astype(f) + f(0))).astype(f)
        v = np.minimum(np.maximum(v, l.astype(f)), u.astype(f))
        np.testing.assert_array_equal(xn.to_host(), v.astype(np.float64))
    else:
        v = np.minimum(np.maximum(x - tau * (c - aty_h + 0.0), l), u)
        np.testing.assert_array_equal(xn.to_host(), v)
        np.testing.assert_array_equal(xbar.to_host(), 2.0 * v - x)
        np.testing.assert_array_equal(sumx.to_host(), 1.0 + v)
    yn, sumy = be.zeros(m), be.zeros(m)
    be.dual_step(dy, ax, sigma, yn, sumy)
    if vec == "f64":
        q = y - sigma * ax.to_host()
        t = np.minimum(np.maximum(-q, sigma * scaled["lo"]), sigma * scaled["hi"])
        np.testing.assert_array_equal(yn.to_host(), q + t)
        np.testing.assert_array_equal(sumy.to_host(), q + t)

    # reductions (backend_cpu.cpp:101-155), FP64 accumulation
    axh = ax.to_host()
    lo, hi = scaled["lo"], scaled["hi"]
    cast = (lambda a: a.astype(np.float32).astype(np.float64)) if vec == "f32" else (lambda a: a)
    p = np.minimum(np.maximum(axh, cast(lo)), cast(hi))
    want = np.sum(((axh - p) / cast(scaled["Rres"])) ** 2)
    assert be.primal_res2(ax) == pytest.approx(want, rel=1e-12)
    rd2, vobj = be.dual_res(aty, None, True)
    z = cast(c) - aty_h
    lf, uf = np.isfinite(cast(l)), np.isfinite(cast(u))
    r = np.where(z > 0, np.where(lf, 0, z), np.where(z < 0, np.where(uf, 0, z), 0)) / cast(scaled["Cres"])
    ob = np.where((z > 0) & lf, z * cast(l), 0) + np.where((z < 0) & uf, z * cast(u), 0)
    assert rd2 == pytest.approx(np.sum(r * r), rel=1e-12, abs=1e-300)
    assert vobj == pytest.approx(np.sum(np.where(np.isfinite(ob), ob, 0)), rel=1e-12)
    rdo = np.sum(np.where((y > 0) & np.isfinite(lo), y * cast(lo), np.where((y < 0) & np.isfinite(hi), y * cast(hi), 0)))
    assert be.row_dual_obj(dy) == pytest.approx(rdo, rel=1e-12)
    assert be.dot(dx, dx) == pytest.approx(float(x @ x), rel=1e-12)
    assert be.dot_c(dx) == pytest.approx(float(cast(c) @ x), rel=1e-12)
    assert be.diff2(dx, xn) == pytest.approx(float(np.sum((x - xn.to_host()) ** 2)), rel=1e-12)
    d = be.zeros(n)
    be.sub(dx, xn, d)
    be.scale_into(d, 0.5, d)
    np.testing.assert_allclose(d.to_host(), cast(0.5 * (x - xn.to_host())), rtol=1e-6 if vec == "f32" else 0)
    be.fill(d, 3.0)
    assert np.all(d.to_host() == 3.0)
    be.copy(dx, d)
    np.testing.assert_array_equal(d.to_host(), x)
