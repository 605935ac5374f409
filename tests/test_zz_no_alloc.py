"""gb_eval_kkt_noalloc: the KKT check for callers that cannot allocate device
memory (a worker with a fixed device-memory budget, or a latency-critical path
where cudaMalloc/cudaFree would synchronise the device).  The caller owns every
buffer; the library's scratch is a fixed __device__ array.

Checked through the C ABI, on two calls in a row, against the oracle's FP64 KKT
(ora_eval_kkt: pdhg_impl.hpp:92-109 over the reductions of backend_cpu.cpp,
sums in index order) and against the KKT the existing Backend entry points
compute for the same point (gb_spmv_A/AT, gb_primal_res2, gb_dual_res,
gb_row_dual_obj, gb_dot_c -- the steps of pdhg_evaluate, pdhg_impl.hpp:202-230),
within the 1e-10 relative tolerance of FP64 sums taken in different orders.
Two problems: a small one of short rows, and one with rows and columns long
enough to take the scratch's chunk slots and arrival counters (more than 4096
nonzeros) and whole-CTA rows (1025..4096 nonzeros) in both A and A^T.  This
file is collected last on purpose."""
import ctypes as C
import math
import os

import numpy as np
import pytest

from tests.golden.make_golden import load_lp

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _backend_kkt(be, x, y, sc):
    dx, dy = be.from_host(x), be.from_host(y)
    ax, aty = be.zeros(be.m), be.zeros(be.n)
    be.spmv_A(dx, ax)
    rp2 = be.primal_res2(ax)
    be.spmv_AT(dy, aty)
    rd2, vobj = be.dual_res(aty, None, True)
    robj = be.row_dual_obj(dy)
    pobj = be.dot_c(dx) * sc["obj_scale"] + sc["obj_const"]
    dobj = (robj + vobj) * sc["obj_scale"] + sc["obj_const"]
    rel_p = math.sqrt(rp2) / (1.0 + sc["bnorm"])
    rel_d = math.sqrt(rd2) / (1.0 + sc["cnorm"])
    rel_gap = abs(pobj - dobj) / (1.0 + abs(pobj) + abs(dobj))
    return dict(pobj=pobj, dobj=dobj, rel_p=rel_p, rel_d=rel_d, rel_gap=rel_gap,
                err=math.sqrt(rel_p * rel_p + rel_d * rel_d + rel_gap * rel_gap))


def _long_row_lp():
    """m = 5000, n = 6000 with ~5 random nonzeros per column, plus row 0
    (5000 nonzeros: chunk slots), row 1 (2000: one CTA), column 0 (4500:
    chunk slots of A^T) and column 1 (1500: one CTA of A^T); mixed finite and
    infinite bounds."""
    import scipy.sparse as sp

    from ganit_v2_b200.lp import LP, Csr

    rng = np.random.default_rng(17)
    m, n = 5000, 6000
    rows = [rng.integers(0, m, size=5 * n)]
    cols = [np.repeat(np.arange(n), 5)]
    rows += [np.zeros(5000, dtype=np.int64), np.ones(2000, dtype=np.int64)]
    cols += [rng.choice(n, 5000, replace=False), rng.choice(n, 2000, replace=False)]
    rows += [rng.choice(m, 4500, replace=False), rng.choice(m, 1500, replace=False)]
    cols += [np.zeros(4500, dtype=np.int64), np.ones(1500, dtype=np.int64)]
    r, c = np.concatenate(rows), np.concatenate(cols)
    A = sp.coo_matrix((rng.standard_normal(r.size), (r, c)), shape=(m, n)).tocsr()
    A.sum_duplicates()
    A = Csr.from_scipy(A)
    lo = np.where(rng.random(m) < 0.5, rng.standard_normal(m), -np.inf)
    hi = np.where(rng.random(m) < 0.5, lo + rng.random(m), np.inf)
    hi = np.where(np.isfinite(lo) | np.isfinite(hi), hi, 1.0)
    l = np.where(rng.random(n) < 0.7, 0.0, -np.inf)
    u = np.where(rng.random(n) < 0.6, 5.0, np.inf)
    return LP(A, rng.standard_normal(n), l, u, lo, hi, name="long_rows")


@pytest.mark.parametrize("problem", ["rand_free", "long_rows"])
def test_noalloc_kkt_matches_oracle_and_backend_entry_points(oracle_built, problem):
    import torch

    import ganit_v2_b200 as gb
    from ganit_v2_b200 import api
    from ganit_v2_b200.lp import Csr

    lib = api.load_library()
    lp = _long_row_lp() if problem == "long_rows" else load_lp(os.path.join(GOLD, problem + ".npz"))[0]
    s = oracle_built.scale(lp)
    A = Csr(lp.m, lp.n, lp.A.ptr, lp.A.idx, s["a_val"])
    AT = A.transpose()
    if problem == "long_rows":  # the rows the scratch's chunk slots and counters serve exist on both sides
        assert np.diff(A.ptr).max() > 4096 and np.diff(AT.ptr).max() > 4096
        assert np.any((np.diff(A.ptr) > 1024) & (np.diff(A.ptr) <= 4096))
        assert np.any((np.diff(AT.ptr) > 1024) & (np.diff(AT.ptr) <= 4096))
    scaled = dict(A=A, AT=AT, c=s["c"], l=s["l"], u=s["u"], lo=s["lo"], hi=s["hi"], Rres=s["Rres"], Cres=s["Cres"])
    sc = dict(obj_scale=s["cscale"] * s["bscale"], obj_const=s["obj_const"], bnorm=s["bnorm"], cnorm=s["cnorm"])
    be = gb.Backend(scaled, "f64", "f64")

    dev = torch.device("cuda:0")
    keep = []

    def d(a, dt=torch.float64):
        t = torch.as_tensor(np.ascontiguousarray(a)).to(dev, dtype=dt)
        keep.append(t)
        return t.data_ptr()

    g = api._GbScaledLp(lp.m, lp.n, d(A.ptr, torch.int32), d(A.idx, torch.int32), d(A.val), d(AT.ptr, torch.int32),
                        d(AT.idx, torch.int32), d(AT.val), None, None, None, d(s["c"]), d(s["l"]), d(s["u"]),
                        d(s["lo"]), d(s["hi"]), d(s["Rres"]), d(s["Cres"]))
    hp = np.ascontiguousarray(A.ptr, dtype=np.int32)
    htp = np.ascontiguousarray(AT.ptr, dtype=np.int32)
    scal = api.GbKktScalars(sc["obj_scale"], sc["obj_const"], sc["bnorm"], sc["cnorm"])
    stream = torch.cuda.Stream()
    rng = np.random.default_rng(5)
    for call in range(2):  # two calls in a row share the scratch array
        x = rng.standard_normal(lp.n) * (call + 1)
        y = rng.standard_normal(lp.m) * (call + 1)
        xd, yd = torch.as_tensor(x).to(dev), torch.as_tensor(y).to(dev)
        torch.cuda.synchronize()
        out = api.GbKkt()
        rc = lib.gb_eval_kkt_noalloc(C.addressof(g), hp.ctypes.data, htp.ctypes.data, xd.data_ptr(), yd.data_ptr(),
                                     C.addressof(scal), stream.cuda_stream, C.addressof(out))
        assert rc == 0, lib.gb_last_error()
        ora = oracle_built.eval_kkt(A, AT, s["c"], s["l"], s["u"], s["lo"], s["hi"], s["Rres"], s["Cres"], x, y,
                                    **sc)
        for k, v in ora.items():
            assert getattr(out, k) == pytest.approx(v, rel=1e-10, abs=1e-14), (problem, call, k, "oracle")
        want = _backend_kkt(be, x, y, sc)
        for k, v in want.items():
            assert getattr(out, k) == pytest.approx(v, rel=1e-10, abs=1e-14), (problem, call, k, "backend")


def test_noalloc_rejects_oversized_problems():
    import torch

    from ganit_v2_b200 import api

    lib = api.load_library()
    m, n = 4_200_000, 1  # 4.2M empty rows -> more than GB_NOALLOC_MAX_BLOCKS row blocks
    hp = np.zeros(m + 1, dtype=np.int32)
    htp = np.zeros(n + 1, dtype=np.int32)
    buf = torch.zeros(16, dtype=torch.float64, device="cuda:0")
    p = buf.data_ptr()
    g = api._GbScaledLp(m, n, *([p] * 6), None, None, None, *([p] * 7))
    scal = api.GbKktScalars(1.0, 0.0, 0.0, 0.0)
    out = api.GbKkt()
    rc = lib.gb_eval_kkt_noalloc(C.addressof(g), hp.ctypes.data, htp.ctypes.data, p, p, C.addressof(scal), None,
                                 C.addressof(out))
    assert rc == -1
    assert b"too large" in lib.gb_last_error()
