"""gb_eval_kkt_noalloc: the KKT check for callers that cannot allocate device
memory (a worker with a fixed device-memory budget, or a latency-critical path
where cudaMalloc/cudaFree would synchronise the device).  The caller owns every
buffer; the library's scratch is a fixed __device__ array.

Checked through the C ABI against the KKT the existing Backend entry points
compute for the same point (gb_spmv_A/AT, gb_primal_res2, gb_dual_res,
gb_row_dual_obj, gb_dot_c -- the steps of pdhg_evaluate, pdhg_impl.hpp:202-230),
on two calls in a row, within the 1e-10 relative tolerance of FP64 sums taken
in different orders.  This file is collected last on purpose."""
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


def test_noalloc_kkt_matches_backend_entry_points(oracle_built):
    import torch

    import ganit_v2_b200 as gb
    from ganit_v2_b200 import api
    from ganit_v2_b200.lp import Csr

    lib = api.load_library()
    lp, _ = load_lp(os.path.join(GOLD, "rand_free.npz"))
    s = oracle_built.scale(lp)
    A = Csr(lp.m, lp.n, lp.A.ptr, lp.A.idx, s["a_val"])
    AT = A.transpose()
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
        want = _backend_kkt(be, x, y, sc)
        for k, v in want.items():
            assert getattr(out, k) == pytest.approx(v, rel=1e-10, abs=1e-14), (call, k)


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
