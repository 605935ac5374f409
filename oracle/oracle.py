"""ctypes bindings of the CPU checkers -- TEST INFRASTRUCTURE ONLY.

* ``liboracle.so``: the plain-C restatement of GANIT's restarted PDHG
  (pdhg_oracle.c / pdhg_phase.inc; reference src/pdhg_impl.hpp,
  src/backend_cpu.cpp, src/scaling.cpp).
* ``_ref/libganit_ref.so``: the reference's own CPU implementation compiled
  from its sources (see Makefile) behind ref_shim.cpp.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference
legs import this module.  The product package never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libganit_ref.so")
# Checkout of the reference project (its src/ and instances/): only the
# checker builds and the tests that read the reference's instance files use
# it; GANIT_REF_ROOT overrides the default location.
REF_ROOT = os.environ.get("GANIT_REF_ROOT", "/root/reference")
REF_INSTANCES = os.path.join(REF_ROOT, "instances")
REF_MISSING = f"reference checkout not found at {REF_ROOT} (set GANIT_REF_ROOT)"
DROPIN_SO = os.path.join(HERE, "_ref", "libganit_dropin.so")

STATUS = {0: "OPTIMAL", 1: "PRIMAL_INFEASIBLE", 2: "ITERATION_LIMIT", 3: "TIME_LIMIT", 4: "NUMERICAL_ERROR"}
PRECISION = {"double": 0, "mixed": 1, "dynamic": 2}


class _Lp(C.Structure):
    _fields_ = [("m", C.c_int), ("n", C.c_int), ("a_ptr", C.c_void_p), ("a_idx", C.c_void_p),
                ("a_val", C.c_void_p), ("c", C.c_void_p), ("l", C.c_void_p), ("u", C.c_void_p),
                ("lo", C.c_void_p), ("hi", C.c_void_p), ("obj_const", C.c_double), ("maximize", C.c_int),
                ("q_ptr", C.c_void_p), ("q_idx", C.c_void_p), ("q_val", C.c_void_p)]


class _Opt(C.Structure):
    _fields_ = [("tol", C.c_double), ("max_iter", C.c_long), ("time_limit", C.c_double),
                ("check_every", C.c_int), ("ruiz_iters", C.c_int), ("pock_chambolle", C.c_int),
                ("infeas_tol", C.c_double), ("precision", C.c_int), ("stall_checks", C.c_int),
                ("stall_checks_l2", C.c_int)]


class _OraRes(C.Structure):
    _fields_ = [("status", C.c_int), ("pobj", C.c_double), ("dobj", C.c_double), ("rel_p", C.c_double),
                ("rel_d", C.c_double), ("rel_gap", C.c_double), ("iterations", C.c_long),
                ("fp32_iterations", C.c_long), ("l2_iterations", C.c_long), ("restarts", C.c_int),
                ("setup_s", C.c_double), ("solve_s", C.c_double), ("norm_a", C.c_double),
                ("w_final", C.c_double)]


class _RefRes(C.Structure):
    _fields_ = [("status", C.c_int), ("pobj", C.c_double), ("dobj", C.c_double), ("rel_p", C.c_double),
                ("rel_d", C.c_double), ("rel_gap", C.c_double), ("iterations", C.c_long),
                ("fp32_iterations", C.c_long), ("l2_iterations", C.c_long), ("restarts", C.c_int),
                ("setup_s", C.c_double), ("solve_s", C.c_double)]


@dataclass
class OracleResult:
    status: str
    pobj: float
    dobj: float
    rel_p: float
    rel_d: float
    rel_gap: float
    iterations: int
    fp32_iterations: int
    l2_iterations: int
    restarts: int
    setup_s: float
    solve_s: float
    x: np.ndarray
    y: np.ndarray
    norm_a: float = float("nan")


def build(ref: bool = True) -> None:
    """Compile the checkers with oracle/Makefile (the reference build only
    when its sources are present on this machine)."""
    targets = ["oracle"]
    if ref and os.path.isdir(os.path.join(REF_ROOT, "src")):
        targets.append("ref")
        lib = os.path.join(os.path.dirname(HERE), "ganit_v2_b200", "libganit_b200.so")
        if os.path.exists(lib):
            targets.append("dropin")
        targets.append("refcuda")
    subprocess.run(["make", "-s", "-C", HERE, f"REF={REF_ROOT}"] + targets, check=True)


_libs: dict = {}


def _load(path: str):
    if path not in _libs:
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run `make -C oracle`)")
        _libs[path] = C.CDLL(path)
    return _libs[path]


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def _p(a):
    return None if a is None else a.ctypes.data


def _options(precision="double", tol=1e-4, max_iter=10_000_000, time_limit=3600.0, check_every=64,
             ruiz_iters=10, pock_chambolle=True, infeas_tol=1e-8, stall_checks=12, stall_checks_l2=24):
    return _Opt(tol, max_iter, time_limit, check_every, ruiz_iters, int(pock_chambolle), infeas_tol,
                PRECISION[precision] if isinstance(precision, str) else int(precision), stall_checks,
                stall_checks_l2)


def _arrays(lp):
    if lp.F is not None:
        raise ValueError("the oracle takes the reference's CSR Hessian; use the lifted QP form")
    arrs = dict(ptr=lp.A.ptr, idx=lp.A.idx, val=lp.A.val, c=lp.c, l=lp.l, u=lp.u, lo=lp.lo, hi=lp.hi)
    if lp.Q is not None and lp.Q.nnz:
        arrs.update(qptr=lp.Q.ptr, qidx=lp.Q.idx, qval=lp.Q.val)
    else:
        arrs.update(qptr=None, qidx=None, qval=None)
    return arrs


def solve(lp, **opts) -> OracleResult:
    """Run the C restatement (single thread)."""
    lib = _load(ORACLE_SO)
    a = _arrays(lp)
    s = _Lp(lp.m, lp.n, _p(a["ptr"]), _p(a["idx"]), _p(a["val"]), _p(a["c"]), _p(a["l"]), _p(a["u"]),
            _p(a["lo"]), _p(a["hi"]), float(lp.obj_const), int(lp.maximize), _p(a["qptr"]), _p(a["qidx"]),
            _p(a["qval"]))
    o = _options(**opts)
    r = _OraRes()
    x = np.zeros(lp.n)
    y = np.zeros(lp.m)
    lib.ora_solve_pdhg.restype = C.c_int
    lib.ora_solve_pdhg.argtypes = [C.c_void_p] * 5
    rc = lib.ora_solve_pdhg(C.byref(s), C.byref(o), C.byref(r), _p(x), _p(y))
    if rc != 0:
        raise RuntimeError(f"ora_solve_pdhg failed ({rc})")
    return OracleResult(STATUS[r.status], r.pobj, r.dobj, r.rel_p, r.rel_d, r.rel_gap, r.iterations,
                        r.fp32_iterations, r.l2_iterations, r.restarts, r.setup_s, r.solve_s, x, y, r.norm_a)


def scale(lp, ruiz_iters=10, pock_chambolle=True) -> dict:
    """Scaled data of src/scaling.cpp:36-155 (see ora_scale)."""
    lib = _load(ORACLE_SO)
    a = _arrays(lp)
    s = _Lp(lp.m, lp.n, _p(a["ptr"]), _p(a["idx"]), _p(a["val"]), _p(a["c"]), _p(a["l"]), _p(a["u"]),
            _p(a["lo"]), _p(a["hi"]), float(lp.obj_const), int(lp.maximize), _p(a["qptr"]), _p(a["qidx"]),
            _p(a["qval"]))
    m, n = lp.m, lp.n
    out = {k: np.zeros(n) for k in ("c", "l", "u", "C", "Cres")}
    out.update({k: np.zeros(m) for k in ("lo", "hi", "R", "Rres")})
    out["a_val"] = np.zeros(lp.A.nnz)
    scal = np.zeros(7)
    lib.ora_scale.restype = C.c_int
    lib.ora_scale.argtypes = [C.c_void_p, C.c_int, C.c_int] + [C.c_void_p] * 11
    rc = lib.ora_scale(C.byref(s), int(ruiz_iters), int(pock_chambolle), _p(out["a_val"]), _p(out["c"]),
                       _p(out["l"]), _p(out["u"]), _p(out["lo"]), _p(out["hi"]), _p(out["R"]), _p(out["C"]),
                       _p(out["Rres"]), _p(out["Cres"]), _p(scal))
    if rc != 0:
        raise RuntimeError("ora_scale failed")
    for i, k in enumerate(("bscale", "cscale", "norm_a", "norm_q", "bnorm", "cnorm", "obj_const")):
        out[k] = float(scal[i])
    return out


def plain_iterations(A, AT, c, l, u, lo, hi, tau, sigma, iters, x0, y0):
    """FP64 PDHG iterations with fixed steps and no restarts (ora_plain_iterations)."""
    lib = _load(ORACLE_SO)
    x = np.array(x0, dtype=np.float64, copy=True)
    y = np.array(y0, dtype=np.float64, copy=True)
    f = lib.ora_plain_iterations
    f.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 6 + [C.c_void_p] * 5 + [C.c_double, C.c_double, C.c_long,
                                                                           C.c_void_p, C.c_void_p]
    arr = [np.ascontiguousarray(v, dtype=np.float64) for v in (c, l, u, lo, hi)]
    f(A.rows, A.cols, _p(A.ptr), _p(A.idx), _p(A.val), _p(AT.ptr), _p(AT.idx), _p(AT.val),
      *[_p(v) for v in arr], float(tau), float(sigma), int(iters), _p(x), _p(y))
    return x, y


def eval_kkt(A, AT, c, l, u, lo, hi, rres, cres, x, y, obj_scale, obj_const, bnorm, cnorm) -> dict:
    """FP64 KKT of (x, y) on an already-scaled LP (ora_eval_kkt,
    pdhg_impl.hpp:92-109 over backend_cpu.cpp:101-149)."""
    lib = _load(ORACLE_SO)
    f = lib.ora_eval_kkt
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 17
    vecs = [np.ascontiguousarray(v, dtype=np.float64) for v in (c, l, u, lo, hi, rres, cres, x, y)]
    ints = [np.ascontiguousarray(v, dtype=np.int32) for v in (A.ptr, A.idx, AT.ptr, AT.idx)]
    vals = [np.ascontiguousarray(v, dtype=np.float64) for v in (A.val, AT.val)]
    sc = np.array([obj_scale, obj_const, bnorm, cnorm], dtype=np.float64)
    out = np.zeros(6)
    f(A.rows, A.cols, _p(ints[0]), _p(ints[1]), _p(vals[0]), _p(ints[2]), _p(ints[3]), _p(vals[1]),
      *[_p(v) for v in vecs], _p(sc), _p(out))
    return dict(zip(("pobj", "dobj", "rel_p", "rel_d", "rel_gap", "err"), (float(v) for v in out)))


def transpose(a):
    """lp.cpp:55-72 (ora_transpose): the counting-sort transpose of a Csr."""
    from ganit_v2_b200.lp import Csr
    lib = _load(ORACLE_SO)
    f = lib.ora_transpose
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 6
    ptr = np.ascontiguousarray(a.ptr, dtype=np.int32)
    idx = np.ascontiguousarray(a.idx, dtype=np.int32)
    val = np.ascontiguousarray(a.val, dtype=np.float64)
    t_ptr = np.empty(a.cols + 1, dtype=np.int32)
    t_idx = np.empty(max(a.nnz, 1), dtype=np.int32)
    t_val = np.empty(max(a.nnz, 1), dtype=np.float64)
    if f(a.rows, a.cols, _p(ptr), _p(idx), _p(val), _p(t_ptr), _p(t_idx), _p(t_val)) != 0:
        raise MemoryError("ora_transpose")
    return Csr(a.cols, a.rows, t_ptr, t_idx[:a.nnz], t_val[:a.nnz])


# ---------------------------------------------------------------- reference build
def ref_solve(lp, threads: int | None = None, **opts) -> OracleResult:
    """Run the UNMODIFIED reference ganit::solve_pdhg_cpu (OpenMP; ``threads``
    sets omp_set_num_threads through libgomp when given)."""
    lib = _load(REF_SO)
    if threads is not None:
        _set_omp_threads(threads)
    a = _arrays(lp)
    o = _options(**opts)
    r = _RefRes()
    x = np.zeros(lp.n)
    y = np.zeros(lp.m)
    f = lib.ref_solve_pdhg
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 8 + [C.c_double, C.c_int] + [C.c_void_p] * 3 + \
                 [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    rc = f(lp.m, lp.n, _p(a["ptr"]), _p(a["idx"]), _p(a["val"]), _p(a["c"]), _p(a["l"]), _p(a["u"]), _p(a["lo"]),
           _p(a["hi"]), float(lp.obj_const), int(lp.maximize), _p(a["qptr"]), _p(a["qidx"]), _p(a["qval"]),
           C.byref(o), C.byref(r), _p(x), _p(y))
    if rc != 0:
        raise RuntimeError("reference solve_pdhg_cpu threw")
    return OracleResult(STATUS[r.status], r.pobj, r.dobj, r.rel_p, r.rel_d, r.rel_gap, r.iterations,
                        r.fp32_iterations, r.l2_iterations, r.restarts, r.setup_s, r.solve_s, x, y)


REFCUDA_SO = os.path.join(HERE, "_ref", "libganit_refcuda.so")


def refcuda_available() -> bool:
    return os.path.exists(REFCUDA_SO)


def refcuda_solve(lp, **opts) -> OracleResult:
    """Run the UNMODIFIED reference ganit::solve_pdhg_gpu (src/backend_cuda.cu,
    built for sm_100a; needs a GPU).  LPs only."""
    lib = _load(REFCUDA_SO)
    a = _arrays(lp)
    if a["qptr"] is not None:
        raise ValueError("refcuda_solve takes LPs only")
    o = _options(**opts)
    r = _RefRes()
    x = np.zeros(lp.n)
    y = np.zeros(lp.m)
    f = lib.refcuda_solve_pdhg_gpu
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 8 + [C.c_double, C.c_int] + [C.c_void_p] * 4
    rc = f(lp.m, lp.n, _p(a["ptr"]), _p(a["idx"]), _p(a["val"]), _p(a["c"]), _p(a["l"]), _p(a["u"]), _p(a["lo"]),
           _p(a["hi"]), float(lp.obj_const), int(lp.maximize), C.byref(o), C.byref(r), _p(x), _p(y))
    if rc != 0:
        raise RuntimeError("reference solve_pdhg_gpu threw")
    return OracleResult(STATUS[r.status], r.pobj, r.dobj, r.rel_p, r.rel_d, r.rel_gap, r.iterations,
                        r.fp32_iterations, r.l2_iterations, r.restarts, r.setup_s, r.solve_s, x, y)


def dropin_available() -> bool:
    return os.path.exists(DROPIN_SO)


def dropin_solve(lp, **opts) -> OracleResult:
    """The reference's unmodified run_pdhg (src/pdhg_impl.hpp) driving the B200
    kernels through include/ganit_b200_backend.hpp (needs a GPU)."""
    lib = _load(DROPIN_SO)
    a = _arrays(lp)
    o = _options(**opts)
    r = _RefRes()
    x = np.zeros(lp.n)
    y = np.zeros(lp.m)
    f = lib.dropin_solve_b200
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 8 + [C.c_double, C.c_int] + [C.c_void_p] * 3 + \
                 [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    rc = f(lp.m, lp.n, _p(a["ptr"]), _p(a["idx"]), _p(a["val"]), _p(a["c"]), _p(a["l"]), _p(a["u"]), _p(a["lo"]),
           _p(a["hi"]), float(lp.obj_const), int(lp.maximize), _p(a["qptr"]), _p(a["qidx"]), _p(a["qval"]),
           C.byref(o), C.byref(r), _p(x), _p(y))
    if rc != 0:
        raise RuntimeError("run_pdhg with B200Backend threw")
    return OracleResult(STATUS[r.status], r.pobj, r.dobj, r.rel_p, r.rel_d, r.rel_gap, r.iterations,
                        r.fp32_iterations, r.l2_iterations, r.restarts, r.setup_s, r.solve_s, x, y)


def _set_omp_threads(k: int) -> None:
    gomp = C.CDLL("libgomp.so.1")
    gomp.omp_set_num_threads(int(k))


def ref_read_mps(path: str):
    """Read an MPS / QPS file with the reference reader (src/mps.cpp:69-272)."""
    from ganit_v2_b200.lp import LP, Csr

    lib = _load(REF_SO)
    lib.ref_read_mps.restype = C.c_void_p
    lib.ref_read_mps.argtypes = [C.c_char_p]
    h = lib.ref_read_mps(path.encode())
    if not h:
        raise RuntimeError(f"reference read_mps failed on {path}")
    try:
        dims = np.zeros(5, dtype=np.int64)
        lib.ref_mps_dims.argtypes = [C.c_void_p, C.c_void_p]
        lib.ref_mps_dims(h, _p(dims))
        m, n, nnz, qnnz, maxi = (int(v) for v in dims)
        ptr = np.zeros(m + 1, np.int32); idx = np.zeros(nnz, np.int32); val = np.zeros(nnz)
        c = np.zeros(n); l = np.zeros(n); u = np.zeros(n); lo = np.zeros(m); hi = np.zeros(m)
        oc = np.zeros(1)
        qptr = np.zeros(n + 1, np.int32) if qnnz else None
        qidx = np.zeros(qnnz, np.int32) if qnnz else None
        qval = np.zeros(qnnz) if qnnz else None
        lib.ref_mps_copy.argtypes = [C.c_void_p] * 13
        lib.ref_mps_copy(h, _p(ptr), _p(idx), _p(val), _p(c), _p(l), _p(u), _p(lo), _p(hi), _p(oc), _p(qptr),
                         _p(qidx), _p(qval))
        is_int = np.zeros(n, np.uint8)
        lib.ref_mps_is_int.argtypes = [C.c_void_p, C.c_void_p]
        lib.ref_mps_is_int(h, _p(is_int))
    finally:
        lib.ref_mps_free.argtypes = [C.c_void_p]
        lib.ref_mps_free(h)
    Q = Csr(n, n, qptr, qidx, qval) if qnnz else None
    return LP(Csr(m, n, ptr, idx, val), c, l, u, lo, hi, obj_const=float(oc[0]), maximize=bool(maxi), Q=Q,
              name=os.path.basename(path), is_int=is_int.astype(bool) if is_int.any() else None)


def ref_dual_simplex(lp, time_limit: float = 300.0) -> dict:
    """Exact vertex from the reference DualSimplex: objective, x, row duals y
    (minimisation sense), basis heads and variable statuses."""
    lib = _load(REF_SO)
    a = _arrays(lp)
    x = np.zeros(lp.n)
    y = np.zeros(lp.m)
    head = np.zeros(lp.m, np.int32)
    status = np.zeros(lp.n + lp.m, np.int8)
    obj = C.c_double(0)
    iters = C.c_long(0)
    f = lib.ref_dual_simplex
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 8 + [C.c_double, C.c_int, C.c_double] + [C.c_void_p] * 6
    rc = f(lp.m, lp.n, _p(a["ptr"]), _p(a["idx"]), _p(a["val"]), _p(a["c"]), _p(a["l"]), _p(a["u"]), _p(a["lo"]),
           _p(a["hi"]), float(lp.obj_const), int(lp.maximize), float(time_limit), C.addressof(obj), _p(x), _p(y),
           _p(head), _p(status), C.addressof(iters))
    return {"status": int(rc), "objective": obj.value, "x": x, "y": y, "head": head, "var_status": status,
            "iterations": iters.value}


# ---- strong branching (src/mip.cpp:668-783) with the reference dual simplex
SIMPLEX_OPTIMAL, SIMPLEX_INFEASIBLE = 0, 1


def _child(lp, j: int, lo: float, hi: float):
    from dataclasses import replace

    l = lp.l.copy()
    u = lp.u.copy()
    l[j], u[j] = lo, hi
    return replace(lp, l=l, u=u, meta={})


def _min_form(lp):
    from dataclasses import replace

    if not lp.maximize:
        return lp
    return replace(lp, c=-lp.c, obj_const=-lp.obj_const, maximize=False, meta={})


def strong_branch_reference(lp, x, candidates, node_obj: float, cutoff: float = np.inf) -> dict:
    """The strong-branching loop of Mip::select_branch (src/mip.cpp:727-783)
    with every child solved to optimality by the reference dual simplex (cold,
    no iteration limit): z per child (+inf when infeasible or >= cutoff), the
    scores, and the decision (action 0 branch / -1 tighten / -2 infeasible,
    column, new bounds).  Minimisation form throughout."""
    lpm = _min_form(lp)
    eps = 1e-6
    k = len(candidates)
    z = np.full((k, 2), np.nan)
    status = np.zeros((k, 2), np.int32)
    for t, j in enumerate(candidates):
        v = float(x[j])
        for d, (lo, hi) in enumerate(((lpm.l[j], np.floor(v)), (np.ceil(v), lpm.u[j]))):
            if not lo <= hi:
                status[t, d] = SIMPLEX_INFEASIBLE
                z[t, d] = np.inf
                continue
            r = ref_dual_simplex(_child(lpm, int(j), lo, hi))
            status[t, d] = r["status"]
            if r["status"] == SIMPLEX_INFEASIBLE:
                z[t, d] = np.inf
            elif r["status"] == SIMPLEX_OPTIMAL:
                z[t, d] = np.inf if r["objective"] >= cutoff else r["objective"]
            else:
                raise RuntimeError(f"dual simplex status {r['status']} on a child")
    score = np.zeros(k)
    action, var, blo, bhi, best = 0, int(candidates[0]), np.nan, np.nan, -1.0
    for t, j in enumerate(candidates):
        inf0, inf1 = not np.isfinite(z[t, 0]), not np.isfinite(z[t, 1])
        if inf0 and inf1:
            action, var = -2, int(j)
            break
        if inf0 or inf1:
            v = float(x[j])
            action, var = -1, int(j)
            blo, bhi = (np.ceil(v), lpm.u[j]) if inf0 else (lpm.l[j], np.floor(v))
            break
        score[t] = max(z[t, 0] - node_obj, eps) * max(z[t, 1] - node_obj, eps)
        if score[t] > best:
            best, var = score[t], int(j)
    return {"z": z, "status": status, "score": score, "action": action, "var": var, "lo": blo, "hi": bhi}


def lagrangian_bound_exact(lp, y, j: int, lo: float, hi: float) -> float:
    """EXACT value (rational arithmetic) of the Lagrangian bound the reference
    certifies child bounds with (Mip::safe_bound, src/mip.cpp:356-410), for
    duals y of the child with column j's bounds set to [lo, hi]:
        sum_i min(y_i lo_i, y_i hi_i) + sum_j min_{x_j in [l_j, u_j]} (c - A'y)_j x_j,
    y_i clamped to <= 0 on rows without a finite lower side and >= 0 without
    a finite upper side; -inf when a column with an infinite bound has a
    reduced cost of the wrong sign.  Minimisation form."""
    from fractions import Fraction as F

    lpm = _min_form(lp)
    m, n = lpm.m, lpm.n
    yy = []
    total = F(0)
    for i in range(m):
        yi = float(y[i])
        if not np.isfinite(lpm.lo[i]):
            yi = min(yi, 0.0)
        if not np.isfinite(lpm.hi[i]):
            yi = max(yi, 0.0)
        yy.append(F(yi))
        if yi > 0:
            total += F(yi) * F(float(lpm.lo[i]))
        elif yi < 0:
            total += F(yi) * F(float(lpm.hi[i]))
    d = [F(float(v)) for v in lpm.c]
    ptr, idx, val = lpm.A.ptr, lpm.A.idx, lpm.A.val
    for i in range(m):
        if yy[i] == 0:
            continue
        for t in range(ptr[i], ptr[i + 1]):
            d[idx[t]] -= yy[i] * F(float(val[t]))
    for c in range(n):
        l, u = (lo, hi) if c == j else (float(lpm.l[c]), float(lpm.u[c]))
        if (not np.isfinite(l) and d[c] > 0) or (not np.isfinite(u) and d[c] < 0):
            return -np.inf
        cands = [d[c] * F(v) for v in (l, u) if np.isfinite(v)]
        total += min(cands) if cands else F(0)
    return total  # a Fraction: compare it with floats exactly


def ref_strong_branch(lp, x, candidates, iter_limit: int = 60) -> dict:
    """The reference's own strong-branching loop (warm dual simplex per child,
    src/mip.cpp:738-760) through ref_shim.cpp: z per child in its mapping,
    simplex statuses and iterations, the node objective, and the loop's wall
    time (the node solve before it is not timed).  Minimisation LPs."""
    lib = _load(REF_SO)
    a = _arrays(lp)
    cand = np.ascontiguousarray(candidates, dtype=np.int32)
    x = np.ascontiguousarray(x, dtype=np.float64)
    k = int(cand.size)
    z = np.zeros(2 * k)
    st = np.zeros(2 * k, np.int32)
    it = np.zeros(2 * k, np.int64)
    zn = C.c_double(0)
    secs = C.c_double(0)
    f = lib.ref_strong_branch
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 8 + [C.c_double, C.c_void_p, C.c_void_p, C.c_int, C.c_long] + \
        [C.c_void_p] * 5
    rc = f(lp.m, lp.n, _p(a["ptr"]), _p(a["idx"]), _p(a["val"]), _p(a["c"]), _p(a["l"]), _p(a["u"]), _p(a["lo"]),
           _p(a["hi"]), float(lp.obj_const), _p(x), _p(cand), k, int(iter_limit), C.addressof(zn), _p(z), _p(st),
           _p(it), C.addressof(secs))
    if rc != 0:
        raise RuntimeError(f"reference strong branching failed ({rc})")
    return {"z": z.reshape(k, 2), "status": st.reshape(k, 2), "iterations": it.reshape(k, 2), "z_node": zn.value,
            "seconds": secs.value}
