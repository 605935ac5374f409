"""Python host API over libganit_b200.so.

Mirrors the reference's public PDHG interface (include/ganit/pdhg.hpp):
``Precision``, ``Options`` (same fields and defaults), ``Status``, ``Result``
and ``solve_pdhg_gpu(lp, opt)`` (here backed by the B200 engine; also exported
as ``solve_pdhg_b200``).  ``Problem`` keeps a scaled problem resident on the
GPU for repeated solves.  ``Backend`` exposes the Backend-concept operations
that src/pdhg_impl.hpp drives.

There is no CPU fallback: if the library is missing or no sm_100 GPU is
visible, every call raises.
"""
from __future__ import annotations

import ctypes as C
import enum
import os
from dataclasses import dataclass, field

import numpy as np

from .lp import LP, Csr

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libganit_b200.so")

GB_OK = 0


class GanitError(RuntimeError):
    """Error reported by libganit_b200 (status code + message)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"libganit_b200 error {code}: {msg}")
        self.code = code


class Precision(enum.IntEnum):  # include/ganit/pdhg.hpp:10
    Double = 0
    Mixed = 1
    Dynamic = 2
    MixedBf16 = 3  # extension: BF16-matrix phase first (LPs)


class Status(enum.IntEnum):  # include/ganit/pdhg.hpp:27
    Optimal = 0
    PrimalInfeasible = 1
    IterationLimit = 2
    TimeLimit = 3
    NumericalError = 4
    DualInfeasible = 5  # extension (Options.detect_unbounded)


STATUS_NAMES = {0: "OPTIMAL", 1: "PRIMAL_INFEASIBLE", 2: "ITERATION_LIMIT", 3: "TIME_LIMIT", 4: "NUMERICAL_ERROR",
                5: "DUAL_INFEASIBLE"}


@dataclass
class Options:  # include/ganit/pdhg.hpp:12-25
    tol: float = 1e-4
    max_iter: int = 10_000_000
    time_limit: float = 3600.0
    check_every: int = 64
    ruiz_iters: int = 10
    pock_chambolle: bool = True
    infeas_tol: float = 1e-8
    precision: Precision = Precision.Double
    stall_checks: int = 12
    stall_checks_l2: int = 24
    verbose: int = 0
    detect_unbounded: bool = False  # extension: GB_DUAL_INFEASIBLE from a primal ray (LPs)


@dataclass
class Result:  # include/ganit/pdhg.hpp:30-42
    status: Status
    x: np.ndarray
    y: np.ndarray
    pobj: float
    dobj: float
    rel_primal: float
    rel_dual: float
    rel_gap: float
    iterations: int
    fp32_iterations: int
    l2_iterations: int
    restarts: int
    setup_seconds: float
    solve_seconds: float
    device: str = "b200"
    norm_a: float = float("nan")
    primal_weight: float = float("nan")
    checks: int = 0
    phases: int = 0
    bf16_iterations: int = 0

    @property
    def status_name(self) -> str:
        return STATUS_NAMES[int(self.status)]


# ---------------------------------------------------------------- ctypes mirror of ganit_b200.h
class _GbLp(C.Structure):
    _fields_ = [("m", C.c_int32), ("n", C.c_int32), ("a_ptr", C.c_void_p), ("a_idx", C.c_void_p),
                ("a_val", C.c_void_p), ("c", C.c_void_p), ("l", C.c_void_p), ("u", C.c_void_p), ("lo", C.c_void_p),
                ("hi", C.c_void_p), ("obj_const", C.c_double), ("maximize", C.c_int32), ("q_ptr", C.c_void_p),
                ("q_idx", C.c_void_p), ("q_val", C.c_void_p), ("q_rank", C.c_int32), ("q_F", C.c_void_p),
                ("q_D", C.c_void_p)]


class _GbOptions(C.Structure):
    _fields_ = [("tol", C.c_double), ("max_iter", C.c_int64), ("time_limit", C.c_double),
                ("check_every", C.c_int32), ("ruiz_iters", C.c_int32), ("pock_chambolle", C.c_int32),
                ("infeas_tol", C.c_double), ("precision", C.c_int32), ("stall_checks", C.c_int32),
                ("stall_checks_l2", C.c_int32), ("verbose", C.c_int32), ("detect_unbounded", C.c_int32)]


class _GbResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("pobj", C.c_double), ("dobj", C.c_double), ("rel_primal", C.c_double),
                ("rel_dual", C.c_double), ("rel_gap", C.c_double), ("iterations", C.c_int64),
                ("fp32_iterations", C.c_int64), ("l2_iterations", C.c_int64), ("restarts", C.c_int32),
                ("setup_seconds", C.c_double), ("solve_seconds", C.c_double), ("norm_a", C.c_double),
                ("primal_weight", C.c_double), ("checks", C.c_int32), ("phases", C.c_int32),
                ("bf16_iterations", C.c_int64)]


class _GbBranchCand(C.Structure):
    _fields_ = [("z", C.c_double * 2), ("cert", C.c_double * 2), ("status", C.c_int32 * 2),
                ("iterations", C.c_int64 * 2), ("score", C.c_double)]


class _GbBranchDecision(C.Structure):
    _fields_ = [("action", C.c_int32), ("var", C.c_int32), ("lo", C.c_double), ("hi", C.c_double),
                ("est", C.c_double * 2), ("cert", C.c_double * 2), ("children_solved", C.c_int32),
                ("seconds", C.c_double)]


class _GbScaledLp(C.Structure):
    _fields_ = [("m", C.c_int32), ("n", C.c_int32)] + [
        (k, C.c_void_p) for k in ("a_ptr", "a_idx", "a_val", "at_ptr", "at_idx", "at_val", "q_ptr", "q_idx", "q_val",
                                  "c", "l", "u", "lo", "hi", "rres", "cres")]


class GbKktScalars(C.Structure):
    _fields_ = [("obj_scale", C.c_double), ("obj_const", C.c_double), ("bnorm", C.c_double), ("cnorm", C.c_double)]


class _GbDiffOptions(C.Structure):
    _fields_ = [("implicit_max_iters", C.c_int64), ("implicit_tol", C.c_double), ("polish", C.c_int32),
                ("pad", C.c_int32)]


class _GbDiffInfo(C.Structure):
    _fields_ = [("tau", C.c_double), ("sigma", C.c_double), ("tail_iterations", C.c_int64),
                ("checkpoint_every", C.c_int64), ("implicit_iterations", C.c_int64), ("implicit_residual", C.c_double),
                ("implicit_converged", C.c_int32), ("free_cols", C.c_int32), ("active_rows", C.c_int32),
                ("polished", C.c_int32), ("active_set_repaired", C.c_int32), ("pad", C.c_int32),
                ("polish_iterations", C.c_int64), ("launches", C.c_int64)]


class GbKkt(C.Structure):
    _fields_ = [("pobj", C.c_double), ("dobj", C.c_double), ("rel_p", C.c_double), ("rel_d", C.c_double),
                ("rel_gap", C.c_double), ("err", C.c_double)]


LOAD_MODES = {0: "plain", 1: "stream", 2: "prefetch"}  # GB_LOAD_*


def _load_mode_names(m) -> dict:
    return {"A_f32": LOAD_MODES[int(m[0])], "AT_f32": LOAD_MODES[int(m[1])], "A_f64": LOAD_MODES[int(m[2])],
            "AT_f64": LOAD_MODES[int(m[3])]}


# Every symbol of include/ganit_b200.h (checked by the tests).
EXPORTS = [
    "gb_last_error", "gb_release_cached_memory", "gb_cached_memory_bytes", "gb_version", "gb_default_options", "gb_set_device", "gb_csr_transpose", "gb_solve", "gb_problem_create",
    "gb_problem_solve", "gb_problem_get_solution", "gb_problem_destroy", "gb_problem_stream",
    "gb_problem_time_kernels", "gb_problem_stats", "gb_problem_autotune", "gb_problem_time_kernels_graph",
    "gb_batch_time_kernels_graph", "gb_backend_create", "gb_backend_destroy", "gb_vec_zeros",
    "gb_vec_from_host", "gb_vec_to_host", "gb_vec_size", "gb_vec_destroy", "gb_copy", "gb_fill", "gb_spmv_A",
    "gb_spmv_AT", "gb_spmv_Q", "gb_primal_step", "gb_dual_step", "gb_sub", "gb_scale_into", "gb_primal_res2",
    "gb_dual_res", "gb_row_dual_obj", "gb_dot", "gb_dot_c", "gb_diff2", "gb_batch_create", "gb_batch_solve",
    "gb_batch_get_solution", "gb_batch_schedule", "gb_batch_autotune", "gb_batch_time_kernels", "gb_batch_destroy",
    "gb_diff_create", "gb_diff_forward",
    "gb_diff_default_options", "gb_diff_set_options", "gb_diff_backward", "gb_diff_get_info", "gb_diff_tail_start", "gb_diff_destroy",
    "gb_eval_kkt_noalloc", "gb_read_mps", "gb_model_lp", "gb_model_name", "gb_model_free", "gb_factor_detect",
    "gb_factor_lp", "gb_factor_expand", "gb_factor_free", "gb_model_is_int", "gb_strong_branch",
    "gb_problem_set_start", "gb_batch_set_start", "gb_batch_clear_start", "gb_batch_load_modes",
    "gb_problem_load_modes",
]

_lib = None


def load_library(path: str = LIB_PATH):
    """Load libganit_b200.so (raises if it is missing -- no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise GanitError(-4, f"{path} is not built; run `python -m ganit_v2_b200.build`")
    lib = C.CDLL(path)
    vp, i32, i64, dbl = C.c_void_p, C.c_int, C.c_int64, C.c_double
    sig = {
        "gb_last_error": (C.c_char_p, []), "gb_release_cached_memory": (None, []),
        "gb_cached_memory_bytes": (i64, []), "gb_version": (i32, []), "gb_default_options": (None, [vp]),
        "gb_set_device": (i32, [i32]), "gb_csr_transpose": (i32, [i32, i32, vp, vp, vp, vp, vp, vp]),
        "gb_solve": (i32, [vp, vp, vp, vp, vp]),
        "gb_problem_create": (i32, [vp, vp, vp]), "gb_problem_solve": (i32, [vp, vp, vp]),
        "gb_problem_get_solution": (i32, [vp, vp, vp]), "gb_problem_destroy": (None, [vp]),
        "gb_problem_stream": (vp, [vp]), "gb_problem_time_kernels": (i32, [vp, i32, i32, vp, vp, vp]),
        "gb_problem_stats": (i32, [vp, vp, vp]), "gb_problem_autotune": (i32, [vp, i32, vp, vp, vp, vp]),
        "gb_problem_time_kernels_graph": (i32, [vp, i32, i32, vp, vp, vp]),
        "gb_batch_time_kernels_graph": (i32, [vp, i32, i32, vp, vp, vp]), "gb_backend_create": (i32, [vp, i32, i32, vp]),
        "gb_backend_destroy": (None, [vp]), "gb_vec_zeros": (i32, [vp, i32, vp]),
        "gb_vec_from_host": (i32, [vp, vp, i32, vp]), "gb_vec_to_host": (i32, [vp, vp, vp]),
        "gb_vec_size": (i32, [vp]), "gb_vec_destroy": (None, [vp]), "gb_copy": (i32, [vp, vp, vp]),
        "gb_fill": (i32, [vp, vp, dbl]), "gb_spmv_A": (i32, [vp, vp, vp]), "gb_spmv_AT": (i32, [vp, vp, vp]),
        "gb_spmv_Q": (i32, [vp, vp, vp]), "gb_primal_step": (i32, [vp, vp, vp, vp, dbl, vp, vp, vp]),
        "gb_dual_step": (i32, [vp, vp, vp, dbl, vp, vp]), "gb_sub": (i32, [vp, vp, vp, vp]),
        "gb_scale_into": (i32, [vp, vp, dbl, vp]), "gb_primal_res2": (i32, [vp, vp, vp]),
        "gb_dual_res": (i32, [vp, vp, vp, i32, vp, vp]), "gb_row_dual_obj": (i32, [vp, vp, vp]),
        "gb_dot": (i32, [vp, vp, vp, vp]), "gb_dot_c": (i32, [vp, vp, vp]), "gb_diff2": (i32, [vp, vp, vp, vp]),
        "gb_batch_create": (i32, [i32, vp, vp, vp]), "gb_batch_solve": (i32, [vp, vp, vp]),
        "gb_batch_get_solution": (i32, [vp, i32, vp, vp]), "gb_batch_schedule": (i32, [vp, vp, vp, vp]),
        "gb_batch_autotune": (i32, [vp, i32, vp, vp, vp, vp]),
        "gb_batch_load_modes": (i32, [vp, vp]), "gb_problem_load_modes": (i32, [vp, vp]),
        "gb_batch_time_kernels": (i32, [vp, i32, i32, vp, vp, vp, vp]),
        "gb_batch_destroy": (None, [vp]), "gb_diff_create": (i32, [i32, vp, vp, i32, i32, vp]),
        "gb_diff_forward": (i32, [vp, vp, vp, vp, vp]), "gb_diff_default_options": (None, [vp]),
        "gb_diff_set_options": (i32, [vp, vp]),
        "gb_diff_backward": (i32, [vp, vp, vp, vp, vp, vp, vp]), "gb_diff_get_info": (i32, [vp, i32, vp]),
        "gb_diff_tail_start": (i32, [vp, vp, vp]), "gb_diff_destroy": (None, [vp]),
        "gb_eval_kkt_noalloc": (i32, [vp, vp, vp, vp, vp, vp, vp, vp]),
        "gb_read_mps": (i32, [C.c_char_p, vp]), "gb_model_lp": (vp, [vp]), "gb_model_name": (C.c_char_p, [vp]),
        "gb_model_free": (None, [vp]), "gb_factor_detect": (i32, [vp, vp]), "gb_factor_lp": (vp, [vp]),
        "gb_factor_expand": (i32, [vp, vp, vp, vp, vp]), "gb_factor_free": (None, [vp]),
        "gb_model_is_int": (vp, [vp]),
        "gb_strong_branch": (i32, [vp, vp, vp, i32, vp, dbl, dbl, vp, vp, vp]),
        "gb_problem_set_start": (i32, [vp, vp, vp]), "gb_batch_set_start": (i32, [vp, i32, vp, vp]),
        "gb_batch_clear_start": (i32, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _check(rc: int):
    if rc != GB_OK:
        raise GanitError(rc, _lib.gb_last_error().decode(errors="replace"))


def _p(a):
    return None if a is None else a.ctypes.data


def _vec(a, k: int, name: str) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.shape != (k,):
        raise ValueError(f"{name} must have {k} entries")
    return a


class _LpView:
    """Keeps the numpy arrays of an LP alive while the C struct points at them."""

    def __init__(self, lp: LP):
        self.arrays = []

        def keep(a, dt):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=dt)
            self.arrays.append(a)
            return a

        ptr = keep(lp.A.ptr, np.int32)
        idx = keep(lp.A.idx, np.int32)
        val = keep(lp.A.val, np.float64)
        vecs = [keep(getattr(lp, k), np.float64) for k in ("c", "l", "u", "lo", "hi")]
        q = lp.Q if (lp.Q is not None and lp.Q.nnz) else None
        qp = keep(q.ptr, np.int32) if q else None
        qi = keep(q.idx, np.int32) if q else None
        qv = keep(q.val, np.float64) if q else None
        F = keep(lp.F, np.float64) if lp.F is not None else None
        D = keep(lp.D, np.float64) if lp.F is not None else None
        self.s = _GbLp(lp.m, lp.n, _p(ptr), _p(idx), _p(val), *[_p(v) for v in vecs], float(lp.obj_const),
                       int(lp.maximize), _p(qp), _p(qi), _p(qv), int(F.shape[1]) if F is not None else 0, _p(F),
                       _p(D))


def _opts(opt: Options | None) -> _GbOptions:
    o = opt or Options()
    return _GbOptions(o.tol, o.max_iter, o.time_limit, o.check_every, o.ruiz_iters, int(o.pock_chambolle),
                      o.infeas_tol, int(o.precision), o.stall_checks, o.stall_checks_l2, int(o.verbose),
                      int(bool(o.detect_unbounded)))


def _result(r: _GbResult, x, y) -> Result:
    return Result(Status(r.status), x, y, r.pobj, r.dobj, r.rel_primal, r.rel_dual, r.rel_gap, r.iterations,
                  r.fp32_iterations, r.l2_iterations, r.restarts, r.setup_seconds, r.solve_seconds, "b200",
                  r.norm_a, r.primal_weight, r.checks, r.phases, r.bf16_iterations)


def read_mps(path: str) -> LP:
    """Read an MPS / QPS file with the library's reader (gb_read_mps; the
    format rules of the reference's src/mps.cpp:69-272).  No GPU needed."""
    lib = load_library()
    h = C.c_void_p()
    _check(lib.gb_read_mps(os.fsencode(path), C.byref(h)))
    try:
        name = lib.gb_model_name(h).decode(errors="replace") or os.path.basename(path)
        lp = _lp_from_view(_GbLp.from_address(lib.gb_model_lp(h)), name=name)
        if lp.n:
            flags = np.ctypeslib.as_array(C.cast(lib.gb_model_is_int(h), C.POINTER(C.c_uint8)), shape=(lp.n,))
            if flags.any():
                lp.is_int = flags.astype(bool)
        return lp
    finally:
        lib.gb_model_free(h)


def _lp_from_view(v: "_GbLp", name: str = "") -> LP:
    """Copy of a library-owned gb_lp (CSR or diagonal-plus-low-rank Hessian)."""
    m, n = v.m, v.n

    def arr(ptr, k, dt):
        if not ptr or k == 0:
            return np.zeros(k, dtype=dt)
        ct = C.c_int32 if dt == np.int32 else C.c_double
        return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), shape=(k,)).astype(dt, copy=True)

    ptr = arr(v.a_ptr, m + 1, np.int32)
    nnz = int(ptr[-1]) if m else 0
    A = Csr(m, n, ptr, arr(v.a_idx, nnz, np.int32), arr(v.a_val, nnz, np.float64))
    Q = F = D = None
    if v.q_ptr:
        qp = arr(v.q_ptr, n + 1, np.int32)
        Q = Csr(n, n, qp, arr(v.q_idx, int(qp[-1]), np.int32), arr(v.q_val, int(qp[-1]), np.float64))
    if v.q_rank > 0:
        F = arr(v.q_F, n * v.q_rank, np.float64).reshape(n, v.q_rank)
        D = arr(v.q_D, n, np.float64)
    return LP(A, arr(v.c, n, np.float64), arr(v.l, n, np.float64), arr(v.u, n, np.float64),
              arr(v.lo, m, np.float64), arr(v.hi, m, np.float64), obj_const=float(v.obj_const),
              maximize=bool(v.maximize), Q=Q, F=F, D=D, name=name)


class FactorForm:
    """A lifted factor-model QP rewritten for the diagonal-plus-low-rank Q x
    kernel (gb_factor_detect).  ``lp`` is the rewritten problem over x alone;
    ``expand(x, y)`` maps its solution back to the input's variables and rows.
    Raises GanitError (GB_ERR_UNSUPPORTED) when the input has no such structure."""

    def __init__(self, lp: LP):
        self._lib = load_library()
        self._view = _LpView(lp)
        self.m_full, self.n_full = lp.m, lp.n
        h = C.c_void_p()
        _check(self._lib.gb_factor_detect(C.byref(self._view.s), C.byref(h)))
        self._h = h
        self.lp = _lp_from_view(_GbLp.from_address(self._lib.gb_factor_lp(h)), name=(lp.name or "") + "_dplr")
        self.factors = self.lp.F.shape[1]

    def expand(self, x, y):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        xf = np.zeros(self.n_full)
        yf = np.zeros(self.m_full)
        _check(self._lib.gb_factor_expand(self._h, _p(x), _p(y), _p(xf), _p(yf)))
        return xf, yf

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                self._lib.gb_factor_free(self._h)
                self._h = None
        except Exception:
            pass


BRANCH_VAR, BRANCH_TIGHTEN, BRANCH_NODE_INFEASIBLE = 0, -1, -2


@dataclass
class StrongBranch:
    """Outcome of gb_strong_branch: per candidate (rows) and child (columns:
    down, up) the objective estimate, certified bound, status and iterations;
    the candidates' scores; and the decision Mip::select_branch would take
    (action BRANCH_VAR / BRANCH_TIGHTEN / BRANCH_NODE_INFEASIBLE)."""

    candidates: np.ndarray
    z: np.ndarray
    cert: np.ndarray
    status: np.ndarray
    iterations: np.ndarray
    score: np.ndarray
    action: int
    var: int
    lo: float
    hi: float
    est: np.ndarray
    cert_choice: np.ndarray
    children_solved: int
    seconds: float


def fractional(x, is_int, int_tol: float = 1e-6) -> np.ndarray:
    """Integer columns whose value is fractional beyond int_tol (Mip::fractional,
    src/mip.cpp:256-263), in column order."""
    x = np.asarray(x, dtype=np.float64)
    f = x - np.floor(x)
    return np.flatnonzero(np.asarray(is_int, dtype=bool) & (f > int_tol) & (f < 1.0 - int_tol)).astype(np.int32)


def most_fractional(x, cols, k: int) -> np.ndarray:
    """The k columns of `cols` closest to half-integral, most fractional first
    (the expert order of full strong branching, src/mip.cpp:709-714; stable)."""
    x = np.asarray(x, dtype=np.float64)
    cols = np.asarray(cols, dtype=np.int32)
    f = x[cols] - np.floor(x[cols])
    order = np.argsort(-np.minimum(f, 1.0 - f), kind="stable")
    return cols[order[:k]]


def strong_branch(lp: LP, x, candidates, node_obj: float, cutoff: float = float("inf"),
                  opt: Options | None = None, y=None) -> StrongBranch:
    """Strong-branch the candidate columns of a MILP node LP on the GPU
    (gb_strong_branch): both children of every candidate solved as one batch,
    each with a rigorous bound from its duals.  Objectives in minimisation form.
    With the node's duals ``y`` the children start from the node's point."""
    lib = load_library()
    view = _LpView(lp)
    x = np.ascontiguousarray(x, dtype=np.float64)
    cand = np.ascontiguousarray(candidates, dtype=np.int32)
    if x.shape != (lp.n,) or cand.ndim != 1 or cand.size == 0:
        raise ValueError("x must have n entries and candidates at least one")
    if y is not None:
        y = np.ascontiguousarray(y, dtype=np.float64)
        if y.shape != (lp.m,):
            raise ValueError("y must have m entries")
    o = _opts(opt)
    out = (_GbBranchCand * cand.size)()
    dec = _GbBranchDecision()
    _check(lib.gb_strong_branch(C.byref(view.s), _p(x), _p(y), int(cand.size), _p(cand), float(node_obj),
                                float(cutoff), C.addressof(o), out, C.byref(dec)))
    return StrongBranch(
        candidates=cand.copy(),
        z=np.array([[c.z[0], c.z[1]] for c in out]),
        cert=np.array([[c.cert[0], c.cert[1]] for c in out]),
        status=np.array([[c.status[0], c.status[1]] for c in out], dtype=np.int32),
        iterations=np.array([[c.iterations[0], c.iterations[1]] for c in out], dtype=np.int64),
        score=np.array([c.score for c in out]),
        action=int(dec.action), var=int(dec.var), lo=float(dec.lo), hi=float(dec.hi),
        est=np.array(list(dec.est)), cert_choice=np.array(list(dec.cert)),
        children_solved=int(dec.children_solved), seconds=float(dec.seconds))


def release_cached_memory() -> None:
    """Return the device blocks the library keeps for reuse to the driver."""
    load_library().gb_release_cached_memory()


def cached_memory_bytes() -> int:
    return int(load_library().gb_cached_memory_bytes())


def set_device(device: int) -> None:
    lib = load_library()
    _check(lib.gb_set_device(int(device)))


def transpose(a: Csr) -> Csr:
    """ganit::transpose (include/ganit/lp.hpp:32, src/lp.cpp:55-72) on the
    device, as the solver builds A^T (gb_csr_transpose): each row of the
    result lists its entries in increasing source row."""
    lib = load_library()
    t_ptr = np.empty(a.cols + 1, dtype=np.int32)
    t_idx = np.empty(a.nnz, dtype=np.int32)
    t_val = np.empty(a.nnz, dtype=np.float64)
    _check(lib.gb_csr_transpose(int(a.rows), int(a.cols), _p(a.ptr), _p(a.idx), _p(a.val), _p(t_ptr), _p(t_idx),
                                _p(t_val)))
    return Csr(a.cols, a.rows, t_ptr, t_idx, t_val)


def solve_pdhg_gpu(lp: LP, opt: Options | None = None, out=None) -> Result:
    """Same contract as ganit::solve_pdhg_gpu (include/ganit/pdhg.hpp:44-47):
    scale, restarted PDHG with the precision schedule of ``opt``, FP64
    certification and unscaling -- all on the B200.  ``out=(x, y)`` are
    caller-owned float64 arrays (e.g. page-locked) that receive the solution."""
    lib = load_library()
    v = _LpView(lp)
    o = _opts(opt)
    r = _GbResult()
    if out is None:
        x = np.zeros(lp.n)
        y = np.zeros(lp.m)
    else:
        x, y = out
        if not (x.dtype == np.float64 and y.dtype == np.float64 and x.shape == (lp.n,) and y.shape == (lp.m,)
                and x.flags.c_contiguous and y.flags.c_contiguous):
            raise ValueError("out must be two contiguous float64 arrays of n and m entries")
    _check(lib.gb_solve(C.addressof(v.s), C.addressof(o), C.addressof(r), _p(x), _p(y)))
    return _result(r, x, y)


solve_pdhg_b200 = solve_pdhg_gpu


class Problem:
    """A problem uploaded and scaled once, resident in HBM for repeated solves."""

    def __init__(self, lp: LP, opt: Options | None = None):
        self._lib = load_library()
        self.lp = lp
        self.m, self.n = lp.m, lp.n
        v = _LpView(lp)
        o = _opts(opt)
        h = C.c_void_p()
        _check(self._lib.gb_problem_create(C.addressof(v.s), C.addressof(o), C.byref(h)))
        self._h = h

    def set_start(self, x=None, y=None) -> None:
        """Warm start of later solves (gb_problem_set_start): (x, y) in
        original units, x projected onto the bounds; None / NaN entries keep
        the default start; both None restores it."""
        x = None if x is None else _vec(x, self.n, "x")
        y = None if y is None else _vec(y, self.m, "y")
        _check(self._lib.gb_problem_set_start(self._h, _p(x), _p(y)))

    def solve(self, opt: Options | None = None, fetch: bool = True) -> Result:
        o = _opts(opt)
        r = _GbResult()
        _check(self._lib.gb_problem_solve(self._h, C.addressof(o), C.addressof(r)))
        x = y = None
        if fetch:
            x, y = self.solution()
        return _result(r, x, y)

    def solution(self):
        x = np.zeros(self.n)
        y = np.zeros(self.m)
        _check(self._lib.gb_problem_get_solution(self._h, _p(x), _p(y)))
        return x, y

    def time_kernels(self, level: int, iters: int = 50):
        mp, md = C.c_double(), C.c_double()
        nl = C.c_int64()
        _check(self._lib.gb_problem_time_kernels(self._h, int(level), int(iters), C.byref(mp), C.byref(md),
                                                 C.byref(nl)))
        return mp.value, md.value, nl.value

    def autotune(self, iters: int = 50) -> dict:
        """Pick the row-block cut by timing (gb_problem_autotune); solve once first."""
        bn, mr = np.zeros(2, dtype=np.int32), np.zeros(2, dtype=np.int32)
        t0, t1 = np.zeros(2), np.zeros(2)
        _check(self._lib.gb_problem_autotune(self._h, int(iters), _p(bn), _p(mr), _p(t0), _p(t1)))
        return {"block_nnz": int(bn[0]), "max_rows": int(mr[0]), "ms_per_iter_default": float(t0[0]),
                "ms_per_iter_tuned": float(t1[0]), "block_nnz_f64": int(bn[1]), "max_rows_f64": int(mr[1]),
                "ms_per_iter_default_f64": float(t0[1]), "ms_per_iter_tuned_f64": float(t1[1]),
                "load_modes": self.load_modes()}

    def load_modes(self) -> dict:
        """Load variant per matrix and precision class (gb_problem_load_modes)."""
        m = np.zeros(4, dtype=np.int32)
        _check(self._lib.gb_problem_load_modes(self._h, _p(m)))
        return _load_mode_names(m)

    def time_kernels_graph(self, level: int, iters: int = 200) -> dict:
        """Back-to-back launches captured in CUDA graphs (gb_problem_time_kernels_graph)."""
        mp, md, mi = C.c_double(), C.c_double(), C.c_double()
        _check(self._lib.gb_problem_time_kernels_graph(self._h, int(level), int(iters), C.byref(mp), C.byref(md),
                                                       C.byref(mi)))
        return {"ms_primal": mp.value, "ms_dual": md.value, "ms_iteration": mi.value}

    def stats(self):
        nl = C.c_int64()
        bpi = np.zeros(3)
        _check(self._lib.gb_problem_stats(self._h, C.byref(nl), _p(bpi)))
        return nl.value, bpi

    @property
    def stream(self) -> int:
        return self._lib.gb_problem_stream(self._h) or 0

    def close(self):
        if getattr(self, "_h", None):
            self._lib.gb_problem_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class BatchSolver:
    """Many independent LPs solved together on one GPU (gb_batch_*).

    The batch is one block-diagonal problem: every instance keeps its own
    scaling, step sizes, restarts, primal weight, precision phases and FP64
    certification, exactly as if solved alone; a finished instance stops
    costing bandwidth.  LPs only (no Hessian)."""

    def __init__(self, lps, opt: Options | None = None):
        self._lib = load_library()
        self.lps = list(lps)
        self._views = [_LpView(lp) for lp in self.lps]
        arr = (_GbLp * len(self._views))(*[v.s for v in self._views])
        o = _opts(opt)
        h = C.c_void_p()
        _check(self._lib.gb_batch_create(len(self._views), arr, C.addressof(o), C.byref(h)))
        self._h = h

    def __len__(self):
        return len(self.lps)

    def solve(self, opt: Options | None = None, fetch: bool = True) -> list:
        o = _opts(opt)
        res = (_GbResult * len(self.lps))()
        _check(self._lib.gb_batch_solve(self._h, C.addressof(o), res))
        out = []
        for i, r in enumerate(res):
            x = y = None
            if fetch:
                x, y = self.solution(i)
            out.append(_result(r, x, y))
        return out

    def set_start(self, i: int, x=None, y=None) -> None:
        """Warm start of instance i (gb_batch_set_start)."""
        lp = self.lps[i]
        x = None if x is None else _vec(x, lp.n, "x")
        y = None if y is None else _vec(y, lp.m, "y")
        _check(self._lib.gb_batch_set_start(self._h, int(i), _p(x), _p(y)))

    def clear_start(self) -> None:
        _check(self._lib.gb_batch_clear_start(self._h))

    def solution(self, i: int):
        lp = self.lps[i]
        x = np.zeros(lp.n)
        y = np.zeros(lp.m)
        _check(self._lib.gb_batch_get_solution(self._h, int(i), _p(x), _p(y)))
        return x, y

    def schedule(self) -> dict:
        t, b = C.c_int(), C.c_int()
        g = np.zeros(2 * len(self.lps), dtype=np.int32)
        _check(self._lib.gb_batch_schedule(self._h, C.byref(t), C.byref(b), _p(g)))
        return {"threads": t.value, "blocks_per_sm": b.value, "groups_A": g[0::2].copy(), "groups_AT": g[1::2].copy()}

    def autotune(self, iters: int = 30) -> dict:
        """Pick row-split schedules per instance-size class by timing (gb_batch_autotune)."""
        k = len(self.lps)
        bn = np.zeros(2 * k, dtype=np.int32)
        mr = np.zeros(2 * k, dtype=np.int32)
        t0, t1 = np.zeros(2), np.zeros(2)
        _check(self._lib.gb_batch_autotune(self._h, int(iters), _p(bn), _p(mr), _p(t0), _p(t1)))
        return {"block_nnz": bn[:k], "max_rows": mr[:k], "block_nnz_f64": bn[k:], "max_rows_f64": mr[k:],
                "ms_per_iter_default": float(t0[0]), "ms_per_iter_tuned": float(t1[0]),
                "ms_per_iter_default_f64": float(t0[1]), "ms_per_iter_tuned_f64": float(t1[1]),
                "load_modes": self.load_modes()}

    def load_modes(self) -> dict:
        """Load variant per matrix and precision class (gb_batch_load_modes)."""
        m = np.zeros(4, dtype=np.int32)
        _check(self._lib.gb_batch_load_modes(self._h, _p(m)))
        return _load_mode_names(m)

    def time_kernels(self, level: int = 0, iters: int = 50) -> dict:
        """Device time of the fused iteration kernels with every instance active."""
        mp, md, bpi = C.c_double(), C.c_double(), C.c_double()
        nl = C.c_int64()
        _check(self._lib.gb_batch_time_kernels(self._h, int(level), int(iters), C.byref(mp), C.byref(md),
                                               C.byref(nl), C.byref(bpi)))
        return {"ms_primal": mp.value, "ms_dual": md.value, "launches": nl.value, "bytes_per_iter": bpi.value}

    def time_kernels_graph(self, level: int = 0, iters: int = 100) -> dict:
        """Back-to-back launches captured in CUDA graphs (gb_batch_time_kernels_graph)."""
        mp, md, mi = C.c_double(), C.c_double(), C.c_double()
        _check(self._lib.gb_batch_time_kernels_graph(self._h, int(level), int(iters), C.byref(mp), C.byref(md),
                                                     C.byref(mi)))
        return {"ms_primal": mp.value, "ms_dual": md.value, "ms_iteration": mi.value}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.gb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class DiffSolver:
    """Differentiable batch of LPs (gb_diff_*).

    ``forward`` solves every instance with restarted PDHG to ``opt.tol`` and
    then runs ``tail_iters`` (K) plain FP64 PDHG iterations, checkpointed every
    ``ckpt_every`` (R); its outputs are the last tail iterate.  ``backward``
    maps dL/dx*, dL/dy* to dL/dc, dL/dlo, dL/dhi and dL/d(A values) by exact
    reverse mode through the K tail iterations plus the implicit completion
    at the tail start (``implicit_iters`` MINRES steps at most, relative
    residual ``implicit_tol``; ``implicit_iters=0`` gives the truncated
    gradient).  With ``polish`` the tail starts from the vertex of the active
    set the solver's point identifies, when that vertex certifies better.
    All vectors are the concatenation of the instances' vectors.  LPs must
    not use a Hessian."""

    def __init__(self, lps, opt: Options | None = None, tail_iters: int = 200, ckpt_every: int = 20,
                 implicit_iters: int = 20000, implicit_tol: float = 1e-10, polish: bool = True):
        self._lib = load_library()
        self.lps = list(lps)
        self._views = [_LpView(lp) for lp in self.lps]
        arr = (_GbLp * len(self._views))(*[v.s for v in self._views])
        o = _opts(opt)
        h = C.c_void_p()
        _check(self._lib.gb_diff_create(len(self._views), arr, C.addressof(o), int(tail_iters), int(ckpt_every),
                                        C.byref(h)))
        self._h = h
        self.n_off = np.concatenate([[0], np.cumsum([lp.n for lp in self.lps])]).astype(np.int64)
        self.m_off = np.concatenate([[0], np.cumsum([lp.m for lp in self.lps])]).astype(np.int64)
        self.nnz_off = np.concatenate([[0], np.cumsum([lp.A.nnz for lp in self.lps])]).astype(np.int64)
        self.set_options(implicit_iters, implicit_tol, polish)

    def __len__(self):
        return len(self.lps)

    def set_options(self, implicit_iters: int = 20000, implicit_tol: float = 1e-10, polish: bool = True):
        o = _GbDiffOptions(int(implicit_iters), float(implicit_tol), int(bool(polish)), 0)
        _check(self._lib.gb_diff_set_options(self._h, C.byref(o)))

    def forward(self, opt: Options | None = None):
        """Returns (results, x, y): per-instance results and the concatenated x*, y*."""
        o = _opts(opt)
        res = (_GbResult * len(self.lps))()
        x = np.zeros(int(self.n_off[-1]))
        y = np.zeros(int(self.m_off[-1]))
        _check(self._lib.gb_diff_forward(self._h, C.addressof(o), res, _p(x), _p(y)))
        out = [_result(r, x[self.n_off[i]:self.n_off[i + 1]], y[self.m_off[i]:self.m_off[i + 1]])
               for i, r in enumerate(res)]
        return out, x, y

    def backward(self, dl_dx=None, dl_dy=None) -> dict:
        """Returns {"c", "lo", "hi", "a_val"} gradients (concatenated)."""
        gx = None if dl_dx is None else np.ascontiguousarray(dl_dx, dtype=np.float64)
        gy = None if dl_dy is None else np.ascontiguousarray(dl_dy, dtype=np.float64)
        if gx is not None and gx.shape != (int(self.n_off[-1]),):
            raise ValueError("dl_dx must have the total column count")
        if gy is not None and gy.shape != (int(self.m_off[-1]),):
            raise ValueError("dl_dy must have the total row count")
        out = {"c": np.zeros(int(self.n_off[-1])), "lo": np.zeros(int(self.m_off[-1])),
               "hi": np.zeros(int(self.m_off[-1])), "a_val": np.zeros(int(self.nnz_off[-1]))}
        _check(self._lib.gb_diff_backward(self._h, _p(gx), _p(gy), _p(out["c"]), _p(out["lo"]), _p(out["hi"]),
                                          _p(out["a_val"])))
        return out

    def info(self, i: int) -> dict:
        r = _GbDiffInfo()
        _check(self._lib.gb_diff_get_info(self._h, int(i), C.byref(r)))
        return {k: getattr(r, k) for k, _ in _GbDiffInfo._fields_ if k != "pad"}

    def tail_start(self):
        """Scaled start point (x, y) of the tail iterations (concatenated)."""
        x = np.zeros(int(self.n_off[-1]))
        y = np.zeros(int(self.m_off[-1]))
        _check(self._lib.gb_diff_tail_start(self._h, _p(x), _p(y)))
        return x, y

    def close(self):
        if getattr(self, "_h", None):
            self._lib.gb_diff_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


# ---------------------------------------------------------------- Backend concept
class Vec:
    def __init__(self, be: "Backend", h):
        self.be = be
        self._h = h

    @property
    def size(self) -> int:
        return self.be._lib.gb_vec_size(self._h)

    def to_host(self) -> np.ndarray:
        out = np.zeros(self.size)
        _check(self.be._lib.gb_vec_to_host(self.be._h, self._h, _p(out)))
        return out

    def __del__(self):
        try:
            if self._h:
                self.be._lib.gb_vec_destroy(self._h)
                self._h = None
        except Exception:
            pass


class Backend:
    """The Backend concept of src/pdhg_impl.hpp on B200 kernels.

    ``scaled`` is a dict with the ScaledLP arrays (src/scaling.hpp:8-23):
    A, AT (Csr), optional Q (Csr), c, l, u, lo, hi, Rres, Cres.  ``mat`` and
    ``vec`` are "f32" / "f64" (L1 = f32/f32, L2 = f32/f64, L3 = f64/f64)."""

    def __init__(self, scaled: dict, mat: str = "f64", vec: str = "f64"):
        self._lib = load_library()
        self._keep = []

        def k(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            self._keep.append(a)
            return _p(a)

        A, AT, Q = scaled["A"], scaled["AT"], scaled.get("Q")
        self.m, self.n = A.rows, A.cols
        s = _GbScaledLp(A.rows, A.cols, k(A.ptr, np.int32), k(A.idx, np.int32), k(A.val, np.float64),
                        k(AT.ptr, np.int32), k(AT.idx, np.int32), k(AT.val, np.float64),
                        k(Q.ptr, np.int32) if Q is not None else None, k(Q.idx, np.int32) if Q is not None else None,
                        k(Q.val, np.float64) if Q is not None else None,
                        *[k(scaled[n], np.float64) for n in ("c", "l", "u", "lo", "hi", "Rres", "Cres")])
        h = C.c_void_p()
        _check(self._lib.gb_backend_create(C.addressof(s), 0 if mat == "f32" else 1, 0 if vec == "f32" else 1,
                                           C.byref(h)))
        self._h = h

    def zeros(self, k: int) -> Vec:
        h = C.c_void_p()
        _check(self._lib.gb_vec_zeros(self._h, int(k), C.byref(h)))
        return Vec(self, h)

    def from_host(self, a) -> Vec:
        a = np.ascontiguousarray(a, dtype=np.float64)
        h = C.c_void_p()
        _check(self._lib.gb_vec_from_host(self._h, _p(a), int(a.shape[0]), C.byref(h)))
        return Vec(self, h)

    def to_host(self, v: Vec) -> np.ndarray:
        return v.to_host()

    def copy(self, src: Vec, dst: Vec):
        _check(self._lib.gb_copy(self._h, src._h, dst._h))

    def fill(self, v: Vec, a: float):
        _check(self._lib.gb_fill(self._h, v._h, float(a)))

    def spmv_A(self, x, ax):
        _check(self._lib.gb_spmv_A(self._h, x._h, ax._h))

    def spmv_AT(self, y, aty):
        _check(self._lib.gb_spmv_AT(self._h, y._h, aty._h))

    def spmv_Q(self, x, qx):
        _check(self._lib.gb_spmv_Q(self._h, x._h, qx._h))

    def primal_step(self, x, aty, qx, tau, xn, xbar, sumx):
        _check(self._lib.gb_primal_step(self._h, x._h, aty._h, qx._h if qx is not None else None, float(tau),
                                        xn._h, xbar._h, sumx._h))

    def dual_step(self, y, axbar, sigma, yn, sumy):
        _check(self._lib.gb_dual_step(self._h, y._h, axbar._h, float(sigma), yn._h, sumy._h))

    def sub(self, a, b, d):
        _check(self._lib.gb_sub(self._h, a._h, b._h, d._h))

    def scale_into(self, src, a, dst):
        _check(self._lib.gb_scale_into(self._h, src._h, float(a), dst._h))

    def _r1(self, fn, *args):
        out = C.c_double()
        _check(fn(self._h, *args, C.byref(out)))
        return out.value

    def primal_res2(self, ax):
        return self._r1(self._lib.gb_primal_res2, ax._h)

    def dual_res(self, aty, qx=None, with_c=True):
        a, b = C.c_double(), C.c_double()
        _check(self._lib.gb_dual_res(self._h, aty._h, qx._h if qx is not None else None, int(with_c), C.byref(a),
                                     C.byref(b)))
        return a.value, b.value

    def row_dual_obj(self, y):
        return self._r1(self._lib.gb_row_dual_obj, y._h)

    def dot(self, a, b):
        return self._r1(self._lib.gb_dot, a._h, b._h)

    def dot_c(self, x):
        return self._r1(self._lib.gb_dot_c, x._h)

    def diff2(self, a, b):
        return self._r1(self._lib.gb_diff2, a._h, b._h)

    def __del__(self):
        try:
            if self._h:
                self._lib.gb_backend_destroy(self._h)
                self._h = None
        except Exception:
            pass
