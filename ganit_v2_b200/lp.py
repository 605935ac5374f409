"""Host-side LP / QP container mirroring GANIT's ``ganit::LP`` and ``ganit::Csr``.

Reference: include/ganit/lp.hpp:19-47 (``Csr``: int32 ``ptr``/``idx`` and
float64 ``val``; ``LP``: ``min c'x + 0.5 x'Qx + obj_const`` subject to
``lo <= A x <= hi`` and ``l <= x <= u``, bounds may be +-inf).

Besides the reference's full-storage CSR Hessian ``Q`` this container can also
carry a diagonal-plus-low-rank Hessian ``Q = 2 (F F^T + diag(D))`` (``F`` is
n x k, row-major), which the B200 engine applies with a dedicated kernel
instead of storing the dense n x n product.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np


@dataclass
class Csr:
    """Compressed sparse row matrix (lp.hpp:19-25)."""

    rows: int
    cols: int
    ptr: np.ndarray  # int32[rows+1]
    idx: np.ndarray  # int32[nnz]
    val: np.ndarray  # float64[nnz]

    def __post_init__(self):
        self.ptr = np.ascontiguousarray(self.ptr, dtype=np.int32)
        self.idx = np.ascontiguousarray(self.idx, dtype=np.int32)
        self.val = np.ascontiguousarray(self.val, dtype=np.float64)
        if self.ptr.shape != (self.rows + 1,):
            raise ValueError("Csr.ptr must have rows+1 entries")
        if self.idx.shape != self.val.shape or self.idx.shape[0] != int(self.ptr[-1]):
            raise ValueError("Csr.idx/val must have ptr[rows] entries")

    @property
    def nnz(self) -> int:
        return int(self.val.shape[0])

    @staticmethod
    def from_scipy(a) -> "Csr":
        a = a.tocsr()
        a.sum_duplicates()
        a.sort_indices()
        return Csr(a.shape[0], a.shape[1], a.indptr, a.indices, a.data)

    def to_scipy(self):
        import scipy.sparse as sp

        return sp.csr_matrix((self.val, self.idx, self.ptr), shape=(self.rows, self.cols))

    def transpose(self) -> "Csr":
        """Counting-sort transpose (lp.cpp:55-72): entries of each output row
        come in increasing source-row order."""
        counts = np.bincount(self.idx, minlength=self.cols)
        ptr = np.zeros(self.cols + 1, dtype=np.int64)
        np.cumsum(counts, out=ptr[1:])
        rows_of = np.repeat(np.arange(self.rows, dtype=np.int32), np.diff(self.ptr))
        order = np.argsort(self.idx, kind="stable")
        return Csr(self.cols, self.rows, ptr.astype(np.int32), rows_of[order], self.val[order])


@dataclass
class LP:
    """LP / convex QP in GANIT's form (lp.hpp:27-47)."""

    A: Csr
    c: np.ndarray
    l: np.ndarray
    u: np.ndarray
    lo: np.ndarray
    hi: np.ndarray
    obj_const: float = 0.0
    maximize: bool = False
    Q: Optional[Csr] = None          # full-storage symmetric Hessian (reference form)
    F: Optional[np.ndarray] = None   # n x k factor matrix of Q = 2 (F F^T + diag(D))
    D: Optional[np.ndarray] = None   # n diagonal of the same
    name: str = "lp"
    meta: dict = field(default_factory=dict)
    is_int: Optional[np.ndarray] = None  # n bools: integer columns of a MILP (the LP solvers ignore them)

    def __post_init__(self):
        for k in ("c", "l", "u", "lo", "hi"):
            setattr(self, k, np.ascontiguousarray(getattr(self, k), dtype=np.float64))
        if self.c.shape != (self.n,) or self.l.shape != (self.n,) or self.u.shape != (self.n,):
            raise ValueError("c, l, u must have n entries")
        if self.lo.shape != (self.m,) or self.hi.shape != (self.m,):
            raise ValueError("lo, hi must have m entries")
        if self.F is not None:
            self.F = np.ascontiguousarray(self.F, dtype=np.float64)
            self.D = np.ascontiguousarray(self.D, dtype=np.float64)
            if self.F.ndim != 2 or self.F.shape[0] != self.n or self.D.shape != (self.n,):
                raise ValueError("F must be n x k and D must have n entries")

    @property
    def m(self) -> int:
        return self.A.rows

    @property
    def n(self) -> int:
        return self.A.cols

    def has_q(self) -> bool:
        return (self.Q is not None and self.Q.nnz > 0) or self.F is not None

    def objective(self, x: np.ndarray) -> float:
        """Objective value c'x + 0.5 x'Qx + obj_const in the original space."""
        v = float(self.c @ x)
        if self.Q is not None and self.Q.nnz:
            v += 0.5 * float(x @ (self.Q.to_scipy() @ x))
        if self.F is not None:
            fx = self.F.T @ x
            v += float(fx @ fx) + float(self.D @ (x * x))
        return v + self.obj_const
