"""Batched LP layer for PyTorch: (c, lo, hi, A values) -> (x*, y*) with gradients.

Forward and backward run on the B200 through :class:`DiffSolver`
(``gb_diff_forward`` / ``gb_diff_backward``); torch is only the autograd
plumbing.  Every instance keeps the sparsity pattern and the column boxes
``l <= x <= u`` of its template LP; the differentiable inputs are the
concatenated cost vectors ``c``, row bounds ``lo`` / ``hi`` (pass the same
tensor for both to tie the two sides of equality rows to one ``b``) and
matrix values ``a_val`` (CSR order of the templates).
"""
from __future__ import annotations

import numpy as np
import torch
from torch.autograd.function import once_differentiable

from .api import DiffSolver, Options
from .lp import LP, Csr


class LPLayer:
    """Batch of LPs solved by restarted PDHG, differentiable in c, lo, hi and A."""

    def __init__(self, templates, opt: Options | None = None, tail_iters: int = 200, ckpt_every: int = 20,
                 implicit_iters: int = 20000, implicit_tol: float = 1e-10, polish: bool = True):
        self.templates = list(templates)
        for lp in self.templates:
            if lp.Q is not None or lp.F is not None:
                raise ValueError("LPLayer takes LPs only")
        self.opt = opt or Options(tol=1e-6)
        self.tail_iters, self.ckpt_every = int(tail_iters), int(ckpt_every)
        self.implicit_iters, self.implicit_tol = int(implicit_iters), float(implicit_tol)
        self.polish = bool(polish)
        self.n_off = np.concatenate([[0], np.cumsum([lp.n for lp in self.templates])]).astype(np.int64)
        self.m_off = np.concatenate([[0], np.cumsum([lp.m for lp in self.templates])]).astype(np.int64)
        self.z_off = np.concatenate([[0], np.cumsum([lp.A.nnz for lp in self.templates])]).astype(np.int64)
        self.last_results = None
        self.last_solver = None

    def template_parameters(self, device="cpu"):
        """(c, lo, hi, a_val) of the templates as float64 tensors."""
        cat = lambda k: torch.from_numpy(np.concatenate([np.asarray(getattr(lp, k), np.float64)
                                                         for lp in self.templates])).to(device)
        a = torch.from_numpy(np.concatenate([np.asarray(lp.A.val, np.float64) for lp in self.templates])).to(device)
        return cat("c"), cat("lo"), cat("hi"), a

    def instances(self, c, lo, hi, a_val) -> list:
        """LP objects of the batch for the given concatenated data (numpy)."""
        out = []
        for i, t in enumerate(self.templates):
            n0, n1 = self.n_off[i], self.n_off[i + 1]
            m0, m1 = self.m_off[i], self.m_off[i + 1]
            z0, z1 = self.z_off[i], self.z_off[i + 1]
            A = Csr(t.m, t.n, t.A.ptr, t.A.idx, np.ascontiguousarray(a_val[z0:z1]))
            out.append(LP(A, np.ascontiguousarray(c[n0:n1]), t.l, t.u, np.ascontiguousarray(lo[m0:m1]),
                          np.ascontiguousarray(hi[m0:m1]), obj_const=t.obj_const, maximize=t.maximize,
                          name=t.name))
        return out

    def __call__(self, c, lo, hi, a_val):
        return LPFunction.apply(self, c, lo, hi, a_val)


def _np(t):
    return None if t is None else t.detach().to("cpu", torch.float64).contiguous().numpy()


class LPFunction(torch.autograd.Function):
    """forward: gb_diff_forward; backward: gb_diff_backward."""

    @staticmethod
    def forward(ctx, layer: LPLayer, c, lo, hi, a_val):
        solver = DiffSolver(layer.instances(_np(c), _np(lo), _np(hi), _np(a_val)), layer.opt, layer.tail_iters,
                            layer.ckpt_every, layer.implicit_iters, layer.implicit_tol, layer.polish)
        results, x, y = solver.forward(layer.opt)
        layer.last_results, layer.last_solver = results, solver
        ctx.solver = solver
        ctx.device = c.device
        return torch.from_numpy(x).to(c.device), torch.from_numpy(y).to(c.device)

    @staticmethod
    @once_differentiable
    def backward(ctx, gx, gy):
        g = ctx.solver.backward(_np(gx), _np(gy))
        to = lambda a: torch.from_numpy(a).to(ctx.device)
        return None, to(g["c"]), to(g["lo"]), to(g["hi"]), to(g["a_val"])
