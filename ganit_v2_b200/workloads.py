"""Seeded synthetic LP / QP workloads for the PDHG engine.

All generators use ``numpy.random.default_rng(seed)`` and return
:class:`ganit_v2_b200.lp.LP` objects.  They stand in for the reference's
generated benchmark models (bench/gen_blending.py, bench/gen_portfolio.py) and
for the random feasible LPs the engine is measured on:

* :func:`random_feasible_lp` -- feasible-by-construction random LP
  (m rows, half equalities and half ``<=`` rows, n columns boxed in [0, 10],
  a fixed number of N(0,1) nonzeros per column at distinct random rows).
* :func:`blending_lp` -- multi-period crude-blending LP with the row / column
  structure of bench/gen_blending.py:4-15, 63-100 (crude balance, product
  balance, quality-spec rows, CDU capacity, inventory links t -> t+1).
* :func:`portfolio_qp` -- factor-model portfolio QP, either in the engine's
  diagonal-plus-low-rank form or in the lifted form of
  bench/gen_portfolio.py:4-8 that the reference can read.
* :func:`lp_batch` -- many random feasible LPs of log-uniform size.
* :func:`nondegenerate_lp` / :func:`diff_batch` -- random LPs of the same
  shape whose optimum is a unique, strictly complementary vertex (the
  instances on which solution derivatives exist and equal basis
  sensitivities).

Dual sign convention (reference backend_cpu.cpp:73, 81-92): the reduced cost is
``c - A^T y``, so the dual of a ``<=`` row is <= 0.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .lp import LP, Csr


def _distinct_rows(rng, n_cols: int, m: int, k_per_col: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """For column j draw k_per_col[j] distinct row indices in [0, m)."""
    kmax = int(k_per_col.max()) if n_cols else 0
    if kmax > m:
        raise ValueError("more nonzeros per column than rows")
    r = rng.integers(0, m, size=(n_cols, kmax))
    active = np.arange(kmax)[None, :] < k_per_col[:, None]
    for _ in range(1000):
        # duplicates among the active entries of a column are re-drawn
        key = np.where(active, r, m + np.arange(kmax)[None, :])
        order = np.argsort(key, axis=1, kind="stable")
        srt = np.take_along_axis(key, order, axis=1)
        dup_sorted = np.zeros_like(srt, dtype=bool)
        dup_sorted[:, 1:] = srt[:, 1:] == srt[:, :-1]
        if not dup_sorted.any():
            break
        dup = np.zeros_like(dup_sorted)
        np.put_along_axis(dup, order, dup_sorted, axis=1)
        r[dup] = rng.integers(0, m, size=int(dup.sum()))
    cols = np.repeat(np.arange(n_cols), kmax).reshape(n_cols, kmax)
    return r[active], cols[active]


def random_feasible_lp(m: int = 2000, n: int = 5000, nnz_per_col=8, seed: int = 0, ub: float = 10.0,
                       eq_frac: float = 0.5, bound_frac: float = 0.3, name: str | None = None,
                       free_frac: float = 0.0) -> LP:
    """Feasible-by-construction random LP.

    Rows ``[0, m*eq_frac)`` are equalities, the rest ``<=`` rows.  Columns are
    boxed ``0 <= x <= ub``.  A point ``x0 ~ U(0, ub)`` with ``bound_frac`` of its
    entries moved to a bound (half to 0, half to ub) fixes ``b = A x0`` (plus
    ``U(0,1)`` slack on ``<=`` rows).  A dual point ``y0 ~ N(0,1)`` (``<= 0`` on
    ``<=`` rows) and reduced costs ``s0`` complementary to ``x0`` give
    ``c = A^T y0 + s0``.  ``nnz_per_col`` is an int or an array of per-column
    counts.  ``free_frac`` of the columns (drawn after everything else, so
    the default stream is unchanged) become free (-inf, +inf) with zero
    reduced cost, which keeps the LP bounded.
    """
    rng = np.random.default_rng(seed)
    k = np.full(n, nnz_per_col, dtype=np.int64) if np.isscalar(nnz_per_col) else np.asarray(nnz_per_col)
    rows, cols = _distinct_rows(rng, n, m, k)
    vals = rng.standard_normal(rows.shape[0])
    A = sp.csr_matrix((vals, (rows, cols)), shape=(m, n))
    A.sum_duplicates()
    A.sort_indices()
    n_eq = int(round(m * eq_frac))

    x0 = rng.uniform(0.0, ub, size=n)
    at_bound = rng.random(n) < bound_frac
    at_upper = at_bound & (rng.random(n) < 0.5)
    at_lower = at_bound & ~at_upper
    x0[at_lower] = 0.0
    x0[at_upper] = ub
    b = A @ x0
    slack = np.zeros(m)
    slack[n_eq:] = rng.uniform(0.0, 1.0, size=m - n_eq)
    b = b + slack

    y0 = rng.standard_normal(m)
    y0[n_eq:] = -np.abs(y0[n_eq:])
    s0 = np.zeros(n)
    s0[at_lower] = np.abs(rng.standard_normal(int(at_lower.sum())))
    s0[at_upper] = -np.abs(rng.standard_normal(int(at_upper.sum())))
    c = A.T @ y0 + s0

    lo = np.empty(m)
    hi = b.copy()
    lo[:n_eq] = b[:n_eq]
    lo[n_eq:] = -np.inf
    l = np.zeros(n)
    u = np.full(n, ub)
    if free_frac > 0:
        free = (rng.random(n) < free_frac) & ~at_bound
        l[free] = -np.inf
        u[free] = np.inf
        c = c - s0 * free  # s0 is already 0 there; kept explicit
    return LP(Csr.from_scipy(A), c, l, u, lo, hi,
              name=name or f"rand_m{m}_n{n}_s{seed}", meta={"x0": x0, "y0": y0})


def blending_lp(crudes: int = 60, products: int = 16, specs: int = 5, periods: int = 365, seed: int = 1,
                name: str | None = None) -> LP:
    """Multi-period crude-blending LP.

    Variables per period t: ``buy[c]`` (<= supply), ``inv[c]`` (<= tank), flows
    ``x[c,p]`` (free above 0), ``sell[p]`` (<= demand), ``pinv[p]`` (<= tank).
    Rows per period: CDU capacity ``sum x <= cap``, crude balance
    ``inv[c,t-1] + buy - sum_p x - inv[c,t] = 0``, product balance
    ``pinv[p,t-1] + sum_c x - sell - pinv[p,t] = 0``, quality specs
    ``sum_c (q[c,k] - s[p,k]) x[c,p] <= 0``.  Distributions: q ~ U(0,1) with
    crude 0 light (0.05) so every spec stays satisfiable, s ~ U(0.3,0.7), crude
    cost ~ U(1,100), product price ~ U(60,160).  At 60/16/5/365: m = 57,305,
    n = 405,880, nnz = 2,886,344.
    """
    rng = np.random.default_rng(seed)
    C, P, K, T = crudes, products, specs, periods
    q = rng.uniform(0.0, 1.0, size=(C, K))
    q[0, :] = 0.05
    smax = rng.uniform(0.3, 0.7, size=(P, K))
    cost = rng.uniform(1.0, 100.0, size=C)
    price = rng.uniform(60.0, 160.0, size=P)
    cap = 1000.0 * P
    coef = q[:, None, :] - smax[None, :, :]  # C x P x K

    rows_per = 1 + C + P + P * K
    cols_per = C * (2 + P) + 2 * P
    m, n = rows_per * T, cols_per * T
    # row offsets inside a period
    r_cap, r_cb, r_pb, r_q = 0, 1, 1 + C, 1 + C + P
    # column offsets inside a period: for each crude [buy, inv, x_0..x_{P-1}], then for each product [sell, pinv]
    c_crude = np.arange(C) * (2 + P)
    c_prod = C * (2 + P) + np.arange(P) * 2

    R, Cc, V = [], [], []
    obj = np.zeros(n)
    ub = np.full(n, np.inf)
    for t in range(T):
        r0, c0 = t * rows_per, t * cols_per
        nxt = t + 1 < T
        buy = c0 + c_crude
        inv = buy + 1
        R += [r0 + r_cb + np.arange(C)]; Cc += [buy]; V += [np.ones(C)]
        obj[buy] = cost * rng.uniform(0.9, 1.1, size=C)
        ub[buy] = rng.uniform(200.0, 1500.0, size=C)
        R += [r0 + r_cb + np.arange(C)]; Cc += [inv]; V += [-np.ones(C)]
        if nxt:
            R += [r0 + rows_per + r_cb + np.arange(C)]; Cc += [inv]; V += [np.ones(C)]
        obj[inv] = 0.2
        ub[inv] = 5000.0
        xc = (buy[:, None] + 2 + np.arange(P)[None, :])  # C x P column ids
        cc = np.repeat(np.arange(C), P)
        pp = np.tile(np.arange(P), C)
        xcol = xc.ravel()
        R += [r0 + r_cb + cc]; Cc += [xcol]; V += [-np.ones(C * P)]
        R += [r0 + r_pb + pp]; Cc += [xcol]; V += [np.ones(C * P)]
        R += [np.full(C * P, r0 + r_cap)]; Cc += [xcol]; V += [np.ones(C * P)]
        for k in range(K):
            cf = coef[cc, pp, k]
            keep = np.abs(cf) > 1e-12
            R += [r0 + r_q + pp[keep] * K + k]; Cc += [xcol[keep]]; V += [cf[keep]]
        sell = c0 + c_prod
        pinv = sell + 1
        R += [r0 + r_pb + np.arange(P)]; Cc += [sell]; V += [-np.ones(P)]
        obj[sell] = -price * rng.uniform(0.95, 1.05, size=P)
        ub[sell] = rng.uniform(300.0, 1200.0, size=P)
        R += [r0 + r_pb + np.arange(P)]; Cc += [pinv]; V += [-np.ones(P)]
        if nxt:
            R += [r0 + rows_per + r_pb + np.arange(P)]; Cc += [pinv]; V += [np.ones(P)]
        obj[pinv] = 0.5
        ub[pinv] = 3000.0
    A = sp.csr_matrix((np.concatenate(V), (np.concatenate(R), np.concatenate(Cc))), shape=(m, n))
    A.sum_duplicates()
    A.sort_indices()
    lo = np.zeros(m)
    hi = np.zeros(m)
    for t in range(T):
        r0 = t * rows_per
        lo[r0 + r_cap] = -np.inf
        hi[r0 + r_cap] = cap
        lo[r0 + r_q: r0 + rows_per] = -np.inf
    return LP(Csr.from_scipy(A), obj, np.zeros(n), ub, lo, hi, name=name or f"blend_C{C}_P{P}_K{K}_T{T}")


def portfolio_qp(assets: int = 100_000, factors: int = 50, seed: int = 7, gamma: float = 1.0,
                 max_weight: float = 0.05, lifted: bool = False, name: str | None = None) -> LP:
    """Factor-model portfolio QP: ``min x'(F F^T + D) x - gamma mu'x``,
    ``sum x = 1``, ``0 <= x <= max_weight``, with F ~ N(0, 0.1^2),
    D ~ U(0.01, 0.1), mu ~ N(0.05, 0.02^2).

    ``lifted=False`` returns the engine's form (one budget row, DPLR Hessian
    ``Q = 2 (F F^T + diag(D))``).  ``lifted=True`` returns the equivalent QP over
    ``(x, f)`` with rows ``f - F^T x = 0`` and Hessian ``diag(2D, 2I)`` (the form
    of bench/gen_portfolio.py:4-8), which a full-storage CSR Hessian can hold.
    """
    rng = np.random.default_rng(seed)
    N, K = assets, factors
    F = rng.normal(0.0, 0.1, size=(N, K))
    D = rng.uniform(0.01, 0.1, size=N)
    mu = rng.normal(0.05, 0.02, size=N)
    if not lifted:
        A = Csr(1, N, np.array([0, N]), np.arange(N), np.ones(N))
        return LP(A, -gamma * mu, np.zeros(N), np.full(N, max_weight), np.ones(1), np.ones(1), F=F, D=D,
                  name=name or f"port_N{N}_K{K}")
    # rows: 0 = budget, 1..K = factor definitions f_k - sum_i F_ik x_i = 0
    nx = N + K
    budget = sp.csr_matrix((np.ones(N), (np.zeros(N, dtype=np.int64), np.arange(N))), shape=(1, nx))
    fac = sp.hstack([sp.csr_matrix(-F.T), sp.identity(K, format="csr")], format="csr")
    A = sp.vstack([budget, fac], format="csr")
    qd = np.concatenate([2.0 * D, 2.0 * np.ones(K)])
    Q = Csr(nx, nx, np.arange(nx + 1), np.arange(nx), qd)
    c = np.concatenate([-gamma * mu, np.zeros(K)])
    l = np.concatenate([np.zeros(N), np.full(K, -np.inf)])
    u = np.concatenate([np.full(N, max_weight), np.full(K, np.inf)])
    lo = np.concatenate([[1.0], np.zeros(K)])
    hi = lo.copy()
    return LP(Csr.from_scipy(A), c, l, u, lo, hi, Q=Q, name=name or f"port_lifted_N{N}_K{K}")


def lp_batch(count: int = 512, seed: int = 1000, m_min: int = 50, m_max: int = 4000, n_ratio: float = 2.5,
             k_min: int = 4, k_max: int = 12) -> list[LP]:
    """``count`` random feasible LPs with m log-uniform in [m_min, m_max],
    n = round(n_ratio * m) and U{k_min..k_max} nonzeros per column; instance i
    is generated from seed ``seed + i``."""
    out = []
    for i in range(count):
        rng = np.random.default_rng(seed + i)
        m = int(round(float(np.exp(rng.uniform(np.log(m_min), np.log(m_max))))))
        n = int(round(n_ratio * m))
        k = rng.integers(k_min, k_max + 1, size=n)
        k = np.minimum(k, m)
        out.append(random_feasible_lp(m, n, k, seed=seed + i, name=f"batch{i}_m{m}_n{n}"))
    return out


def nondegenerate_lp(m: int = 500, n: int = 1000, nnz_per_col: int = 10, seed: int = 0, ub: float = 10.0,
                     eq_frac: float = 0.5, tight_frac: float = 0.8, max_cond: float | None = None,
                     name: str | None = None) -> LP:
    """Random LP whose optimum (x0, y0) is a nondegenerate vertex.

    Same matrix family as :func:`random_feasible_lp` (N(0,1) values, a fixed
    count of distinct random rows per column, boxes [0, ub], the first
    ``eq_frac`` of the rows equalities, the rest ``<=``).  That generator makes
    every column with x0 strictly inside its box carry zero reduced cost, so
    its optimal face has dimension (#interior - #tight rows), about 200 at
    m=500, n=1000, and the solution map has no derivative.  Here instead:

    * ``tight`` rows: all equalities and a ``tight_frac`` share of the ``<=``
      rows, whose duals y0 are nonzero (<= -0.1 on ``<=`` rows); the other
      ``<=`` rows get y0 = 0 and slack U(0.1, 1);
    * exactly #tight columns are interior, x0 ~ U(0.1 ub, 0.9 ub); the rest
      sit at 0 or ub with reduced costs |s0| ~ U(0.1, 1) of the right sign;
    * the basis matrix A[tight, interior] is checked nonsingular by a sparse
      LU and the draw is repeated (same stream) otherwise; with ``max_cond``
      set, draws whose 1-norm condition estimate ||B||_1 ||B^-1||_1
      (scipy's onenormest) exceeds it are repeated too (PDHG's iteration
      count grows with that condition number).

    Then c = A^T y0 + s0 and x0, y0 are the unique optimal pair with strict
    complementarity.  ``meta`` holds x0, y0 and the boolean masks.
    """
    import scipy.sparse.linalg as spla

    rng = np.random.default_rng(seed)
    k = np.full(n, nnz_per_col, dtype=np.int64)
    n_eq = int(round(m * eq_frac))
    for _ in range(100):
        rows, cols = _distinct_rows(rng, n, m, k)
        vals = rng.standard_normal(rows.shape[0])
        A = sp.csr_matrix((vals, (rows, cols)), shape=(m, n))
        A.sum_duplicates()
        A.sort_indices()
        tight = np.ones(m, dtype=bool)
        tight[n_eq:] = rng.random(m - n_eq) < tight_frac
        r = int(tight.sum())
        if r > n:
            raise ValueError("more tight rows than columns")
        interior = np.zeros(n, dtype=bool)
        interior[rng.choice(n, r, replace=False)] = True
        B = A[np.flatnonzero(tight)][:, np.flatnonzero(interior)].tocsc()
        try:
            lu = spla.splu(B)
        except RuntimeError:
            continue
        if max_cond is not None:
            inv = spla.LinearOperator(B.shape, matvec=lu.solve, rmatvec=lambda v: lu.solve(v, trans="T"),
                                      dtype=np.float64)
            if spla.onenormest(inv) * spla.norm(B, 1) > max_cond:
                continue
        break
    else:
        raise RuntimeError("no nonsingular basis found")
    x0 = np.where(interior, rng.uniform(0.1 * ub, 0.9 * ub, size=n), 0.0)
    upper = ~interior & (rng.random(n) < 0.5)
    x0[upper] = ub
    y0 = rng.standard_normal(m)
    y0[n_eq:] = -np.abs(y0[n_eq:]) - 0.1
    y0[~tight] = 0.0
    s0 = rng.uniform(0.1, 1.0, size=n)
    s0[interior] = 0.0
    s0[upper] *= -1.0
    c = A.T @ y0 + s0
    b = A @ x0
    hi = b.copy()
    hi[~tight] += rng.uniform(0.1, 1.0, size=int((~tight).sum()))
    lo = np.where(np.arange(m) < n_eq, b, -np.inf)
    return LP(Csr.from_scipy(A), c, np.zeros(n), np.full(n, ub), lo, hi, name=name or f"nondeg_m{m}_n{n}_s{seed}",
              meta={"x0": x0, "y0": y0, "interior": interior, "tight": tight})


def diff_batch(count: int = 256, m: int = 500, n: int = 1000, nnz_per_col: int = 10, seed: int = 2000,
               max_cond: float | None = 5e4) -> list:
    """Batch of the differentiable-layer workload: ``count`` nondegenerate LPs
    of one shape, seeds ``seed + i``, basis 1-norm condition estimate <=
    ``max_cond``."""
    return [nondegenerate_lp(m, n, nnz_per_col, seed=seed + i, max_cond=max_cond) for i in range(count)]


def unbounded_lp(m: int = 200, n: int = 500, nnz_per_col: int = 6, seed: int = 4) -> LP:
    """Feasible LP with an unbounded objective (dual infeasible).

    A :func:`random_feasible_lp` plus two columns ``a`` and ``-a`` (a random
    sparse column), both in ``[0, inf)`` with costs ``(-1, 0)``: the ray
    ``d = e_{n} + e_{n+1}`` keeps ``A x`` fixed, stays in the bounds and
    lowers the objective without limit, while x0 (extended by zeros) stays
    feasible.  ``meta['ray']`` holds d."""
    base = random_feasible_lp(m, n, nnz_per_col, seed=seed)
    rng = np.random.default_rng(seed + 7919)
    A = base.A.to_scipy().tocsc()
    rows = rng.choice(m, size=min(nnz_per_col, m), replace=False)
    vals = rng.standard_normal(rows.shape[0])
    col = sp.csc_matrix((vals, (rows, np.zeros_like(rows))), shape=(m, 1))
    A2 = sp.hstack([A, col, -col], format="csr")
    A2.sort_indices()
    c = np.concatenate([base.c, [-1.0, 0.0]])
    l = np.concatenate([base.l, [0.0, 0.0]])
    u = np.concatenate([base.u, [np.inf, np.inf]])
    ray = np.zeros(n + 2)
    ray[n] = ray[n + 1] = 1.0
    return LP(Csr.from_scipy(A2), c, l, u, base.lo, base.hi, name=f"unbounded_m{m}_n{n}_s{seed}",
              meta={"x0": np.concatenate([base.meta["x0"], [0.0, 0.0]]), "ray": ray})


def infeasible_lp(m: int = 200, n: int = 500, seed: int = 3) -> LP:
    """A random feasible LP made primal infeasible by two contradicting rows
    ``a'x <= b - 1`` and ``a'x >= b`` on the same random row vector a."""
    base = random_feasible_lp(m, n, 6, seed=seed)
    A = base.A.to_scipy().tolil()
    rng = np.random.default_rng(seed + 99)
    cols = rng.choice(n, size=10, replace=False)
    a = np.zeros(n)
    a[cols] = rng.standard_normal(10)
    A = sp.vstack([A.tocsr(), sp.csr_matrix(a), sp.csr_matrix(a)], format="csr")
    bval = float(a @ base.meta["x0"])
    lo = np.concatenate([base.lo, [-np.inf, bval]])
    hi = np.concatenate([base.hi, [bval - 1.0, np.inf]])
    return LP(Csr.from_scipy(A), base.c, base.l, base.u, lo, hi, name=f"infeas_m{m}_n{n}_s{seed}")


def milp_node(n: int = 120, knapsacks: int = 8, density: float = 0.3, up_blocked: int = 2, down_blocked: int = 2,
              both_blocked: int = 0, seed: int = 11) -> LP:
    """Root node of a synthetic MILP for strong branching: a multi-dimensional
    knapsack (maximise profit, written as minimise -profit; integer columns in
    [0, U_j], U_j in {1, 2, 3}; rows W x <= 0.3 * W U) whose LP relaxation has
    fractional columns, plus three planted kinds of integer column:

    * ``up_blocked``: a row 5 x_j <= 3 (so x_j <= 0.6) and a high profit --
      the relaxation takes x_j = 0.6 and the up child (x_j >= 1) is infeasible;
    * ``down_blocked``: a row x_j >= 0.4 and a negative profit -- the relaxation
      takes x_j = 0.4 and the down child (x_j <= 0) is infeasible;
    * ``both_blocked``: both rows -- either child is infeasible.

    ``is_int`` marks every column; ``meta`` lists the planted columns."""
    rng = np.random.default_rng(seed)
    nk = n + up_blocked + down_blocked + both_blocked
    U = rng.integers(1, 4, size=nk).astype(np.float64)
    p = rng.uniform(1.0, 10.0, size=nk)
    W = sp.random(knapsacks, n, density=density, random_state=np.random.RandomState(seed),
                  data_rvs=lambda k: np.random.RandomState(seed + 1).uniform(1.0, 10.0, size=k)).tocsr()
    W = sp.hstack([W, sp.csr_matrix((knapsacks, nk - n))], format="csr")
    cap = 0.3 * (W @ U)
    up = np.arange(n, n + up_blocked)
    down = np.arange(n + up_blocked, n + up_blocked + down_blocked)
    both = np.arange(n + up_blocked + down_blocked, nk)
    U[up] = U[down] = U[both] = 1.0
    p[up] = 50.0
    p[down] = -1.0
    p[both] = 1.0
    rows = [W]
    lo = [np.full(knapsacks, -np.inf)]
    hi = [cap]
    for j in np.concatenate([up, both]):
        rows.append(sp.csr_matrix(([5.0], ([0], [j])), shape=(1, nk)))
        lo.append([-np.inf])
        hi.append([3.0])
    for j in np.concatenate([down, both]):
        rows.append(sp.csr_matrix(([1.0], ([0], [j])), shape=(1, nk)))
        lo.append([0.4])
        hi.append([np.inf])
    A = sp.vstack(rows, format="csr")
    A.sort_indices()
    return LP(Csr.from_scipy(A), -p, np.zeros(nk), U, np.concatenate(lo), np.concatenate(hi),
              name=f"milp_node_n{n}_k{knapsacks}_s{seed}", is_int=np.ones(nk, dtype=bool),
              meta={"up_blocked": up, "down_blocked": down, "both_blocked": both})
