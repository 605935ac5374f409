"""Instance sharding of LP batches over ranks (one process per GPU).

Batched instances are independent, so N GPUs split a batch with no exchange
during the iterations: a greedy longest-processing-time partition by
per-iteration work (nonzeros + rows + columns, what one PDHG iteration
streams) gives every rank its own resident block-diagonal batch; the only
collective is one gather of the per-instance results at the end.  A single
LP does not shard (its iterations would need an all-gather of x and y every
step) -- on N GPUs it runs as N replicas.
"""
from __future__ import annotations

from typing import Callable, Sequence


def instance_weight(lp) -> int:
    """Per-iteration work of one instance (matrix stream + vectors)."""
    return int(lp.A.nnz) + int(lp.m) + int(lp.n)


def partition(weights: Sequence[float], parts: int) -> list[list[int]]:
    """Greedy LPT: heaviest instance first, onto the least-loaded part (lowest
    index on ties).  Deterministic, so every rank computes the same split.
    Max load <= total / parts + max weight."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    load = [0.0] * parts
    out: list[list[int]] = [[] for _ in range(parts)]
    for i in order:
        r = min(range(parts), key=lambda p: (load[p], p))
        out[r].append(i)
        load[r] += weights[i]
    return [sorted(o) for o in out]


def _rank_world(group=None):
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def _batch_solve(lps, opt):
    from .api import BatchSolver

    with BatchSolver(lps, opt) as bs:
        return bs.solve(opt)


def shard_solve(lps: Sequence, opt=None, solve: Callable | None = None, group=None) -> list:
    """Solve a batch split over the ranks of the current process group.

    Every rank passes the full list; rank r solves partition(...)[r] with
    ``solve(list_of_lps, opt) -> list_of_results`` (default: one BatchSolver
    on this rank's GPU) and all ranks return the full result list, in input
    order, after one all_gather_object."""
    rank, world = _rank_world(group)
    parts = partition([instance_weight(lp) for lp in lps], world)
    mine = parts[rank]
    solve = solve or _batch_solve
    local = list(solve([lps[i] for i in mine], opt)) if mine else []
    if world == 1:
        return local
    import torch.distributed as dist

    gathered: list = [None] * world
    dist.all_gather_object(gathered, list(zip(mine, local)), group=group)
    out: list = [None] * len(lps)
    for part in gathered:
        for i, r in part:
            out[i] = r
    return out
