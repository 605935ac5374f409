"""Child process of tests/test_gpu_phase_lists.py: solves a workload and
prints a digest of every result bit (status, iterations, objective, x, y).
GANIT_B200_PHASE_LISTS is read once per process, hence the child."""
import hashlib
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import ganit_v2_b200 as gb  # noqa: E402
from ganit_v2_b200 import workloads as W  # noqa: E402


def digest(parts) -> str:
    h = hashlib.sha256()
    for p in parts:
        h.update(np.ascontiguousarray(p).tobytes())
    return h.hexdigest()


def main(which: str, tol: float) -> None:
    if which == "batch":
        lps = W.lp_batch(48, seed=77, m_min=40, m_max=600)
        with gb.BatchSolver(lps, gb.Options(tol=tol, precision=gb.Precision.Mixed)) as bs:
            res = bs.solve(gb.Options(tol=tol, precision=gb.Precision.Mixed))
            parts = []
            for i, r in enumerate(res):
                x, y = bs.solution(i)
                parts += [np.array([r.status, r.iterations, r.fp32_iterations]), np.array([r.pobj]), x, y]
    else:
        lps = W.diff_batch(256)  # its 1e-4 round ends with a few instances in the FP64 phase
        opt = gb.Options(tol=1e-6, precision=gb.Precision.Mixed)
        ds = gb.DiffSolver(lps, opt, tail_iters=40, ckpt_every=10)
        res, x, y = ds.forward(opt)
        rng = np.random.default_rng(0)
        g = ds.backward(rng.standard_normal(int(ds.n_off[-1])), rng.standard_normal(int(ds.m_off[-1])))
        parts = [np.array([[r.status, r.iterations] for r in res]), x, y] + [g[k] for k in sorted(g)]
        ds.close()
    print(digest(parts))


if __name__ == "__main__":
    main(sys.argv[1], float(sys.argv[2]) if len(sys.argv) > 2 else 1e-6)
