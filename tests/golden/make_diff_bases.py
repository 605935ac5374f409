"""Optimal bases of the differentiable-layer workload from the REFERENCE dual
simplex (src/simplex.hpp:37-93, built into oracle/_ref/libganit_ref.so).

The workload is workloads.diff_batch(256): nondegenerate LPs m=500, n=1000,
10 nonzeros per column, seeds 2000..2255.  For the first COUNT instances this
writes ``diff_bases.npz``: the instance digests, the dual simplex's basis
heads (int32[m] each: basic columns j < n, slack of row j - n otherwise), its
vertex (x, y) and objective, so the GPU test can form the exact basis sensitivities
(dL/dc = B^-1 v_D, dL/db = B^-T w_F, dL/dA = -(dL/db) x^T - y (dL/dc)^T) with
dense solves of 500 x 500, without the reference build.

Usage (in a container with the reference checked out):
    python tests/golden/make_diff_bases.py
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from ganit_v2_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.golden.make_golden import lp_digest  # noqa: E402

COUNT = 16
OUT = os.path.join(HERE, "diff_bases.npz")


def main():
    O.build(ref=True)
    lps = W.diff_batch(256)[:COUNT]
    heads, objs, digests, xs, ys = [], [], [], [], []
    for i, lp in enumerate(lps):
        t = time.time()
        r = O.ref_dual_simplex(lp)
        assert r["status"] == 0, (i, r["status"])
        heads.append(r["head"].astype(np.int32))
        objs.append(r["objective"])
        xs.append(r["x"])
        ys.append(r["y"])
        digests.append(lp_digest(lp))
        print(i, r["objective"], r["iterations"], f"{time.time() - t:.1f}s", flush=True)
    np.savez_compressed(OUT, heads=np.stack(heads), objective=np.array(objs), digests=np.array(digests),
                        x=np.stack(xs), y=np.stack(ys))


if __name__ == "__main__":
    main()
