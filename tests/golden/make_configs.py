"""Reference results at the benchmark configurations' full sizes.

Runs the unmodified reference CPU PDHG (ganit::solve_pdhg_cpu, built from the
reference sources into oracle/_ref/libganit_ref.so) on the seeded synthetic
workloads of ganit_v2_b200.workloads at their full sizes and writes
``configs.json`` (scalars only; the tests regenerate the data from the same
seeds and check its digest first):

* ``blending``   multi-period blending LP, 60 crudes x 16 products x 5 specs x
                 365 periods (m 57,305, n 405,880, nnz 2,886,344), double and
                 mixed, tol 1e-4, one thread;
* ``batch512``   the 512 random feasible LPs of uneven size (m log-uniform in
                 [50, 4000], n = 2.5 m, 4-12 nonzeros per column, seeds
                 1000..1511), each solved alone at double, tol 1e-4, one thread;
* ``portfolio``  the 100,000-asset, 50-factor portfolio QP in the lifted form
                 the reference can hold (rows f - F^T x = 0, Hessian
                 diag(2D, 2I); the form of the reference's
                 bench/gen_portfolio.py), double, tol 1e-4, all host threads
                 (about two minutes on 8 cores).

Usage (in a container with the reference checked out):
    python tests/golden/make_configs.py [blending] [batch512] [portfolio]
"""
from __future__ import annotations

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from ganit_v2_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.golden.make_golden import lp_digest  # noqa: E402

OUT = os.path.join(HERE, "configs.json")


def scalars(r) -> dict:
    return dict(status=r.status, pobj=r.pobj, dobj=r.dobj, rel_p=r.rel_p, rel_d=r.rel_d, rel_gap=r.rel_gap,
                iterations=int(r.iterations), fp32_iterations=int(r.fp32_iterations), restarts=int(r.restarts),
                solve_s=r.solve_s)


def blending() -> dict:
    lp = W.blending_lp()
    out = {"workload": "workloads.blending_lp() (60/16/5/365, seed 1)", "m": lp.m, "n": lp.n, "nnz": lp.A.nnz,
           "digest": lp_digest(lp), "threads": 1, "results": {}}
    for prec in ("double", "mixed"):
        out["results"][prec] = scalars(O.ref_solve(lp, threads=1, precision=prec))
        print("blending", prec, out["results"][prec], flush=True)
    return out


def batch512() -> dict:
    lps = W.lp_batch(512, seed=1000)
    out = {"workload": "workloads.lp_batch(512, seed=1000)", "threads": 1, "instances": []}
    for lp in lps:
        r = O.ref_solve(lp, threads=1, precision="double")
        out["instances"].append(dict(m=lp.m, n=lp.n, nnz=lp.A.nnz, digest=lp_digest(lp), status=r.status,
                                     pobj=r.pobj, dobj=r.dobj, iterations=int(r.iterations)))
    print("batch512", len(out["instances"]), flush=True)
    return out


def portfolio() -> dict:
    lp = W.portfolio_qp(100_000, 50, seed=7, lifted=True)
    threads = os.cpu_count() or 1
    r = O.ref_solve(lp, threads=threads, precision="double")
    out = {"workload": "workloads.portfolio_qp(100000, 50, seed=7, lifted=True)", "m": lp.m, "n": lp.n,
           "nnz": lp.A.nnz, "digest": lp_digest(lp), "threads": threads, "results": {"double": scalars(r)}}
    print("portfolio", out["results"], flush=True)
    return out


def main():
    which = sys.argv[1:] or ["blending", "batch512", "portfolio"]
    O.build(ref=True)
    data = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    data["generator"] = "tests/golden/make_configs.py"
    data["reference"] = "ganit::solve_pdhg_cpu (oracle/_ref), tol 1e-4"
    for name in which:
        t = time.time()
        data[name] = {"blending": blending, "batch512": batch512, "portfolio": portfolio}[name]()
        data[name]["generated_s"] = round(time.time() - t, 1)
        with open(OUT, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
