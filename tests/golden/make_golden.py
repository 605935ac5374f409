"""Generate the golden fixtures of the parity tests from the REFERENCE itself.

Runs the unmodified reference CPU PDHG (ganit::solve_pdhg_cpu, built from the
reference sources by oracle/Makefile into oracle/_ref/libganit_ref.so) on
OMP_NUM_THREADS=1 and records its results:

* synthetic instances (seeded generators of ganit_v2_b200.workloads): the
  problem arrays go to ``<name>.npz`` together with the reference's x and y,
  the scalar results to ``golden.json``;
* the reference's own Netlib / QP instances: read with the reference's MPS
  reader (src/mps.cpp) from its instances/ directory; the parsed arrays go to
  ``instances/<name>.npz`` (so GPU tests run where no reference checkout
  exists) and the scalar results to ``golden.json["reference_instances"]``.

Usage (in a container that has the reference checked out; GANIT_REF_ROOT or
--ref-root names the checkout):
    python tests/golden/make_golden.py            # everything
    python tests/golden/make_golden.py --instances-only [--recompute]
        # instance arrays; results only for instances golden.json lacks
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from ganit_v2_b200 import workloads as W  # noqa: E402
from ganit_v2_b200.lp import LP, Csr  # noqa: E402
from oracle import oracle as O  # noqa: E402

PRECISIONS = ("double", "mixed", "dynamic")

SYNTHETIC = {
    # name: (factory, solve options)
    "rand_small": (lambda: W.random_feasible_lp(200, 500, 6, seed=11), {}),
    "rand_free": (lambda: W.random_feasible_lp(150, 400, 5, seed=12, free_frac=0.2), {}),
    "rand_tight": (lambda: W.random_feasible_lp(300, 700, 7, seed=13), {"tol": 1e-6}),
    "rand_cfg0": (lambda: W.random_feasible_lp(2000, 5000, 8, seed=0), {}),
    "infeasible": (lambda: W.infeasible_lp(200, 500, seed=3), {}),
    "blend_small": (lambda: W.blending_lp(6, 3, 2, 10, seed=5), {}),
    "port_lifted_small": (lambda: W.portfolio_qp(300, 5, seed=21, lifted=True), {}),
    "rand_max": (None, {}),  # maximisation variant of rand_small, built below
}

REFERENCE_INSTANCES = ["afiro", "adlittle", "bgetam", "etamacro", "shell", "25fv47", "stair", "greenbea",
                       "qp/port_tiny", "qp/port_small", "qp/qblend_small"]
INSTANCE_DIR = os.path.join(HERE, "instances")


def instance_path(inst: str) -> str:
    """Fixture of a reference instance (qp/port_tiny -> instances/qp_port_tiny.npz)."""
    return os.path.join(INSTANCE_DIR, inst.replace("/", "_") + ".npz")


def lp_digest(lp: LP) -> str:
    h = hashlib.sha256()
    for a in (lp.A.ptr, lp.A.idx, lp.A.val, lp.c, lp.l, lp.u, lp.lo, lp.hi):
        h.update(np.ascontiguousarray(a).tobytes())
    if lp.Q is not None:
        for a in (lp.Q.ptr, lp.Q.idx, lp.Q.val):
            h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def save_lp(path: str, lp: LP, extra: dict):
    arrs = dict(a_ptr=lp.A.ptr, a_idx=lp.A.idx, a_val=lp.A.val, c=lp.c, l=lp.l, u=lp.u, lo=lp.lo, hi=lp.hi,
                meta=np.array([lp.obj_const, float(lp.maximize), lp.m, lp.n]))
    if lp.Q is not None:
        arrs.update(q_ptr=lp.Q.ptr, q_idx=lp.Q.idx, q_val=lp.Q.val)
    arrs.update(extra)
    np.savez_compressed(path, **arrs)


def load_lp(path: str) -> tuple[LP, dict]:
    z = np.load(path)
    oc, mx, m, n = z["meta"]
    m, n = int(m), int(n)
    Q = Csr(n, n, z["q_ptr"], z["q_idx"], z["q_val"]) if "q_ptr" in z else None
    lp = LP(Csr(m, n, z["a_ptr"], z["a_idx"], z["a_val"]), z["c"], z["l"], z["u"], z["lo"], z["hi"],
            obj_const=float(oc), maximize=bool(mx), Q=Q, name=os.path.basename(path)[:-4])
    return lp, {k: z[k] for k in z.files}


def result_dict(r) -> dict:
    return dict(status=r.status, pobj=r.pobj, dobj=r.dobj, rel_p=r.rel_p, rel_d=r.rel_d, rel_gap=r.rel_gap,
                iterations=int(r.iterations), fp32_iterations=int(r.fp32_iterations),
                l2_iterations=int(r.l2_iterations), restarts=int(r.restarts),
                x_sum=float(np.sum(r.x)), y_sum=float(np.sum(r.y)), x_norm=float(np.linalg.norm(r.x)),
                y_norm=float(np.linalg.norm(r.y)))


def reference_instances(ref_root: str, known: dict, recompute: bool) -> dict:
    """Parse every reference instance with the reference reader, write its
    arrays, and solve it with the reference (double and mixed) unless `known`
    already holds its results for the same data."""
    os.makedirs(INSTANCE_DIR, exist_ok=True)
    out = {}
    for inst in REFERENCE_INSTANCES:
        path = os.path.join(ref_root, "instances", inst + ".mps")
        lp = O.ref_read_mps(path)
        save_lp(instance_path(inst), lp, {})
        entry = {"m": lp.m, "n": lp.n, "nnz": lp.A.nnz, "digest": lp_digest(lp), "results": {}}
        old = known.get(inst)
        if old is not None and old["digest"] == entry["digest"] and not recompute:
            out[inst] = old
            continue
        for prec in ("double", "mixed"):
            r = O.ref_solve(lp, threads=1, precision=prec)
            entry["results"][prec] = result_dict(r)
            print(f"{inst:18s} {prec:8s} {r.status:18s} it={r.iterations:6d} pobj={r.pobj:.10g}", flush=True)
        out[inst] = entry
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=O.REF_ROOT)
    ap.add_argument("--instances-only", action="store_true")
    ap.add_argument("--recompute", action="store_true")
    a = ap.parse_args()
    O.build(ref=True)
    O._set_omp_threads(1)
    gpath = os.path.join(HERE, "golden.json")
    if a.instances_only:
        with open(gpath) as f:
            out = json.load(f)
        out["reference_instances"] = reference_instances(a.ref_root, out.get("reference_instances", {}),
                                                         a.recompute)
        with open(gpath, "w") as f:
            json.dump(out, f, indent=1, sort_keys=True)
        return
    out = {"generator": "tests/golden/make_golden.py", "reference": "ganit::solve_pdhg_cpu, OMP_NUM_THREADS=1",
           "synthetic": {}, "reference_instances": {}}
    lps = {}
    for name, (factory, opts) in SYNTHETIC.items():
        if factory is None:
            continue
        lps[name] = (factory(), opts)
    base = lps["rand_small"][0]
    lps["rand_max"] = (LP(base.A, -base.c, base.l, base.u, base.lo, base.hi, obj_const=1.5, maximize=True,
                          name="rand_max"), {})
    for name, (lp, opts) in lps.items():
        entry = {"m": lp.m, "n": lp.n, "nnz": lp.A.nnz, "digest": lp_digest(lp), "options": opts, "results": {}}
        extra = {}
        for prec in PRECISIONS:
            r = O.ref_solve(lp, threads=1, precision=prec, **opts)
            entry["results"][prec] = result_dict(r)
            extra[f"x_{prec}"] = r.x
            extra[f"y_{prec}"] = r.y
            print(f"{name:18s} {prec:8s} {r.status:18s} it={r.iterations:6d} pobj={r.pobj:.10g}")
        save_lp(os.path.join(HERE, f"{name}.npz"), lp, extra)
        out["synthetic"][name] = entry
    out["reference_instances"] = reference_instances(a.ref_root, {}, True)
    with open(gpath, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
