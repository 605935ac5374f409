#!/usr/bin/env python3
"""Benchmark of the B200 restarted-PDHG engine (one JSON line on rank 0).

Metric: PDHG solves/s at 1e-4 relative KKT (mixed precision L1 -> L3, every
result FP64-certified), with the FP64 single-instance path and the fused SpMV
kernels' HBM GB/s alongside.  Workload: the multi-period blending LP (60
crudes x 16 products x 5 specs x 365 periods: m = 57,305, n = 405,880,
nnz = 2,886,344), seeded synthetic data.

A step is one full solve.  ``value`` times the solve of the problem already
resident in HBM (upload + device scaling done once before timing) with CUDA
events on the problem's stream, L2 flushed (256 MiB write) before every step.
``e2e`` times the public one-shot call (gb_solve through ctypes) from pinned
host arrays: upload, device scaling, solve, FP64 certification and the
download of x and y all inside the timed region.

Multi-GPU (torchrun): a single LP does not shard, so every rank solves its
own replica (weak scaling); value = all ranks' solves / max-over-ranks time.

``--impl reference`` times the reference's own CPU implementation
(ganit::solve_pdhg_cpu, oracle/_ref/libganit_ref.so built from the reference
sources) with all host threads, on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "PDHG solves/s & SpMV HBM GB/s at 1e-4 rel KKT, mixed vs FP64, one B200"
UNIT = "solves/s"
PUBLISHED_GPU_S = 0.80  # blend_big (2.9M nnz) GPU PDHG at 1e-4, README.md:104-109 of the reference


def workload():
    from ganit_v2_b200 import workloads as W

    return W.blending_lp()


WORKLOAD_DESC = ("multi-period blending LP, 60 crudes x 16 products x 5 specs x 365 periods "
                 "(m=57305, n=405880, nnz=2886344), tol 1e-4, mixed L1->L3 with FP64 certification")


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        self.p.wait()
        self.f.seek(0)
        rows = [r.split(", ") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, name in enumerate(names):
                if len(r) >= 9 and r[5 + k].strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline_run(lp, sample_steps: int = 1):
    """Reference CPU PDHG (oracle/_ref) with all host threads on the same LP;
    falls back to the C oracle port (single thread) if the reference build is
    absent.  Returns (solves/s, kind, cores, seconds list, result)."""
    from oracle import oracle as O

    cores = os.cpu_count() or 1
    if O.ref_available():
        kind = "reference"
        run = lambda: O.ref_solve(lp, threads=cores, precision="mixed")  # noqa: E731
    else:
        if not os.path.exists(O.ORACLE_SO):
            O.build(ref=False)
        kind, cores = "port", 1
        run = lambda: O.solve(lp, precision="mixed")  # noqa: E731
    secs = []
    res = None
    for _ in range(sample_steps):
        t0 = time.perf_counter()
        res = run()
        secs.append(time.perf_counter() - t0)
    return sample_steps / sum(secs), kind, cores, secs, res


def dist_setup(n_gpus: int):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        import torch

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return rank, world, local, dist


def barrier(dist):
    if dist is not None:
        dist.barrier()


def reduce_max(dist, v: float) -> float:
    if dist is None:
        return v
    import torch

    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    lp = workload()
    from oracle import oracle as O

    for _ in range(args.warmup):
        cpu_baseline_run(lp, 1)
    vals, kind, cores, secs, res = None, None, None, [], None
    for _ in range(args.steps):
        v, kind, cores, s, res = cpu_baseline_run(lp, 1)
        secs += s
    value = len(secs) / sum(secs)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(secs) / len(secs),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": WORKLOAD_DESC, "parallelism": "cpu-openmp" if kind == "reference" else "cpu-1-thread"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"{args.steps} full mixed-precision solves of the blending LP "
                                   f"({res.iterations} iterations, status {res.status})"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "result": {"status": res.status, "pobj": res.pobj, "iterations": res.iterations},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_profile_case():
    """The workload of the bench, shortened for ncu: one problem, a warm-up
    solve and one measured solve (mixed), then 3 plain iterations per level."""
    import ganit_v2_b200 as gb

    gb.set_device(0)
    lp = workload()
    p = gb.Problem(lp)
    for _ in range(2):
        r = p.solve(gb.Options(precision=gb.Precision.Mixed), fetch=False)
    for lvl in (0, 2):
        p.time_kernels(lvl, 3)
    print(json.dumps({"profile_case": WORKLOAD_DESC, "status": r.status_name, "iterations": r.iterations,
                      "launches_per_solve": p.stats()[0]}))
    p.close()
    return 0


def batch_measure(steps: int = 3, seq_sample: int = 24) -> dict:
    """512 random feasible LPs of log-uniform size (m in [50, 4000],
    n = 2.5 m, 4-12 nonzeros per column, seeds 1000..1511): LPs/s of the
    batched mixed-precision solver (every result FP64-certified) against the
    plain FP64 single-instance path on the same GPU, looping over the first
    `seq_sample` instances one by one (each resident beforehand)."""
    import ganit_v2_b200 as gb
    from ganit_v2_b200 import workloads as W

    lps = W.lp_batch(512, seed=1000)
    mixed = gb.Options(precision=gb.Precision.Mixed)
    fp64 = gb.Options(precision=gb.Precision.Double)
    t0 = time.perf_counter()
    bs = gb.BatchSolver(lps, mixed)
    setup_s = time.perf_counter() - t0
    res = bs.solve(mixed, fetch=False)
    secs = []
    for _ in range(steps):
        t0 = time.perf_counter()
        res = bs.solve(mixed, fetch=False)
        secs.append(time.perf_counter() - t0)
    sched = bs.schedule()
    bs.close()
    n_opt = sum(r.status == gb.Status.Optimal for r in res)
    certified = sum(r.status == gb.Status.Optimal and max(r.rel_primal, r.rel_dual, r.rel_gap) <= 1e-4 * 1.0000001
                    for r in res)
    probs = [gb.Problem(lp, fp64) for lp in lps[:seq_sample]]
    for p in probs[:2]:
        p.solve(fp64, fetch=False)
    t0 = time.perf_counter()
    for p in probs:
        p.solve(fp64, fetch=False)
    seq_s = time.perf_counter() - t0
    for p in probs:
        p.close()
    batch_lps = len(lps) / min(secs)
    seq_lps = seq_sample / seq_s
    return {"workload": "512 random feasible LPs, m log-uniform [50,4000], n=2.5m, 4-12 nnz/col "
                        f"(sum nnz {sum(lp.A.nnz for lp in lps)})",
            "lps_per_s": batch_lps, "ms_per_batch": 1e3 * min(secs), "setup_s": setup_s,
            "optimal": n_opt, "certified_1e-4": certified, "iterations_max": max(r.iterations for r in res),
            "iterations_mean": float(np.mean([r.iterations for r in res])),
            "fp64_single_instance_loop_lps_per_s": seq_lps,
            "fp64_loop_sample": f"first {seq_sample} instances solved one by one (FP64, resident)",
            "speedup_vs_fp64_loop": batch_lps / seq_lps,
            "schedule": {"threads": sched["threads"], "blocks_per_sm": sched["blocks_per_sm"],
                         "group_A_hist": np.bincount(np.log2(sched["groups_A"]).astype(int), minlength=6).tolist(),
                         "group_AT_hist": np.bincount(np.log2(sched["groups_AT"]).astype(int), minlength=6).tolist()},
            "timing": "host wall clock around gb_batch_solve (synchronous), best of %d" % steps}


def pinned_copy(lp):
    """Copy the LP's host arrays into page-locked memory (torch pin_memory)."""
    import torch

    from ganit_v2_b200.lp import LP, Csr

    def pin(a):
        t = torch.empty(a.shape, dtype=getattr(torch, str(a.dtype)), pin_memory=True)
        t.numpy()[...] = a
        return t.numpy()

    A = Csr(lp.m, lp.n, pin(lp.A.ptr), pin(lp.A.idx), pin(lp.A.val))
    out = LP(A, pin(lp.c), pin(lp.l), pin(lp.u), pin(lp.lo), pin(lp.hi), lp.obj_const, lp.maximize, name=lp.name)
    nbytes = sum(a.nbytes for a in (A.ptr, A.idx, A.val, out.c, out.l, out.u, out.lo, out.hi))
    return out, nbytes


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--kernel-iters", type=int, default=200)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the 512-LP batch measurement")
    ap.add_argument("--profile", action="store_true",
                    help="short fixed sequence for ncu: upload + one warm-up solve + one solve + 3 timed iterations")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.profile:
        return run_profile_case()

    import torch

    import ganit_v2_b200 as gb

    rank, world, local, dist = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    gb.set_device(local)
    lp = workload()
    mixed = gb.Options(precision=gb.Precision.Mixed)
    fp64 = gb.Options(precision=gb.Precision.Double)
    prob = gb.Problem(lp, mixed)
    stream = torch.cuda.ExternalStream(prob.stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def timed(opt, k):
        """k solves, each bracketed by CUDA events on the problem's stream,
        L2 flushed before each; returns (total ms, last result, launches)."""
        total = 0.0
        res = None
        launches = 0
        for _ in range(k):
            with torch.cuda.stream(stream):
                flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            res = prob.solve(opt, fetch=False)
            e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
            launches += prob.stats()[0]
        return total, res, launches

    for _ in range(args.warmup):
        prob.solve(mixed, fetch=False)
        prob.solve(fp64, fetch=False)
    torch.cuda.synchronize()
    barrier(dist)
    torch.cuda.synchronize()
    clocks = Clocks(local)
    ms_mixed, r_mixed, launches = timed(mixed, args.steps)
    torch.cuda.synchronize()
    barrier(dist)
    ms_fp64, r_fp64, _ = timed(fp64, max(1, args.steps // 2))
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms_mixed_max = reduce_max(dist, ms_mixed)
    ms_fp64_max = reduce_max(dist, ms_fp64)
    value = world * args.steps / (ms_mixed_max / 1e3)
    fp64_value = world * max(1, args.steps // 2) / (ms_fp64_max / 1e3)

    # kernel roofline: fused SpMV + step kernels at the FP32 level that dominates the mixed solve
    ms_p, ms_d, _ = prob.time_kernels(0, args.kernel_iters)
    ms_p64, ms_d64, _ = prob.time_kernels(2, args.kernel_iters)
    nnz, m, n = lp.A.nnz, lp.m, lp.n
    bytes_dual32 = nnz * 8 + 4 * (m + 1) + 4 * n + 4 * 6 * m
    bytes_primal32 = nnz * 8 + 4 * (n + 1) + 4 * m + 4 * 8 * n
    bytes_dual64 = nnz * 12 + 4 * (m + 1) + 8 * n + 8 * 6 * m
    bytes_primal64 = nnz * 12 + 4 * (n + 1) + 8 * m + 8 * 8 * n
    peak, peak_kind = measured_peaks()
    dom = ("k_dual<float,float>", bytes_dual32, ms_d) if ms_d >= ms_p else ("k_primal<float,float>", bytes_primal32, ms_p)
    achieved = dom[1] / (dom[2] / 1e3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get(dom[0])

    # end to end through the public one-shot API from pinned host memory
    plp, h2d = pinned_copy(lp)
    d2h = 8 * (lp.m + lp.n)
    gb.solve_pdhg_gpu(plp, mixed)
    torch.cuda.synchronize()
    barrier(dist)
    e2e_steps = max(3, args.steps // 2)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        re2e = gb.solve_pdhg_gpu(plp, mixed)
    e2e_s = time.perf_counter() - t0
    e2e_s = reduce_max(dist, e2e_s)
    e2e_value = world * e2e_steps / e2e_s

    batch = None
    if not args.no_batch:
        batch = batch_measure()
    line = None
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            cv, kind, cores, secs, cres = cpu_baseline_run(lp, 1)
            cpu = {"value": cv, "unit": UNIT, "cores": cores, "kind": kind,
                   "sample": f"1 full mixed-precision solve of the same blending LP on the host "
                             f"({cres.iterations} iterations, {secs[0]:.2f} s, status {cres.status})"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_mixed_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": value / (1.0 / PUBLISHED_GPU_S),
            "vs_baseline_source": "reference README.md:104-109 blend_big GPU PDHG 0.80 s at 1e-4 (unspecified GPU)",
            "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": WORKLOAD_DESC, "precision": "mixed (FP32 matrix+iterates, FP64 finish/certify)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "flushed (256 MiB write) before every timed step"},
            "result": {"status": r_mixed.status_name, "iterations": r_mixed.iterations,
                       "fp32_iterations": r_mixed.fp32_iterations, "restarts": r_mixed.restarts,
                       "pobj": r_mixed.pobj, "rel_primal": r_mixed.rel_primal, "rel_dual": r_mixed.rel_dual,
                       "rel_gap": r_mixed.rel_gap},
            "fp64": {"value": fp64_value, "unit": UNIT, "ms_per_step": ms_fp64_max / max(1, args.steps // 2),
                     "status": r_fp64.status_name, "iterations": r_fp64.iterations, "pobj": r_fp64.pobj,
                     "mixed_speedup": value / fp64_value},
            "spmv_gbs": {"k_primal_f32": bytes_primal32 / (ms_p / 1e3) / 1e9,
                         "k_dual_f32": bytes_dual32 / (ms_d / 1e3) / 1e9,
                         "k_primal_f64": bytes_primal64 / (ms_p64 / 1e3) / 1e9,
                         "k_dual_f64": bytes_dual64 / (ms_d64 / 1e3) / 1e9,
                         "ms": {"primal_f32": ms_p, "dual_f32": ms_d, "primal_f64": ms_p64, "dual_f64": ms_d64}},
            "roofline": {"bound": "hbm", "kernel": dom[0], "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": f"{peak_kind} hbm_gbs",
                         "algorithmic_bytes_per_launch": dom[1]},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "status": re2e.status_name, "note": "gb_solve: upload + device scaling + solve + download"},
            "gpu_launches": launches,
            "clocks": clk,
            "cpu_baseline": cpu,
            "batch": batch,
        }
        print(json.dumps(line), flush=True)
    prob.close()
    if dist is not None:
        barrier(dist)
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
