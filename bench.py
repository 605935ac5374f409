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
The batched workloads reported alongside (``batch``: 512 random LPs;
``diff``: the differentiable layer on 256 LPs) split their instances over the
ranks by the nnz-balanced partition of ganit_v2_b200.shard (no exchange;
time = max over ranks).

``--impl reference`` times the reference's own CPU implementation
(ganit::solve_pdhg_cpu, oracle/_ref/libganit_ref.so built from the reference
sources) with all host threads, on rank 0 only.  The default arm also times
the reference's own CUDA backend (ganit::solve_pdhg_gpu, built unmodified for
sm_100a into oracle/_ref/libganit_refcuda.so) on the same LP and GPU
(``reference_cuda``).
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
# The same config object on both arms (the reference arm solves the same LP with the same options).
CONFIG = {"workload": WORKLOAD_DESC, "precision": "mixed (FP32 matrix+iterates, FP64 finish/certify)"}


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
        "config": dict(CONFIG), "parallelism": "cpu-openmp" if kind == "reference" else "cpu-1-thread",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"{args.steps} full mixed-precision solves of the blending LP "
                                   f"({res.iterations} iterations, status {res.status})"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "result": {"status": res.status, "pobj": res.pobj, "iterations": res.iterations},
    }
    print(json.dumps(line), flush=True)
    return 0


def refcuda_measure(lp, steps: int = 2) -> dict:
    """The reference's own CUDA backend (ganit::solve_pdhg_gpu of
    src/backend_cuda.cu, unmodified, built for sm_100a into
    oracle/_ref/libganit_refcuda.so) on the same LP and options on this GPU:
    wall time of the whole call (host scaling, uploads, the solve with its
    blocking reductions, unscaling), best of `steps` after one warm-up."""
    from oracle import oracle as O

    if not O.refcuda_available():
        return {"unavailable": "oracle/_ref/libganit_refcuda.so not built (needs the reference sources)"}
    try:
        O.refcuda_solve(lp, precision="mixed")
        secs, res = [], None
        for _ in range(steps):
            t0 = time.perf_counter()
            res = O.refcuda_solve(lp, precision="mixed")
            secs.append(time.perf_counter() - t0)
    except Exception as e:  # a failing reference leg must not hide the rest of the line
        return {"unavailable": f"reference solve_pdhg_gpu failed: {e}"}
    return {"solves_per_s": 1.0 / min(secs), "seconds": min(secs), "solve_s": res.solve_s, "setup_s": res.setup_s,
            "status": res.status, "iterations": res.iterations, "fp32_iterations": res.fp32_iterations,
            "pobj": res.pobj, "rel_p": res.rel_p, "rel_d": res.rel_d, "rel_gap": res.rel_gap,
            "source": "src/backend_cuda.cu:382-393 (thread/warp-per-row SpMV, atomicAdd reductions read back "
                      "per call), built with nvcc -O3 -DNDEBUG for sm_100a"}


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


def reduce_sum(dist, v: float) -> float:
    if dist is None:
        return v
    import torch

    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def run_profile_batch():
    """The 512-LP batch shortened for ncu: one mixed solve (launch it with
    GANIT_B200_LAUNCH=stream so no conditional graph is involved), then 3
    plain FP32 iterations with every instance active."""
    import ganit_v2_b200 as gb
    from ganit_v2_b200 import workloads as W

    gb.set_device(0)
    lps = W.lp_batch(512, seed=1000)
    opt = gb.Options(precision=gb.Precision.Mixed)
    with gb.BatchSolver(lps, opt) as bs:
        res = bs.solve(opt, fetch=False)
        k = bs.time_kernels(0, 3)
    print(json.dumps({"profile_case": "512-LP batch", "optimal": sum(r.status_name == "OPTIMAL" for r in res),
                      "bytes_per_iter_f32": k["bytes_per_iter"]}))
    return 0


def run_profile_qp():
    """The portfolio QP for ncu: one one-shot mixed solve (launch it with
    GANIT_B200_LAUNCH=stream so every iteration kernel is a separate launch)."""
    import ganit_v2_b200 as gb
    from ganit_v2_b200 import workloads as W

    gb.set_device(0)
    lp = W.portfolio_qp(100_000, 50, seed=7)
    r = gb.solve_pdhg_gpu(lp, gb.Options(precision=gb.Precision.Mixed))
    print(json.dumps({"profile_case": "portfolio QP, 100000 assets x 50 factors (DPLR Hessian), mixed, tol 1e-4",
                      "status": r.status_name, "iterations": r.iterations}))
    return 0


def run_profile_diff():
    """The differentiable layer for ncu: 256 LPs (workloads.diff_batch), one
    forward and one backward.  The PDHG rounds of the forward and the MINRES
    loops of the polishing and the backward run as CUDA graphs (ncu sees
    their kernels only with GANIT_B200_LAUNCH=stream, which turns them into
    ~50,000 separate launches); the tail and the reverse pass are plain
    launches either way."""
    import numpy as np

    import ganit_v2_b200 as gb
    from ganit_v2_b200 import workloads as W

    gb.set_device(0)
    lps = W.diff_batch(256)
    opt = gb.Options(tol=1e-6, precision=gb.Precision.Mixed)
    ds = gb.DiffSolver(lps, opt, tail_iters=200, ckpt_every=20)
    rng = np.random.default_rng(3)
    res, x, y = ds.forward(opt)
    g = ds.backward(rng.standard_normal(int(ds.n_off[-1])), rng.standard_normal(int(ds.m_off[-1])))
    print(json.dumps({"profile_case": "differentiable layer, 256 LPs m=500 n=1000, forward + backward",
                      "optimal": int(sum(r.status == gb.Status.Optimal for r in res)),
                      "grad_finite": bool(all(np.all(np.isfinite(v)) for v in g.values()))}))
    return 0


def qp_measure(steps: int = 2) -> dict:
    """Convex portfolio QP: 100,000 assets, 50-factor risk model, Q = 2(FF^T + D)
    as the diagonal-plus-low-rank Hessian (workloads.portfolio_qp, seed 7),
    resident; mixed and FP64 solves to 1e-4, CUDA events on the problem's stream."""
    import torch

    import ganit_v2_b200 as gb
    from ganit_v2_b200 import workloads as W

    lp = W.portfolio_qp(100_000, 50, seed=7)
    out = {"workload": "portfolio QP, 100000 assets x 50 factors, budget row, 0 <= x <= 0.05 (DPLR Hessian)"}
    for name, prec in (("mixed", gb.Precision.Mixed), ("fp64", gb.Precision.Double)):
        opt = gb.Options(precision=prec)
        with gb.Problem(lp, opt) as p:
            stream = torch.cuda.ExternalStream(p.stream)
            r = p.solve(opt, fetch=False)
            ms = []
            for _ in range(steps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                r = p.solve(opt, fetch=False)
                e1.record(stream)
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
        out[name] = {"solves_per_s": 1e3 / min(ms), "ms": min(ms), "status": r.status_name,
                     "iterations": r.iterations, "pobj": r.pobj,
                     "rel_kkt": max(r.rel_primal, r.rel_dual, r.rel_gap)}
    return out


def branch_measure(cpu: bool, steps: int = 3, candidates: int = 32) -> dict:
    """Strong branching of a synthetic MILP node (workloads.milp_node: 20000
    integer columns, 500 knapsack rows at 1% density, seed 11): the node LP
    solved on the GPU (FP64, 1e-7), its `candidates` most fractional columns
    strong-branched -- 2 * candidates child LPs as one batch, mixed precision to
    1e-6 from the node's point, rigorous child bounds -- through
    gb_strong_branch (host arrays in and out, wall clock).  CPU leg: the
    reference's own loop (warm dual simplex per child, its default limit of 60
    iterations, src/mip.cpp:738-760) from the same node point and candidates,
    the node's simplex solve before it untimed."""
    import numpy as np

    import ganit_v2_b200 as gb
    from ganit_v2_b200 import workloads as W

    lp = W.milp_node(n=20000, knapsacks=500, density=0.01, up_blocked=0, down_blocked=0, seed=11)
    root = gb.solve_pdhg_gpu(lp, gb.Options(tol=1e-7, precision=gb.Precision.Double))
    x, y, z = root.x, root.y, root.pobj
    cands = gb.most_fractional(x, gb.fractional(x, lp.is_int), candidates)
    opt = gb.Options(tol=1e-6, precision=gb.Precision.Mixed)
    sb = gb.strong_branch(lp, x, cands, z, opt=opt, y=y)
    secs = []
    for _ in range(steps):
        t0 = time.perf_counter()
        sb = gb.strong_branch(lp, x, cands, z, opt=opt, y=y)
        secs.append(time.perf_counter() - t0)
    t = min(secs)
    out = {"workload": "MILP node: multi-dimensional knapsack, 20000 integer columns, 500 rows, 1% density "
                       f"(nnz {lp.A.nnz}); {len(cands)} most fractional candidates, {2 * len(cands)} child LPs",
           "children_per_s": 2 * len(cands) / t, "seconds": t, "seconds_all": secs,
           "children_solved": sb.children_solved, "action": sb.action, "var": sb.var,
           "iterations_mean": float(sb.iterations.mean()), "iterations_max": int(sb.iterations.max()),
           "settings": "children: mixed precision to 1e-6 relative KKT, started from the node point; every "
                       "child bound certified on the device (directed rounding)"}
    if cpu:
        from oracle import oracle as O

        if O.ref_available():
            ref = O.ref_strong_branch(lp, x, cands, 60)
            zc, zn = ref["z"], ref["z_node"]
            score = np.maximum(zc[:, 0] - zn, 1e-6) * np.maximum(zc[:, 1] - zn, 1e-6)
            fin = np.isfinite(zc)
            rel = np.abs(sb.z[fin] - zc[fin]) / (1.0 + np.abs(zc[fin]))
            out["cpu_reference"] = {
                "children_per_s": 2 * len(cands) / ref["seconds"], "seconds": ref["seconds"], "cores": 1,
                "kind": "reference", "sample": "warm dual simplex per child, 60-iteration limit (the reference's "
                "sb_iter_limit default), the whole candidate loop",
                "statuses": {str(k): int(v) for k, v in zip(*np.unique(ref["status"], return_counts=True))},
                "same_choice": bool(int(cands[int(np.argmax(score))]) == sb.var) if sb.action == 0 else None,
                "max_rel_z_diff": float(rel.max()) if rel.size else None}
            out["speedup_vs_cpu_reference"] = ref["seconds"] / t
    return out


def batch_measure(dist, rank: int, world: int, steps: int = 3) -> dict:
    """512 random feasible LPs of log-uniform size (m in [50, 4000],
    n = 2.5 m, 4-12 nonzeros per column, seeds 1000..1511): LPs/s of the
    batched mixed-precision solver (every result FP64-certified) against the
    plain FP64 single-instance path on the same GPU, looping over all 512
    instances one by one (each resident beforehand).  Row-split schedules come
    from the autotuner.  With N ranks the instances are split by the
    nnz-balanced partition (no exchange; time = max over ranks)."""
    import torch

    import ganit_v2_b200 as gb
    from ganit_v2_b200 import shard, workloads as W

    lps = W.lp_batch(512, seed=1000)
    part = shard.partition([shard.instance_weight(lp) for lp in lps], world)[rank]
    mine = [lps[i] for i in part]
    mixed = gb.Options(precision=gb.Precision.Mixed)
    fp64 = gb.Options(precision=gb.Precision.Double)
    t0 = time.perf_counter()
    bs = gb.BatchSolver(mine, mixed)
    setup_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    tune = bs.autotune(iters=30)
    tune_s = time.perf_counter() - t0
    res = bs.solve(mixed, fetch=False)
    secs = []
    for _ in range(steps):
        torch.cuda.synchronize()
        barrier(dist)
        t0 = time.perf_counter()
        res = bs.solve(mixed, fetch=False)
        secs.append(time.perf_counter() - t0)
    t_batch = reduce_max(dist, min(secs))
    bf16 = gb.Options(precision=gb.Precision.MixedBf16)
    res_bf = bs.solve(bf16, fetch=False)
    torch.cuda.synchronize()
    barrier(dist)
    t0 = time.perf_counter()
    res_bf = bs.solve(bf16, fetch=False)
    t_bf = reduce_max(dist, time.perf_counter() - t0)
    cert_bf = reduce_sum(dist, sum(r.status == gb.Status.Optimal and
                                   max(r.rel_primal, r.rel_dual, r.rel_gap) <= 1e-4 * 1.0000001 for r in res_bf))
    ktb = bs.time_kernels(3, 50)
    kt = bs.time_kernels(0, 50)
    kt64 = bs.time_kernels(2, 20)
    ktg = bs.time_kernels_graph(0, 50)
    sched = bs.schedule()
    bs.close()
    n_opt = reduce_sum(dist, sum(r.status == gb.Status.Optimal for r in res))
    certified = reduce_sum(dist, sum(r.status == gb.Status.Optimal and
                                     max(r.rel_primal, r.rel_dual, r.rel_gap) <= 1e-4 * 1.0000001 for r in res))
    it_max = reduce_max(dist, max(r.iterations for r in res))
    seq_lps = None
    if rank == 0:
        probs = [gb.Problem(lp, fp64) for lp in lps]
        for p in probs[:2]:
            p.solve(fp64, fetch=False)
        t0 = time.perf_counter()
        for p in probs:
            p.solve(fp64, fetch=False)
        seq_lps = len(probs) / (time.perf_counter() - t0)
        for p in probs:
            p.close()
    peak, peak_kind = measured_peaks()
    it_ms = kt["ms_primal"] + kt["ms_dual"]
    gbs = kt["bytes_per_iter"] / (it_ms / 1e3) / 1e9
    gbs64 = kt64["bytes_per_iter"] / ((kt64["ms_primal"] + kt64["ms_dual"]) / 1e3) / 1e9
    batch_lps = len(lps) / t_batch
    bn = tune["block_nnz"]
    mr = tune["max_rows"]
    return {"workload": "512 random feasible LPs, m log-uniform [50,4000], n=2.5m, 4-12 nnz/col "
                        f"(sum nnz {sum(lp.A.nnz for lp in lps)})",
            "lps_per_s": batch_lps, "ms_per_batch": 1e3 * t_batch, "setup_s": setup_s,
            "parallelism": f"instances split over {world} GPUs (nnz-balanced)" if world > 1 else "single GPU",
            "optimal": int(n_opt), "certified_1e-4": int(certified), "iterations_max": int(it_max),
            "iterations_mean_rank0": float(np.mean([r.iterations for r in res])),
            "fp64_single_instance_loop_lps_per_s": seq_lps,
            "fp64_loop_sample": "all 512 instances solved one by one (FP64, each resident beforehand)",
            "speedup_vs_fp64_loop": (batch_lps / seq_lps) if seq_lps else None,
            "iteration_kernels": {"bound": "hbm", "ms_primal_f32": kt["ms_primal"], "ms_dual_f32": kt["ms_dual"],
                                  "ms_per_iter_f32": it_ms, "bytes_per_iter_f32": kt["bytes_per_iter"],
                                  "gbs_f32": gbs, "frac_f32": gbs / peak,
                                  "ms_per_iter_f64": kt64["ms_primal"] + kt64["ms_dual"], "gbs_f64": gbs64,
                                  "frac_f64": gbs64 / peak, "peak": peak, "peak_source": f"{peak_kind} hbm_gbs",
                                  "graph_ms_per_iter_f32": ktg["ms_iteration"],
                                  "graph_gbs_f32": kt["bytes_per_iter"] / (ktg["ms_iteration"] / 1e3) / 1e9,
                                  "graph_frac_f32": kt["bytes_per_iter"] / (ktg["ms_iteration"] / 1e3) / 1e9 / peak,
                                  "note": "k_primal + k_dual over all instances (rank 0's shard), CUDA events, "
                                          "every instance active; bytes = 2 nnz (s_M+4) + 4 (m+n+2) + s_V (9n+7m)"},
            "bf16_trial": {"lps_per_s": len(lps) / t_bf, "certified_1e-4": int(cert_bf),
                           "ms_per_iter_bf16": ktb["ms_primal"] + ktb["ms_dual"],
                           "gbs_bf16": ktb["bytes_per_iter"] / ((ktb["ms_primal"] + ktb["ms_dual"]) / 1e3) / 1e9},
            "autotune": {"seconds": tune_s, "load_modes": tune["load_modes"],
                         "ms_per_iter_default": tune["ms_per_iter_default"],
                         "ms_per_iter_tuned": tune["ms_per_iter_tuned"],
                         "ms_per_iter_default_f64": tune["ms_per_iter_default_f64"],
                         "ms_per_iter_tuned_f64": tune["ms_per_iter_tuned_f64"],
                         "choices_f64": {f"{b}x{r}": int(np.sum((tune["block_nnz_f64"] == b) &
                                                                (tune["max_rows_f64"] == r)))
                                         for b, r in sorted(set(zip(tune["block_nnz_f64"].tolist(),
                                                                    tune["max_rows_f64"].tolist())))},
                         "choices": {f"{b}x{r}": int(np.sum((bn == b) & (mr == r)))
                                     for b, r in sorted(set(zip(bn.tolist(), mr.tolist())))}},
            "schedule": {"threads": sched["threads"], "blocks_per_sm": sched["blocks_per_sm"],
                         "group_A_hist": np.bincount(np.log2(sched["groups_A"]).astype(int), minlength=6).tolist(),
                         "group_AT_hist": np.bincount(np.log2(sched["groups_AT"]).astype(int), minlength=6).tolist()},
            "timing": "host wall clock around gb_batch_solve (synchronous), best of %d, max over ranks" % steps}


def diff_measure(dist, rank: int, world: int, count: int = 256, steps: int = 2, check: int = 16) -> dict:
    """Differentiable batched LP layer: `count` nondegenerate LPs of m=500,
    n=1000, 10 nnz/col (the random-LP family with a unique strictly
    complementary optimum; workloads.diff_batch), forward = mixed-precision
    restarted PDHG to 1e-6 + polishing + K=200 tail iterations checkpointed
    every R=20, backward = reverse pass + implicit completion for
    L = w.x* + v.y*.  Gradients of the first `check` instances are compared
    with the exact basis sensitivities of the reference dual simplex's optimal
    bases."""
    import torch

    import ganit_v2_b200 as gb
    from ganit_v2_b200 import shard, workloads as W

    lps = W.diff_batch(count)
    part = shard.partition([shard.instance_weight(lp) for lp in lps], world)[rank]
    mine = [lps[i] for i in part]
    opt = gb.Options(tol=1e-6, precision=gb.Precision.Mixed)
    t0 = time.perf_counter()
    ds = gb.DiffSolver(mine, opt, tail_iters=200, ckpt_every=20)
    setup_s = time.perf_counter() - t0
    rng = np.random.default_rng(3)
    w = rng.standard_normal(int(ds.n_off[-1]))
    v = rng.standard_normal(int(ds.m_off[-1]))
    res, x, y = ds.forward(opt)
    g = ds.backward(w, v)
    tf, tb = [], []
    launches_f = launches_b = 0
    for _ in range(steps):
        torch.cuda.synchronize()
        barrier(dist)
        t0 = time.perf_counter()
        res, x, y = ds.forward(opt)
        tf.append(time.perf_counter() - t0)
        launches_f = ds.info(0)["launches"]
        torch.cuda.synchronize()
        barrier(dist)
        t0 = time.perf_counter()
        g = ds.backward(w, v)
        tb.append(time.perf_counter() - t0)
        launches_b = ds.info(0)["launches"]
    t_f = reduce_max(dist, min(tf))
    t_b = reduce_max(dist, min(tb))
    infos = [ds.info(i) for i in range(len(mine))]
    opt_n = reduce_sum(dist, sum(r.status == gb.Status.Optimal for r in res))
    pol = reduce_sum(dist, sum(i["polished"] for i in infos))
    conv = reduce_sum(dist, sum(i["implicit_converged"] for i in infos))
    mr_max = reduce_max(dist, max(i["implicit_iterations"] for i in infos))
    its_max = reduce_max(dist, max(r.iterations for r in res))
    errs = []
    if rank == 0 and world == 1:
        # exact basis sensitivities of the reference dual simplex's optimal bases
        # (tests/golden/diff_bases.npz, make_diff_bases.py) for the first instances
        ref = np.load(os.path.join(ROOT, "tests", "golden", "diff_bases.npz"))
        n0, m0, z0 = ds.n_off, ds.m_off, ds.nnz_off
        for i in range(min(check, len(ref["heads"]), len(mine))):
            lp = mine[i]
            head = ref["heads"][i]
            basic = np.sort(head[head < lp.n])
            act = np.ones(lp.m, dtype=bool)
            act[head[head >= lp.n] - lp.n] = False
            X, Y = ref["x"][i], ref["y"][i]
            A = lp.A.to_scipy().tocsr()
            B = A[np.flatnonzero(act)][:, basic].toarray()
            wi, vi = w[n0[i]:n0[i + 1]], v[m0[i]:m0[i + 1]]
            p = np.zeros(lp.m)
            q = np.zeros(lp.n)
            p[act] = np.linalg.solve(B.T, wi[basic])
            q[basic] = np.linalg.solve(B, vi[act])
            rows = np.repeat(np.arange(lp.m), np.diff(lp.A.ptr))
            da = -(p[rows] * X[lp.A.idx] + Y[rows] * q[lp.A.idx])
            rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))  # noqa: E731
            errs.append([rel(g["c"][n0[i]:n0[i + 1]], q), rel(g["lo"][m0[i]:m0[i + 1]] + g["hi"][m0[i]:m0[i + 1]], p),
                         rel(g["a_val"][z0[i]:z0[i + 1]], da)])
    return {"workload": f"{count} nondegenerate LPs m=500 n=1000 10 nnz/col (sum nnz {sum(lp.A.nnz for lp in lps)})",
            "lps_per_s_forward_backward": count / (t_f + t_b), "forward_ms": 1e3 * t_f, "backward_ms": 1e3 * t_b,
            "setup_s": setup_s, "tail_iters": 200, "ckpt_every": 20,
            "optimal_1e-6": int(opt_n), "polished": int(pol), "implicit_converged": int(conv),
            "implicit_minres_iters_max": int(mr_max), "pdhg_iterations_max": int(its_max),
            "forward_launches": launches_f, "backward_launches": launches_b,
            "grad_rel_err_vs_basis_sensitivities": {"instances": len(errs),
                                                   "max_c": max((e[0] for e in errs), default=None),
                                                   "max_b": max((e[1] for e in errs), default=None),
                                                   "max_A": max((e[2] for e in errs), default=None)},
            "grad_checks": "vs the basis sensitivities of the reference dual simplex's optimal bases of the first "
                           "instances (tests/golden/diff_bases.npz); central differences in tests/test_gpu_diff.py",
            "parallelism": f"instances split over {world} GPUs (nnz-balanced)" if world > 1 else "single GPU",
            "timing": f"host wall clock around gb_diff_forward / gb_diff_backward (synchronous), best of {steps}, "
                      "max over ranks"}


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
    ap.add_argument("--no-diff", action="store_true", help="skip the differentiable-layer measurement")
    ap.add_argument("--no-qp", action="store_true", help="skip the portfolio-QP measurement")
    ap.add_argument("--no-branch", action="store_true", help="skip the strong-branching measurement")
    ap.add_argument("--no-reference-cuda", action="store_true",
                    help="skip timing the reference's own CUDA backend on the headline LP")
    ap.add_argument("--profile", nargs="?", const="single", choices=["single", "batch", "qp", "diff"],
                    help="short fixed sequence for ncu: 'single' = the blending LP (upload, two solves, 3 timed "
                         "iterations per level); 'batch' = the 512-LP batch (one solve, 3 timed FP32 iterations); "
                         "'qp' = the portfolio QP (one mixed solve); 'diff' = the differentiable layer "
                         "(one forward and one backward)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.profile == "qp":
        return run_profile_qp()
    if args.profile == "diff":
        return run_profile_diff()
    if args.profile == "batch":
        return run_profile_batch()
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

    prob.solve(mixed, fetch=False)
    t0 = time.perf_counter()
    tune = prob.autotune(30)  # row cuts and load variants of the iteration kernels (setup, untimed)
    tune_s = time.perf_counter() - t0
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
    barrier(dist)
    bf16 = gb.Options(precision=gb.Precision.MixedBf16)
    prob.solve(bf16, fetch=False)
    ms_bf16, r_bf16, _ = timed(bf16, max(1, args.steps // 2))
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms_mixed_max = reduce_max(dist, ms_mixed)
    ms_fp64_max = reduce_max(dist, ms_fp64)
    value = world * args.steps / (ms_mixed_max / 1e3)
    fp64_value = world * max(1, args.steps // 2) / (ms_fp64_max / 1e3)

    # kernel roofline: fused SpMV + step kernels at the FP32 level that dominates the mixed solve
    ms_p, ms_d, _ = prob.time_kernels(0, args.kernel_iters)
    ms_p64, ms_d64, _ = prob.time_kernels(2, args.kernel_iters)
    ms_pbf, ms_dbf, _ = prob.time_kernels(3, args.kernel_iters)
    kg = prob.time_kernels_graph(0, args.kernel_iters)
    kg64 = prob.time_kernels_graph(2, args.kernel_iters)
    nnz, m, n = lp.A.nnz, lp.m, lp.n
    bytes_dual32 = nnz * 8 + 4 * (m + 1) + 4 * n + 4 * 6 * m
    bytes_primal32 = nnz * 8 + 4 * (n + 1) + 4 * m + 4 * 8 * n
    bytes_dual64 = nnz * 12 + 4 * (m + 1) + 8 * n + 8 * 6 * m
    bytes_dualbf = nnz * 6 + 4 * (m + 1) + 4 * n + 4 * 6 * m
    bytes_primalbf = nnz * 6 + 4 * (n + 1) + 4 * m + 4 * 8 * n
    bytes_primal64 = nnz * 12 + 4 * (n + 1) + 8 * m + 8 * 8 * n
    peak, peak_kind = measured_peaks()
    dom = (("k_dual<float,float>", bytes_dual32, kg["ms_dual"]) if kg["ms_dual"] >= kg["ms_primal"]
           else ("k_primal<float,float>", bytes_primal32, kg["ms_primal"]))
    achieved = dom[1] / (dom[2] / 1e3) / 1e9
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    traffic_of = {}
    if os.path.exists(tp):
        with open(tp) as f:
            traffic_of = json.load(f)
    traffic = traffic_of.get(dom[0])
    # both iteration kernels (they split the iteration's time about evenly)
    pair = {name: {"achieved": b / (ms / 1e3) / 1e9, "frac": b / (ms / 1e3) / 1e9 / peak, "launch_ms": ms,
                   "algorithmic_bytes_per_launch": b, "traffic": traffic_of.get(name)}
            for name, b, ms in (("k_dual<float,float>", bytes_dual32, kg["ms_dual"]),
                                ("k_primal<float,float>", bytes_primal32, kg["ms_primal"]))}

    # end to end through the public one-shot API from pinned host memory
    plp, h2d = pinned_copy(lp)
    d2h = 8 * (lp.m + lp.n)
    pin = lambda k: torch.empty(k, dtype=torch.float64, pin_memory=True).numpy()  # noqa: E731
    xo, yo = pin(lp.n), pin(lp.m)
    gb.solve_pdhg_gpu(plp, mixed, out=(xo, yo))
    torch.cuda.synchronize()
    barrier(dist)
    e2e_steps = max(3, args.steps // 2)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        re2e = gb.solve_pdhg_gpu(plp, mixed, out=(xo, yo))
    e2e_s = time.perf_counter() - t0
    e2e_s = reduce_max(dist, e2e_s)
    e2e_value = world * e2e_steps / e2e_s

    # the reference's CUDA backend right after our own single-LP legs: its
    # per-call host work (scaling, launches, blocking read-backs) measured
    # 2-7x slower after the OpenMP-threaded CPU reference legs below had run
    refcuda = None
    if not args.no_reference_cuda and rank == 0:
        refcuda = refcuda_measure(lp)
        if "solves_per_s" in refcuda:
            refcuda["value_over_reference_cuda"] = value / refcuda["solves_per_s"]
            refcuda["e2e_over_reference_cuda"] = e2e_value / refcuda["solves_per_s"]
    batch = None
    if not args.no_batch:
        batch = batch_measure(dist, rank, world)
    diff = None
    if not args.no_diff:
        diff = diff_measure(dist, rank, world)
    qp = None
    if not args.no_qp and rank == 0:
        qp = qp_measure()
    branch = None
    if not args.no_branch and rank == 0:
        branch = branch_measure(cpu=not args.no_cpu_baseline and world == 1)
    line = None
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            cv, kind, cores, secs, cres = cpu_baseline_run(lp, 1)
            cpu = {"value": cv, "unit": UNIT, "cores": cores, "kind": kind,
                   "sample": f"1 full mixed-precision solve of the same blending LP on the host "
                             f"({cres.iterations} iterations, {secs[0]:.2f} s, status {cres.status})",
                   "solve_s": cres.solve_s, "setup_s": cres.setup_s}
            if kind == "reference":
                # the reference README's convention: OMP_NUM_THREADS=1
                from oracle import oracle as O

                t0 = time.perf_counter()
                r1 = O.ref_solve(lp, threads=1, precision="mixed")
                s1 = time.perf_counter() - t0
                cpu["single_thread"] = {"value": 1.0 / s1, "unit": UNIT, "cores": 1, "seconds": s1,
                                        "solve_s": r1.solve_s, "setup_s": r1.setup_s,
                                        "iterations": r1.iterations, "status": r1.status}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_mixed_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": value / (1.0 / PUBLISHED_GPU_S),
            "vs_baseline_source": "reference README.md:104-109 blend_big GPU PDHG 0.80 s at 1e-4 (unspecified GPU)",
            "dtype": "f32+f64", "data": "synthetic",
            "config": dict(CONFIG), "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "l2": "flushed (256 MiB write) before every timed step",
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
                         "k_primal_bf16": bytes_primalbf / (ms_pbf / 1e3) / 1e9,
                         "k_dual_bf16": bytes_dualbf / (ms_dbf / 1e3) / 1e9,
                         "ms": {"primal_f32": ms_p, "dual_f32": ms_d, "primal_f64": ms_p64, "dual_f64": ms_d64,
                                "primal_bf16": ms_pbf, "dual_bf16": ms_dbf},
                         "graph": {"k_primal_f32": bytes_primal32 / (kg["ms_primal"] / 1e3) / 1e9,
                                   "k_dual_f32": bytes_dual32 / (kg["ms_dual"] / 1e3) / 1e9,
                                   "k_primal_f64": bytes_primal64 / (kg64["ms_primal"] / 1e3) / 1e9,
                                   "k_dual_f64": bytes_dual64 / (kg64["ms_dual"] / 1e3) / 1e9,
                                   "ms": {"primal_f32": kg["ms_primal"], "dual_f32": kg["ms_dual"],
                                          "iteration_f32": kg["ms_iteration"], "primal_f64": kg64["ms_primal"],
                                          "dual_f64": kg64["ms_dual"], "iteration_f64": kg64["ms_iteration"]}},
                         "timing": "top level: CUDA events around every launch (serialising); 'graph': CUDA "
                                   "events around a CUDA graph of back-to-back launches with programmatic "
                                   "dependent launch, as the solve loop issues them; warm L2 (the FP32 "
                                   "iteration, 64 MB, is L2-resident in the solve too)"},
            "bf16_trial": {"value": max(1, args.steps // 2) / (ms_bf16 / 1e3), "unit": UNIT,
                           "ms_per_step": ms_bf16 / max(1, args.steps // 2), "status": r_bf16.status_name,
                           "iterations": r_bf16.iterations, "bf16_iterations": r_bf16.bf16_iterations,
                           "fp32_iterations": r_bf16.fp32_iterations, "pobj": r_bf16.pobj,
                           "note": "GB_PREC_MIXED_BF16: BF16 matrix values + FP32 iterates until the phase stalls, "
                                   "then FP32, then FP64; FP64-certified"},
            "roofline": {"bound": "hbm", "kernel": dom[0], "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": f"{peak_kind} hbm_gbs",
                         "algorithmic_bytes_per_launch": dom[1], "launch_ms": dom[2],
                         "timing": f"{args.kernel_iters} back-to-back launches in a CUDA graph, CUDA events",
                         "kernel_choice": "the longer of the two iteration kernels in this timing",
                         "working_set": "the FP32 iteration (64 MB) is L2-resident in the solve, so this fraction "
                                        "of the HBM copy peak is reached on L2-served data; the HBM-bound "
                                        "configuration is the 512-LP batch (batch.iteration_kernels)",
                         "kernels": pair},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "status": re2e.status_name, "setup_s_last": re2e.setup_seconds, "solve_s_last": re2e.solve_seconds,
                    "note": "gb_solve: pinned host arrays in, upload + validation + device scaling + solve + "
                            "FP64 certification + download into pinned arrays"},
            "autotune": {"seconds": tune_s, **tune,
                         "note": "the resident problem's iteration kernels after gb_problem_autotune (row-block cuts, "
                                 "load variant per matrix); `value` and the kernel timings use them, the one-shot "
                                 "`e2e` call does not tune"},
            "gpu_launches": launches,
            "clocks": clk,
            "cpu_baseline": cpu,
            "batch": batch,
            "diff": diff,
            "qp": qp,
            "strong_branching": branch,
            "reference_cuda": refcuda,
        }
        print(json.dumps(line), flush=True)
    prob.close()
    if dist is not None:
        barrier(dist)
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
