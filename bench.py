#!/usr/bin/env python
"""Benchmark of the B200 SQP inner loop (iiwa14 end-effector tracking).

Metric: SQP solves/s at N = 128 knots, PCG exit at relative residual 1e-5,
batched (512 instances per GPU in one call) -- the reference's headline
"SQP solves/s @N=128 batched vs plain @rel-res 1e-5".  One step = one
batched sqpSolve (toplevel.cuh:24-503 semantics: up to 40 SQP iterations,
line-search / rho exit, wall-clock cap removed) over seeded synthetic
problems (spline through 5 random joint configurations, dt = 0.01,
semi-implicit Euler, QD = 0.01, R = 1e-4).  `value` times the solve with the
inputs resident in HBM; `e2e` times the same call through the public API
with pinned-host inputs copied in and the result copied out every step.
The plain single-instance path (gpt_sqp_solve) is timed beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank solves its own batch (weak scaling, no collective on
the data path); the reported time is the max over ranks.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SQP solves/s @N=128 batched vs plain @rel-res 1e-5"
SPEC = dict(timestep=0.01, integrator=1, qd_cost=1e-2, r_cost=1e-4)
# Algorithmic bytes of one PCG launch per knot with the exact preconditioner: the FP64 Schur row read
# once (302 doubles: left block 196, diagonal lower triangle 105, pad), gamma (14 doubles), lambda in
# and out (FP32) and the FP64 lambda written for dz
PCG_BYTES_PER_KNOT = 8 * 302 + 8 * 14 + 2 * 4 * 14 + 8 * 14
PCG_BJ_BYTES_PER_KNOT = 4 * 784  # block-Jacobi kernel: FP32 S (588) + Pinv (196) read once
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch, per knot, from ncu captures of
# the bench's batch, 512 instances x 128 knots (the working set of a launch, ~0.26 GB, exceeds the L2, so
# the traffic per knot depends on the batch and is not scaled to other batches)
PCG_DRAM_BYTES_PER_KNOT = {"pcg_pair_kernel": (779.677440e6 + 92.534528e6) / (512 * 128),
                           "pcg_quad_kernel": (536.024320e6 + 146.112256e6) / (512 * 128)}
PCG_DRAM_SOURCE = "ncu capture of the 512 x 128 bench batch, one launch"
ALG_FLOATS_PER_KNOT_SQP = 4058   # every materialised SQP-iteration tensor written once, read once


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--knots", type=int, default=128)
    ap.add_argument("--tol", type=float, default=1e-5)
    ap.add_argument("--pcg-max-iter", type=int, default=10000)
    ap.add_argument("--sqp-max-iter", type=int, default=40)
    ap.add_argument("--plain-solves", type=int, default=20)
    ap.add_argument("--accuracy-instances", type=int, default=8,
                    help="instances of the batch whose every SQP iterate is re-solved in FP64 on the host")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the mixed-horizon batch, the K_sqp = 4 line and the FP64 accuracy block")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="bound of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--pcg-cluster", type=int, default=0, help="CTAs per instance in the PCG (0 = library choice)")
    ap.add_argument("--pcg-precond", type=int, default=1, choices=[0, 1],
                    help="0 block-Jacobi (the reference's), 1 block-tridiagonal LDL^T per CTA chunk")
    ap.add_argument("--batched-only", action="store_true", help="skip the e2e and plain legs (profiling runs)")
    ap.add_argument("--no-track", action="store_true", help="skip the MPC tracking leg")
    ap.add_argument("--sqp-graph", type=int, default=4, choices=range(0, 9),
                    help="0 host loop, 1 one graph per solve, K = 2..8 graph with K concurrent part-batch branches")
    ap.add_argument("--track-sqp-iters", type=int, default=4,
                    help="SQP iterations per solve in the tracking leg (stands in for the wall-clock cap)")
    ap.add_argument("--track-period-us", type=float, default=2000.0, help="plant time per control update")
    ap.add_argument("--sweep-plain", action="store_true",
                    help="only the plain single-instance sweep over N in {64,128,256,512} x tol in {1e-4,1e-5,1e-6}")
    ap.add_argument("--mixed-track", action="store_true",
                    help="only the mixed-horizon tracking workload (2048 instances, N from {64,128,256,512})")
    ap.add_argument("--mixed-batch", type=int, default=2048)
    ap.add_argument("--mixed-rows", type=int, default=512, help="trajectory rows per instance")
    ap.add_argument("--mixed-period-us", type=float, default=10000.0)
    return ap.parse_args()


# --------------------------------------------------------------------------- CPU (oracle) legs
def _cpu_worker(task):
    """Solve seeded instances with the oracle's restatement of the reference's qdldl path (FP32,
    KKT + Schur + LDL^T + dz + merit on one host core) until the time budget is used.  Only the
    solves are timed (the problems are generated before each solve's clock starts); returns
    (completed solves, seconds spent in them)."""
    N, seeds, budget, sqp_max_iter = task
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as O
    P = importlib.import_module("gpu-pcg-tracking_b200.problem")
    par = O.make_params(dt=SPEC["timestep"], integrator=SPEC["integrator"], qd_cost=SPEC["qd_cost"],
                        r_cost=SPEC["r_cost"])
    sv = O.make_solver(linsys=1, sqp_max_iter=sqp_max_iter)
    busy = 0.0
    done = 0
    for s in seeds:
        p = P.make_problem(N, s, dt=SPEC["timestep"])
        t0 = time.perf_counter()
        O.sqp_solve(par, sv, N, p["goal"], p["lam"], p["xu"], 1e-3, precision="f32")
        busy += time.perf_counter() - t0
        done += 1
        if busy > budget:
            break
    return done, busy


class CpuPool:
    """Host processes (spawn, started before the first GPU call) that time the oracle's qdldl path.
    A sample's rate is the sum over processes of completed solves / the time those solves took, so
    no process is charged for another's unfinished solve and no start-up is timed."""

    def __init__(self, cores=None):
        import multiprocessing as mp
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle_py
        oracle_py.build()
        self.cores = cores or (os.cpu_count() or 1)
        self.pool = mp.get_context("spawn").Pool(self.cores)
        self.calls = 0

    def sample(self, N, budget, sqp_max_iter):
        base = 100000 * self.calls
        self.calls += 1
        tasks = [(N, list(range(base + 1000 * i, base + 1000 * i + 1000)), budget, sqp_max_iter)
                 for i in range(self.cores)]
        t0 = time.perf_counter()
        res = self.pool.map(_cpu_worker, tasks)
        wall = time.perf_counter() - t0
        solves = sum(r[0] for r in res)
        rate = sum(r[0] / r[1] for r in res if r[1] > 0)
        return {"value": rate, "unit": "solves/s", "cores": self.cores, "kind": "port",
                "sample": f"{solves} seeded N={N} instances, sqpSolve qdldl path (FP32 KKT/Schur/LDL^T/dz/merit "
                          f"restated in C), {self.cores} processes x ~{budget:.0f}s of solves (sum of per-process "
                          f"solves per busy second), wall {wall:.1f}s"}

    def close(self):
        self.pool.close()
        self.pool.join()


def cpu_baseline(N, budget, sqp_max_iter, cores=None):
    pool = CpuPool(cores)
    try:
        pool.sample(N, min(budget, 3.0), sqp_max_iter)  # warm-up: first solves of fresh processes
        return pool.sample(N, budget, sqp_max_iter)
    finally:
        pool.close()


# --------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
            return
        # nvidia-smi's start-up (NVML initialisation) stays out of the timed region: wait for its
        # first sample, and count only the samples taken after mark()
        t0 = time.time()
        while not self.lines and time.time() - t0 < 10.0 and self.proc.poll() is None:
            time.sleep(0.02)
        self.first = 0

    def mark(self):
        self.first = len(self.lines)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        timed = self.lines[getattr(self, "first", 0):]
        for ln in (timed if timed else self.lines):
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------- reference arm
def run_reference(args, rank, world):
    if rank != 0:
        return
    # every step is a bounded sample of the same per-process rate as the cpu_baseline leg: about 60 s of
    # host work over the timed steps, at least 4 s of solves per process a step
    budget = max(4.0, min(args.cpu_seconds, 60.0 / max(args.steps, 1)))
    pool = CpuPool()
    rates = []
    cb = None
    try:
        for i in range(args.warmup + args.steps):
            r = pool.sample(args.knots, budget if i >= args.warmup else 2.0, args.sqp_max_iter)
            if i >= args.warmup:
                rates.append(r["value"])
                cb = r
    finally:
        pool.close()
    val = statistics.mean(rates)
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * budget,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"plain sqpSolve, qdldl path (the reference's oracle linear solve), N={args.knots}, "
                                   f"dt=0.01 semi-implicit, QD=0.01, R=1e-4, <= {args.sqp_max_iter} SQP iterations",
                       "knot_points": args.knots},
            "cpu_baseline": {"value": val, "unit": "solves/s", "cores": cb["cores"], "kind": cb["kind"],
                             "sample": cb["sample"]},
            "e2e": {"value": val, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- plain sweep
def sweep_diffs(gpt, sv, N, p, x0, g0, l0, iters):
    """Per-iterate linear-solve differences of one traced solve: at every SQP iterate the KKT blocks
    the CUDA kernel formed are solved (a) in FP64 on the host (fp64check: Schur complement, block
    Cholesky, dz) and (b) by the reference's qdldl path -- the CPU baseline's linear solve: FP32 Schur
    complement in CSC form, FP32 LDL^T, FP32 dz (qdldl_helper.cuh:62-180, restated in oracle/); the
    max over iterates of max |err| / max |FP64| for the B200 solve and for the qdldl path."""
    import numpy as np
    import torch
    F = importlib.import_module("gpu-pcg-tracking_b200.fp64check")
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as O
    _, st, tr = sv.sqp_solve_batched_trace([N], g0, l0.clone(), x0.clone(), [1e-3], iters)
    rec = gpt.trace_record_fields(tr["rec"])
    out = {"gpu_vs_fp64": {"lambda": 0.0, "dz": 0.0}, "qdldl_vs_fp64": {"lambda": 0.0, "dz": 0.0},
           "gpu_vs_qdldl": {"lambda": 0.0, "dz": 0.0}}
    xs = torch.as_tensor(p["xu"][:14], device="cuda")
    n_it = min(iters, int(st[0]["sqp_iters"]))
    for i in range(n_it):
        Gd, Cd, gd, cd = (torch.zeros(m, device="cuda") for m in (245 * N - 49, 294 * (N - 1), 21 * N - 7, 14 * N))
        sv.form_kkt(N, tr["xu"][i, :21 * N - 7].contiguous(), g0, xs, Gd, Cd, gd, cd)
        G, Cm, g, c = (t.cpu().numpy() for t in (Gd, Cd, gd, cd))
        rho = float(rec["rho"][i, 0])
        l64, d64 = F.solve_step(N, rho, G, Cm, g, c)
        S32, _, gam32, Gi32 = O.form_schur(N, rho, G, Cm, g, c, "f32")
        lq = O.ldl_solve(N, S32, gam32, "f32")
        dq = O.compute_dz(N, Gi32, Cm, g, lq, "f32")
        lg, dg = tr["lam"][i, :14 * N].cpu().numpy(), tr["dz"][i, :21 * N - 7].cpu().numpy()
        for key, (la, da, lb, db) in {"gpu_vs_fp64": (lg, dg, l64, d64), "qdldl_vs_fp64": (lq, dq, l64, d64),
                                      "gpu_vs_qdldl": (lg, dg, lq, dq)}.items():
            out[key]["lambda"] = max(out[key]["lambda"], F.rel_err(la, lb))
            out[key]["dz"] = max(out[key]["dz"], F.rel_err(da, db))
    out["iterates"] = n_it
    return out


def run_sweep_plain(args, rank, local_rank):
    """The plain method as the drop-in (gpt_sqp_solve, one instance) over N in {64, 128, 256, 512}
    and PCG exit tolerance in {1e-4, 1e-5, 1e-6}: solves/s (graph path, mean of 3 solves after one
    warm-up), device microseconds per linear solve (PCG phase of a profiled solve / its launches),
    PCG iterations per linear solve, and the PCG launch's algorithmic bytes / duration."""
    import torch
    if rank != 0:
        return
    torch.cuda.set_device(local_rank)
    gpt = importlib.import_module("gpu-pcg-tracking_b200")
    P = importlib.import_module("gpu-pcg-tracking_b200.problem")
    stream = torch.cuda.current_stream()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    rows = []
    for N in (64, 128, 256, 512):
        p = P.make_problem(N, 0, dt=SPEC["timestep"])
        x0, g0, l0 = (torch.as_tensor(p[k], device="cuda") for k in ("xu", "goal", "lam"))
        sv = gpt.Solver(max_knot_points=N, max_batch=1, **SPEC)
        sv.set_solver(sqp_max_iter=args.sqp_max_iter, pcg_max_iter=args.pcg_max_iter, pcg_exit_mode=0)
        cs = sv.autotune([N], g0, l0, x0, [1e-3])
        for tol in (1e-4, 1e-5, 1e-6):
            sv.set_solver(pcg_exit_tol=tol)
            ms, its = [], []
            for i in range(4):
                xu, lam = x0.clone(), l0.clone()
                flush.fill_(1.0)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                res = sv.sqp_solve(N, g0, lam, xu, 1e-3)
                e1.record(stream)
                e1.synchronize()
                if i > 0:
                    ms.append(e0.elapsed_time(e1))
                    its.append(res.stats["pcg_iters_total"] / max(res.sqp_iters, 1))
            sv.phase_stats(reset=True)
            sv.set_profiling(True)
            sv.sqp_solve(N, g0, l0.clone(), x0.clone(), 1e-3)
            sv.set_profiling(False)
            pcg_ms, pcg_n = sv.phase_stats(reset=True)["pcg"]
            us = 1000.0 * pcg_ms / max(pcg_n, 1)
            rows.append({"N": N, "tol": tol, "pcg_cluster_size": cs, "solves_per_s": 1000.0 / statistics.mean(ms),
                         "ms_per_solve": statistics.mean(ms), "linsys_us": us,
                         "pcg_iters_per_linsys": statistics.mean(its),
                         "pcg_gbs": PCG_BYTES_PER_KNOT * N / (us * 1e-6) / 1e9 if us > 0 else None,
                         "per_iterate_diffs": sweep_diffs(gpt, sv, N, p, x0, g0, l0, args.sqp_max_iter)})
        sv.close()
    print(json.dumps({"metric": "plain sqpSolve sweep", "unit": "solves/s", "dtype": "f32", "data": "synthetic",
                      "config": {"workload": f"gpt_sqp_solve, one instance, dt 0.01 semi-implicit Euler, QD 0.01, "
                                             f"R 1e-4, <= {args.sqp_max_iter} SQP iterations, exact preconditioner",
                                 "l2": "256 MB buffer written between timed solves"},
                      "rows": rows}), flush=True)


# --------------------------------------------------------------------------- mixed tracking workload
def run_mixed_track(args, rank, world, local_rank):
    """Receding-horizon tracking of B instances of seeded horizon N ~ U{64, 128, 256, 512}, each
    tracking its own seeded spline of `mixed_rows` rows (dt 0.01; the goal rows from the batched FK
    kernel), warm-started through the shift of xu and lambda, 4 SQP iterations per solve, 500 control
    updates, one batched solve (the replayed solve graph) and one simulate / shift launch per update.
    Times the rollout twice: forward only (gpt_track_batched), then with the adjoint of every update's
    solve and the weight gradients accumulated per instance (gpt_track_batched_adjoint); then, outside
    the timed regions, the tracking error of sampled instances against the plain single-instance
    loop (gpt_track) and the FP64 error of the solver's steps on a mixed-horizon batch."""
    import numpy as np
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local_rank)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    gpt = importlib.import_module("gpu-pcg-tracking_b200")
    P = importlib.import_module("gpu-pcg-tracking_b200.problem")
    shard = importlib.import_module("gpu-pcg-tracking_b200.shard")
    B, S = args.mixed_batch, args.mixed_rows
    ids = shard.weak_scaling_ids(rank, world, B)
    rng = np.random.default_rng(4321 + ids[0])
    Ns = [int(n) for n in rng.choice([64, 128, 256, 512], size=B)]
    rows, xs = zip(*(P.make_trajectory_rows(S, i, dt=SPEC["timestep"]) for i in ids))
    xu_traj = torch.as_tensor(np.concatenate(rows).reshape(-1), device="cuda")
    ee = gpt.end_effector_positions(xu_traj, 21).reshape(-1)
    xs0 = torch.as_tensor(np.concatenate(xs), device="cuda")
    solver_kw = dict(sqp_max_iter=args.track_sqp_iters, pcg_max_iter=args.pcg_max_iter, pcg_exit_tol=args.tol,
                     pcg_exit_mode=0, pcg_cluster_size=gpt.PCG_WARP_QUAD, sqp_graph=args.sqp_graph)
    sv = gpt.Solver(max_knot_points=max(Ns), max_batch=B, **SPEC)
    sv.set_solver(**solver_kw)
    n_updates = 500
    tcfg = gpt.default_track_config(sim_period_us=args.mixed_period_us, max_control_updates=n_updates)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    # warm-up: the first 3 control updates of the same rollout, both forms (builds the solve graph)
    warm = gpt.default_track_config(sim_period_us=args.mixed_period_us, max_control_updates=3)
    sv.track_batched(Ns, [S] * B, ee, xu_traj, xs0.clone(), warm, errors=torch.zeros(B * S, device="cuda"))
    sv.track_batched_adjoint(Ns, [S] * B, ee, xu_traj, xs0.clone(), warm, errors=torch.zeros(B * S, device="cuda"))

    def timed(adjoint):
        xs = xs0.clone()
        errs = torch.zeros(B * S, device="cuda")
        clocks = ClockSampler(torch.cuda.current_device())
        clocks.start()
        flush.fill_(1.0)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        clocks.mark()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        if adjoint:
            _, st, wgrad, loss, fails = sv.track_batched_adjoint(Ns, [S] * B, ee, xu_traj, xs, tcfg, errors=errs)
        else:
            _, st = sv.track_batched(Ns, [S] * B, ee, xu_traj, xs, tcfg, errors=errs)
            wgrad = loss = fails = None
        e1.record(stream)
        e1.synchronize()
        clk = clocks.stop()
        return shard.max_over_ranks(e0.elapsed_time(e1), device="cuda"), st, wgrad, loss, fails, clk

    t_ms, st, _, _, _, clk = timed(False)
    t_adj, st_a, wgrad, loss, fails, clk_a = timed(True)
    updates = sum(s["control_updates"] for s in st)
    # the weight gradient summed over the batch (the data-parallel reduction of shard.allreduce_weight_grads)
    wsum = wgrad.sum(0)
    if world > 1:
        dist.all_reduce(wsum)
    wsum = wsum.cpu().numpy()
    adjoint = {
        "ms": t_adj, "solves_per_s": world * updates / (t_adj / 1000.0),
        "overhead_ratio": (t_adj - t_ms) / t_ms,
        "us_per_solve": 1000.0 * (t_adj - t_ms) / max(updates / world, 1),
        "forward_equal": all(st[b] == st_a[b] for b in range(B)),
        "loss_total": float(loss.double().sum()), "adjoint_failures": int(sum(fails)),
        "weight_grad_batch_sum": {"qd": [float(v) for v in wsum[:7]], "r": [float(v) for v in wsum[7:14]],
                                  "q_ee": float(wsum[14])},
        "workload": "gpt_track_batched_adjoint: the same rollout with, after every update's solve, the one-step "
                    "adjoint of that update's horizon tracking loss (KKT, Schur, PCG and dz at the solution, the "
                    "loss gradient, the transposed solve, the weight gradients accumulated per instance)",
        "clocks": clk_a,
    }
    # the plain single-instance loop on sampled instances (one of each horizon), outside the timed region
    sample = [next(b for b in range(B) if Ns[b] == n) for n in (64, 128, 256, 512) if n in Ns]
    plain = []
    for b in sample:
        s1 = gpt.Solver(max_knot_points=Ns[b], **SPEC)
        s1.set_solver(**solver_kw)
        xs1 = xs0[14 * b:14 * b + 14].clone()
        tr_b = xu_traj[21 * S * b:21 * S * (b + 1)]
        ee_b = ee[6 * S * b:6 * S * (b + 1)]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, st1 = s1.track(Ns[b], ee_b, tr_b, xs1, tcfg)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        s1.close()
        plain.append({"instance": b, "N": Ns[b], "batched_tracking_error": st[b]["tracking_error_mean"],
                      "plain_tracking_error": st1["tracking_error_mean"],
                      "plain_solves_per_s": st1["control_updates"] / dt})
    # the FP64 error of the solver's steps on a mixed-horizon batch (one problem of each horizon)
    mb_Ns = [64, 128, 256, 512]
    mb = P.make_batch(mb_Ns, seed0=ids[0], dt=SPEC["timestep"])
    fp64 = fp64_accuracy(gpt, sv, mb_Ns, mb, len(mb_Ns), args.track_sqp_iters)
    line = {
        "metric": "mixed-horizon tracking solves/s", "value": world * updates / (t_ms / 1000.0), "unit": "solves/s",
        "n_gpus": world, "higher_is_better": True, "scaling": "weak", "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"gpt_track_batched: {B} instances/GPU, N ~ U{{64,128,256,512}} (seeded), {S} "
                               f"trajectory rows each, {n_updates} control updates, dt 0.01, plant period "
                               f"{args.mixed_period_us:g} us, {args.track_sqp_iters} SQP iterations per solve, "
                               f"partitioned PCG",
                   "instances_per_gpu": B, "knots_total": int(sum(Ns)), "rows": S},
        "ms": t_ms, "control_updates": st[0]["control_updates"], "ms_per_update": t_ms / max(st[0]["control_updates"], 1),
        "sqp_iters_per_solve": sum(s["sqp_iters_total"] for s in st) / max(updates, 1),
        "tracking_error_mean": statistics.mean(s["tracking_error_mean"] for s in st),
        "final_tracking_error_mean": statistics.mean(s["final_tracking_error"] for s in st),
        "rho_exits": sum(s["rho_exits"] for s in st), "nonfinite": sum(s["nonfinite"] for s in st),
        "clocks": clk, "adjoint": adjoint,
        "plain_vs_batched": {"instances": plain,
                             "max_abs_tracking_error_diff": max(abs(p["batched_tracking_error"] -
                                                                    p["plain_tracking_error"]) for p in plain)},
        "fp64_rel_err": fp64,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


# --------------------------------------------------------------------------- extras of the default line
def fp64_accuracy(gpt, sv, Ns, batch, n_inst, iters):
    """Relative error of the solve's lambda and dz against an FP64 host re-solve of the same KKT
    system, for every SQP iterate of n_inst sampled instances of the batch (a traced solve of the same
    batch, outside the timed region; the KKT blocks at each recorded iterate come from the CUDA KKT
    kernel, the FP64 Schur complement, block Cholesky and dz from fp64check)."""
    import numpy as np
    import torch
    F = importlib.import_module("gpu-pcg-tracking_b200.fp64check")
    B = len(Ns)
    offs = np.concatenate([[0], np.cumsum(Ns)])
    xu = torch.as_tensor(batch["xu"], device="cuda")
    goal = torch.as_tensor(batch["goal"], device="cuda")
    lam = torch.as_tensor(batch["lam"], device="cuda")
    _, stats, tr = sv.sqp_solve_batched_trace(Ns, goal, lam, xu, [1e-3] * B, iters)
    rec = gpt.trace_record_fields(tr["rec"])
    sample = [0] + sorted(np.random.default_rng(5).choice(np.arange(1, B), min(n_inst, B) - 1, replace=False).tolist())
    e_lam, e_dz, n = 0.0, 0.0, 0
    for b in sample:
        N, o = Ns[b], int(offs[b])
        g_b = goal[6 * o:6 * o + 6 * N]
        xs_b = xu.new_tensor(batch["xu"][21 * o:21 * o + 14])
        for i in range(min(iters, int(stats[b]["sqp_iters"]))):
            Gd, Cd, gd, cd = (torch.zeros(m, device="cuda") for m in (245 * N - 49, 294 * (N - 1), 21 * N - 7, 14 * N))
            sv.form_kkt(N, tr["xu"][i, 21 * o:21 * o + 21 * N - 7].contiguous(), g_b, xs_b, Gd, Cd, gd, cd)
            l64, d64 = F.solve_step(N, float(rec["rho"][i, b]), *(t.cpu().numpy() for t in (Gd, Cd, gd, cd)))
            e_lam = max(e_lam, F.rel_err(tr["lam"][i, 14 * o:14 * o + 14 * N].cpu().numpy(), l64))
            e_dz = max(e_dz, F.rel_err(tr["dz"][i, 21 * o:21 * o + 21 * N - 7].cpu().numpy(), d64))
            n += 1
    del tr
    return {"lambda_max_rel_err": e_lam, "dz_max_rel_err": e_dz, "iterates": n, "instances": sample,
            "reference": "FP64 host Schur complement + block Cholesky + dz of the GPU's own KKT blocks at each "
                         "recorded iterate (max |err| / max |FP64|)"}


def mixed_horizon_batch(gpt, P, args, seed0, flush, stream):
    """Batched form with uneven horizons: 512 seeded instances of N ~ U{32, 64, 128, 256}, one batched
    solve (graph, autotuned PCG) per step, against the same 512 instances solved one after another by
    the plain single-instance path (gpt_sqp_solve)."""
    import numpy as np
    import torch
    B = 512
    rng = np.random.default_rng(2024 + seed0)
    Ns = [int(n) for n in rng.choice([32, 64, 128, 256], size=B)]
    batch = P.make_batch(Ns, seed0=seed0, dt=SPEC["timestep"])
    sv = gpt.Solver(max_knot_points=max(Ns), max_batch=B, **SPEC)
    sv.set_solver(sqp_max_iter=args.sqp_max_iter, pcg_max_iter=args.pcg_max_iter, pcg_exit_tol=args.tol,
                  pcg_exit_mode=0, sqp_graph=args.sqp_graph)
    xu0, goal, lam0 = (torch.as_tensor(batch[k], device="cuda") for k in ("xu", "goal", "lam"))
    cs = sv.autotune(Ns, goal, lam0, xu0, [1e-3] * B)
    ms = []
    for i in range(3 + 5):
        xu, lam = xu0.clone(), lam0.clone()
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sv.sqp_solve_batched(Ns, goal, lam, xu, [1e-3] * B)
        e1.record(stream)
        e1.synchronize()
        if i >= 3:
            ms.append(e0.elapsed_time(e1))
    sv.close()
    batched_ms = statistics.mean(ms)
    # the same instances, one plain solve each, in sequence (one solver per horizon, autotuned)
    offs = np.concatenate([[0], np.cumsum(Ns)])
    plains = {}
    for n in sorted(set(Ns)):
        s1 = gpt.Solver(max_knot_points=n, max_batch=1, **SPEC)
        s1.set_solver(sqp_max_iter=args.sqp_max_iter, pcg_max_iter=args.pcg_max_iter, pcg_exit_tol=args.tol,
                      pcg_exit_mode=0)
        b0 = Ns.index(n)
        o = int(offs[b0])
        s1.autotune([n], goal[6 * o:6 * o + 6 * n], lam0[14 * o:14 * o + 14 * n],
                    xu0[21 * o:21 * o + 21 * n - 7].contiguous(), [1e-3])
        s1.sqp_solve(n, goal[6 * o:6 * o + 6 * n], lam0[14 * o:14 * o + 14 * n].clone(),
                     xu0[21 * o:21 * o + 21 * n - 7].clone(), 1e-3)  # builds the graph
        plains[n] = s1
    xs_all = [xu0[21 * int(offs[b]):21 * int(offs[b]) + 21 * Ns[b] - 7].clone() for b in range(B)]
    ls_all = [lam0[14 * int(offs[b]):14 * int(offs[b]) + 14 * Ns[b]].clone() for b in range(B)]
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for b in range(B):
        o = int(offs[b])
        plains[Ns[b]].sqp_solve(Ns[b], goal[6 * o:6 * o + 6 * Ns[b]], ls_all[b], xs_all[b], 1e-3)
    e1.record(stream)
    e1.synchronize()
    seq_ms = e0.elapsed_time(e1)
    for s1 in plains.values():
        s1.close()
    return {"workload": f"{B} instances, N ~ U{{32,64,128,256}} (seeded, {int(sum(Ns))} knots), one batched "
                        f"solve per step (graph, PCG cluster {cs}) vs the same {B} instances solved one after "
                        f"another by gpt_sqp_solve",
            "solves_per_s": B / (batched_ms / 1000.0), "ms_per_batch": batched_ms,
            "sequential_plain_solves_per_s": B / (seq_ms / 1000.0), "sequential_plain_ms": seq_ms,
            "batched_over_sequential_plain": seq_ms / batched_ms}


# --------------------------------------------------------------------------- our arm
def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    if args.mixed_track:
        run_mixed_track(args, rank, world, local_rank)
        return
    if args.sweep_plain:
        run_sweep_plain(args, rank, local_rank)
        return

    # the CPU baseline's process pool starts before the first GPU call
    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(args.knots, args.cpu_seconds, args.sqp_max_iter)

    import numpy as np
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local_rank)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    gpt = importlib.import_module("gpu-pcg-tracking_b200")
    P = importlib.import_module("gpu-pcg-tracking_b200.problem")
    shard = importlib.import_module("gpu-pcg-tracking_b200.shard")

    B, N = args.batch, args.knots
    Ns = [N] * B
    ids = shard.weak_scaling_ids(rank, world, B)  # this rank's instances (problem seeds)
    batch = P.make_batch(Ns, seed0=ids[0], dt=SPEC["timestep"])
    sv = gpt.Solver(max_knot_points=N, max_batch=B, **SPEC)
    sv.set_solver(sqp_max_iter=args.sqp_max_iter, pcg_max_iter=args.pcg_max_iter, pcg_exit_tol=args.tol,
                  pcg_exit_mode=0, pcg_cluster_size=args.pcg_cluster, pcg_precond=args.pcg_precond,
                  sqp_graph=args.sqp_graph)
    stream = torch.cuda.current_stream()
    xu0 = torch.as_tensor(batch["xu"], device="cuda")
    goal = torch.as_tensor(batch["goal"], device="cuda")
    lam0 = torch.as_tensor(batch["lam"], device="cuda")
    xu = torch.empty_like(xu0)
    lam = torch.empty_like(lam0)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def one_step(profile=False):
        xu.copy_(xu0)
        lam.copy_(lam0)
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rho, stats = sv.sqp_solve_batched(Ns, goal, lam, xu, [1e-3] * B)
        e1.record(stream)
        e1.synchronize()
        last_rho[:] = rho
        return e0.elapsed_time(e1), stats

    last_rho = [1e-3] * B
    # the PCG cluster size for this batch shape, chosen by timing (gpt_autotune) unless given
    schedule = {}
    tuned_cs = args.pcg_cluster if args.pcg_cluster else sv.autotune(Ns, goal, lam0, xu0, [1e-3] * B,
                                                                     schedule=schedule)

    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    for _ in range(args.warmup):
        one_step()
    barrier()
    clocks.mark()
    step_ms, all_stats = [], []
    for _ in range(args.steps):
        ms, stats = one_step()
        step_ms.append(ms)
        all_stats.extend(stats)
    barrier()
    clk = clocks.stop()
    # per-phase device time from one more step outside the timed region: profiling records
    # CUDA events between the launches, so that step runs the host-driven loop instead of the graph
    sv.phase_stats(reset=True)
    sv.set_profiling(True)
    one_step()
    sv.set_profiling(False)
    phases = sv.phase_stats(reset=True)
    # kernels per timed step of the graph: the prologue (init, G's weight-only entries, merit, accept),
    # then per SQP iteration (as many as the profiled step's KKT launches) the six phase kernels once
    # per part-batch branch and the while loop's control kernel
    branches = min(args.sqp_graph, B) if args.sqp_graph >= 2 else 1
    launches_per_step = 4 + phases["kkt"][1] * (6 * branches + 1)
    total_ms = sum(step_ms)
    total_ms = shard.max_over_ranks(total_ms, device="cuda")
    ms_per_step = total_ms / args.steps
    value = world * B / (ms_per_step / 1000.0)

    # adjoint of the SQP step at the solutions of the last timed step (gpt_sqp_adjoint): gradients of
    # w . xu+ w.r.t. the goal trajectory and the cost weights, timed like the forward solve
    offs = [sum(Ns[:b]) for b in range(B)]
    xs = torch.cat([xu0[21 * o:21 * o + 14] for o in offs])
    gw = torch.randn(xu.numel(), device="cuda", generator=torch.Generator(device="cuda").manual_seed(7))
    adj_ms, ar_ms = [], []
    for i in range(1 + args.steps):
        flush.fill_(1.0)
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        grads = sv.sqp_adjoint(Ns, goal, xs, xu, last_rho, gw)
        e1.record(stream)
        # the exchange step of data-parallel weight tuning: batch-summed weight gradients, all-reduced
        shard.allreduce_weight_grads(grads["qd"], grads["r"], grads["q_ee"])
        e2.record(stream)
        e2.synchronize()
        if i > 0:
            adj_ms.append(e0.elapsed_time(e1))
            ar_ms.append(e1.elapsed_time(e2))
    adj_step = statistics.mean(adj_ms)
    adj_step = shard.max_over_ranks(adj_step, device="cuda")
    adjoint = {"us_per_solve": 1000.0 * adj_step / B, "ms_per_batch": adj_step,
               "ratio_to_forward_solve": adj_step / ms_per_step,
               "weight_grad_allreduce_us": 1000.0 * shard.max_over_ranks(statistics.mean(ar_ms), device="cuda"),
               "workload": f"gpt_sqp_adjoint at the {B} solutions of the timed step (goal, QD, R, EE-weight "
                           f"gradients), then the 15 batch-summed weight gradients all-reduced over {world} rank(s)"}

    if args.batched_only:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": world * B / (ms_per_step / 1000.0), "unit": "solves/s",
                              "ms_per_step": ms_per_step, "phase_ms_per_step": {k: v[0] for k, v in phases.items()},
                              "pcg_iters_per_solve": sum(x["pcg_iters_total"] for x in all_stats) / len(all_stats),
                              "adjoint": adjoint}),
                  flush=True)
        if world > 1:
            dist.destroy_process_group()
        return

    # e2e through the public API: pinned host in, result out, every step
    h_xu = torch.as_tensor(batch["xu"]).pin_memory()
    h_goal = torch.as_tensor(batch["goal"]).pin_memory()
    h_lam = torch.as_tensor(batch["lam"]).pin_memory()
    o_xu = torch.empty_like(h_xu).pin_memory()
    o_lam = torch.empty_like(h_lam).pin_memory()
    d_xu, d_goal, d_lam = torch.empty_like(xu0), torch.empty_like(goal), torch.empty_like(lam0)
    e2e_ms = []
    for i in range(1 + args.steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        d_xu.copy_(h_xu, non_blocking=True)
        d_goal.copy_(h_goal, non_blocking=True)
        d_lam.copy_(h_lam, non_blocking=True)
        sv.sqp_solve_batched(Ns, d_goal, d_lam, d_xu, [1e-3] * B)
        o_xu.copy_(d_xu, non_blocking=True)
        o_lam.copy_(d_lam, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        if i > 0:
            e2e_ms.append(e0.elapsed_time(e1))
    e2e_step = statistics.mean(e2e_ms)
    e2e_step = shard.max_over_ranks(e2e_step, device="cuda")
    h2d = 4 * (h_xu.numel() + h_goal.numel() + h_lam.numel())
    d2h = 4 * (o_xu.numel() + o_lam.numel())

    # plain single-instance path (gpt_sqp_solve), same seeds
    plain_ms = []
    sv1 = gpt.Solver(max_knot_points=N, max_batch=1, **SPEC)
    sv1.set_solver(sqp_max_iter=args.sqp_max_iter, pcg_max_iter=args.pcg_max_iter, pcg_exit_tol=args.tol,
                   pcg_exit_mode=0, pcg_precond=args.pcg_precond)
    p = P.make_problem(N, ids[0], dt=SPEC["timestep"])
    plain_cs = args.pcg_cluster if args.pcg_cluster else sv1.autotune(
        [N], *(torch.as_tensor(p[k], device="cuda") for k in ("goal", "lam", "xu")), [1e-3])
    for i in range(args.plain_solves + 1):
        p = P.make_problem(N, ids[0] + i, dt=SPEC["timestep"])
        x1, g1, l1 = (torch.as_tensor(p[k], device="cuda") for k in ("xu", "goal", "lam"))
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sv1.sqp_solve(N, g1, l1, x1, 1e-3)
        e1.record(stream)
        e1.synchronize()
        if i > 0:
            plain_ms.append(e0.elapsed_time(e1))
    plain_rate = 1000.0 / statistics.mean(plain_ms) if plain_ms else None

    # extras of the default line (rank 0, outside the timed region, no collective): the headline batch at
    # a fixed K_sqp = 4 iterations per solve, the FP64 accuracy of every iterate of sampled instances, and
    # the batched form with uneven horizons against sequential plain solves
    extras = {}
    if rank == 0 and not args.no_extras:
        sv.set_solver(sqp_max_iter=4)
        k4 = []
        for i in range(args.warmup + args.steps):
            ms4, st4 = one_step()
            if i >= args.warmup:
                k4.append(ms4)
        sv.set_solver(sqp_max_iter=args.sqp_max_iter)
        extras["k_sqp4"] = {"solves_per_s": B / (statistics.mean(k4) / 1000.0), "ms_per_step": statistics.mean(k4),
                            "sqp_iters_mean": statistics.mean(x["sqp_iters"] for x in st4),
                            "workload": f"the headline batch with sqp_max_iter = 4 (the reference's logged mean of "
                                        f"3.96 SQP iterations per control step at N = 128)"}
        extras["fp64_rel_err"] = fp64_accuracy(gpt, sv, Ns, batch, args.accuracy_instances, args.sqp_max_iter)
        extras["mixed_horizon"] = mixed_horizon_batch(gpt, P, args, ids[0], flush, stream)

    # MPC tracking leg (gpt_track_batched): every instance tracks its own spline for as many rows as
    # its horizon (the shortest trajectory the loop accepts); one solve per control update
    track = None
    if not args.no_track:
        sv.set_solver(sqp_max_iter=args.track_sqp_iters, pcg_cluster_size=tuned_cs)
        tcfg = gpt.default_track_config(sim_period_us=args.track_period_us)
        xs_t = torch.cat([xu0[21 * o:21 * o + 14] for o in offs]).contiguous()
        errs = torch.zeros(B * N, device="cuda")
        sv.sqp_solve_batched(Ns, goal, lam, xu, [1e-3] * B)  # builds this shape's solve graph
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _, tstats = sv.track_batched(Ns, [N] * B, goal, xu0, xs_t, tcfg, errors=errs)
        e1.record(stream)
        e1.synchronize()
        t_ms = shard.max_over_ranks(e0.elapsed_time(e1), device="cuda")
        upd = tstats[0]["control_updates"]
        # the plain single-instance loop on instance 0's trajectory
        sv1.set_solver(sqp_max_iter=args.track_sqp_iters)
        xs1 = xs_t[:14].clone()
        e0.record(stream)
        _, pst = sv1.track(N, goal[:6 * N].contiguous(), xu0[:21 * N].contiguous(), xs1, tcfg)
        e1.record(stream)
        e1.synchronize()
        p_ms = e0.elapsed_time(e1)
        track = {
            "workload": f"gpt_track_batched: {B} instances x N={N}, trajectory of {N} rows each (the instance's "
                        f"spline), plant period {args.track_period_us:g} us, {args.track_sqp_iters} SQP iterations "
                        f"per solve, one solve per control update",
            "control_updates": upd, "ms": t_ms, "ms_per_update": t_ms / max(upd, 1),
            "solves_per_s": world * B * upd / (t_ms / 1000.0),
            "sqp_iters_per_solve": sum(t["sqp_iters_total"] for t in tstats) / max(B * upd, 1),
            "tracking_error_mean": statistics.mean(t["tracking_error_mean"] for t in tstats),
            "final_tracking_error_mean": statistics.mean(t["final_tracking_error"] for t in tstats),
            "rho_exits": sum(t["rho_exits"] for t in tstats),
            "plain_solves_per_s": pst["control_updates"] / (p_ms / 1000.0),
            "plain_tracking_error_mean": pst["tracking_error_mean"],
            "batched_over_plain": (B * upd / t_ms) / (pst["control_updates"] / p_ms),
        }

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return

    sqp_iters = [s["sqp_iters"] for s in all_stats]
    pcg_total = sum(s["pcg_iters_total"] for s in all_stats)
    pcg_maxit = sum(s["pcg_maxiter_count"] for s in all_stats)
    n_pcg_solves = sum(sqp_iters)
    # roofline: the PCG kernel dominates; its algorithmic bytes per launch = 784 floats x knots of the batch
    pcg_ms, pcg_launches = phases["pcg"]
    launches_total = launches_per_step * args.steps
    mp = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else None
    peak = mp["hbm_gbs"] if mp else 6650.0
    pcg_kernel = ("pcg_cluster_kernel" if args.pcg_precond == 0 else
                  "pcg_pair_kernel" if tuned_cs == gpt.PCG_WARP_PAIR else
                  "pcg_quad_kernel" if tuned_cs == gpt.PCG_WARP_QUAD else "pcg_chain_kernel")
    per_launch_bytes = (PCG_BJ_BYTES_PER_KNOT if args.pcg_precond == 0 else PCG_BYTES_PER_KNOT) * N * B
    per_launch_s = (pcg_ms / max(pcg_launches, 1)) / 1000.0
    achieved = per_launch_bytes / per_launch_s / 1e9 if per_launch_s > 0 else 0.0
    precond_name = "block-tridiagonal LDL^T" if args.pcg_precond == 1 else "block-Jacobi"
    dram_pk = PCG_DRAM_BYTES_PER_KNOT.get(pcg_kernel)
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"batched sqpSolve, {B} instances/GPU x N={N} knots, dt=0.01 semi-implicit Euler, "
                               f"QD=0.01, R=1e-4, PCG {precond_name} rel-res {args.tol:g} (max {args.pcg_max_iter} it), "
                               f"<= {args.sqp_max_iter} SQP iterations",
                   "instances_per_gpu": B, "knot_points": N, "pcg_exit_tol": args.tol, "parallelism": f"dp{world}",
                   "pcg_precond": precond_name, "pcg_cluster_size": tuned_cs,
                   "launch_schedule_ctas_per_sm": schedule or None,
                   "pcg_cluster_source": "given" if args.pcg_cluster else "gpt_autotune",
                   "l2": "256 MB buffer written between timed steps"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": dram_pk * N * B if (dram_pk and N * B == 512 * 128) else None,
                     "traffic_source": PCG_DRAM_SOURCE,
                     "kernel": pcg_kernel,
                     "bytes_model": ("2752 B per knot per launch: FP64 Schur row 302 doubles read once, gamma, "
                                     "lambda in/out FP32, lambda FP64 out" if args.pcg_precond == 1 else
                                     "784 floats per knot per launch (S 588 + Pinv 196 read once)"),
                     "peak_source": "measured" if mp else "fallback"},
        "cpu_baseline": cb,
        "e2e": {"value": world * B / (e2e_step / 1000.0), "unit": "solves/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches_total),
        "clocks": clk,
        "adjoint": adjoint,
        "plain_solves_per_s": plain_rate, "plain_pcg_cluster_size": plain_cs,
        "batched_over_plain": (value / world) / plain_rate if plain_rate else None,
        "phase_ms_per_step": {k: v[0] for k, v in phases.items()},
        "phase_launches_per_step": {k: v[1] for k, v in phases.items()},
        "sqp_loop": (f"one CUDA graph per solve (device-side while loop), {branches} part-batch branch(es) per "
                     f"iteration; phase times from a profiled host-loop step over the whole batch"),
        "sqp_iters_mean": statistics.mean(sqp_iters), "pcg_iters_per_solve": pcg_total / max(len(all_stats), 1),
        "pcg_iters_per_linsys": pcg_total / max(n_pcg_solves, 1), "pcg_maxiter_solves": pcg_maxit,
        "alg_bytes_per_sqp_iter_per_instance": 4 * N * ALG_FLOATS_PER_KNOT_SQP,
        "track": track,
    }
    line.update(extras)
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
