#!/usr/bin/env python
"""Benchmark of the entropic semi-discrete dual evaluation (LSE dual-gradient pairs/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload trunc_3d|dense_2d|newton_3d] [--precision hybrid|fp64]

A step is one evaluation of the functional and its gradient (the reference's
SotSolver::evaluate_functional) over the whole synthetic workload at psi = 0,
the first evaluation of a solve.  Default workload: the 3D truncated
configuration (64^3 hex cells x 8 Gauss points = 2,097,152 quadrature points,
100,000 Gaussian-mixture targets, Dirichlet(1) weights, eps = 1e-3,
tau = 1e-12); synthetic seeded data (no dataset is published).

value : pairs / device time of one evaluation, inputs resident in HBM
        (sdot_evaluate_device), L2 flushed (256 MiB write) before every step.
e2e   : same metric through sdot_evaluate with pinned host psi in and host
        gradient out, the copies inside the timed region.
N > 1 : one process per GPU (torchrun); source cells sharded, one NCCL
        all-reduce of n_targets + 3 doubles per step; value = total pairs /
        max over ranks of the step time (strong scaling: fixed total work).
--impl reference: the FP64 CPU restatement of the reference's evaluation
        (oracle/, all host threads, WorkStream-like per-cell O(N) overheads)
        on a bounded sample of the same workload's cells, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Algorithmic FP64 flops per pair of the value sweep (FMA = 2): exponent
# A + B.x (d FMA), max and shift (2), exp2 by 16-entry table and degree-5
# polynomial (rint 3, polynomial 5 FMA, table product 1), accumulate (1 FMA).
VALUE_FLOPS_PER_PAIR = {2: 22, 3: 24}
# FP32 flops + one ex2 per pair of the FP32 gradient sweep: d differences,
# d-1 FMA + 1 mul for the square, 1 add + 1 FMA for the exponent, 1 FMA accumulate.
GRAD_FLOPS_PER_PAIR = {2: 10, 3: 13}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="trunc_3d",
                    choices=["trunc_3d", "dense_2d", "newton_3d", "hessian_3d", "batched_2d", "serve_3d"])
    ap.add_argument("--problems", type=int, default=None,
                    help="batched_2d: problems (default 256); serve_3d: requests (default 60)")
    ap.add_argument("--rate", type=float, default=4.0, help="serve_3d: Poisson arrival rate (requests/s)")
    ap.add_argument("--slots", type=int, default=4, help="batched_2d / serve_3d: concurrent solve slots")
    ap.add_argument("--baseline-seconds", type=float, default=60.0,
                    help="solve workloads: wall budget of the one-at-a-time FP64 L-BFGS baseline")
    ap.add_argument("--precision", default="hybrid", choices=["hybrid", "fp64", "mixed"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--scale", type=float, default=None,
                    help="shrink the workload (default 1; serve_3d: 0.5, the request sizes it is documented at)")
    args = ap.parse_args()
    if args.problems is None:
        args.problems = 60 if args.workload == "serve_3d" else 256
    if args.scale is None:
        args.scale = 0.5 if args.workload == "serve_3d" else 1.0
    return args


def make_workload(name: str, scale: float):
    from semidiscreteot_b200 import workloads as W
    if name == "trunc_3d":
        return W.trunc_3d(seed=0, n_cells=max(4, int(round(64 * scale))), n_targets=max(64, int(100_000 * scale ** 3)))
    if name == "dense_2d":
        return W.dense_2d(seed=0, n_cells=max(4, int(round(64 * scale))), n_targets=max(16, int(1000 * scale ** 2)))
    return W.newton_3d(seed=0, n_cells=max(4, int(round(32 * scale))), n_targets=max(64, int(20_000 * scale ** 3)))


def workload_config(wl, args, world):
    src = wl["source"]
    p = wl["params"]
    return {"workload": wl["name"], "dim": wl["dim"], "n_cells": int(src["cell_offsets"].size - 1),
            "n_quadrature": int(src["jxw"].size), "n_targets": int(wl["y"].shape[0]), "epsilon": p.epsilon,
            "tau": p.tau, "log_sum_exp": p.use_log_sum_exp_trick, "psi": "zeros", "precision": args.precision,
            "parallelism": f"source-sharded x{world}" if world > 1 else "single GPU",
            "l2": "flushed before every step (256 MiB write)"}


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (FP64 restatement of the reference) on a sample
# ---------------------------------------------------------------------------

def cpu_sample(wl, seconds: float, threads: int = 0):
    """Time the reference-faithful evaluation (per-cell O(N) CopyData zeroing,
    serialised in-order dense merge) on evenly spaced cells of the workload.
    Returns (pairs/s, cores, description)."""
    from oracle import oracle as orc
    src = wl["source"]
    off = src["cell_offsets"]
    ncell = off.size - 1
    dim = wl["dim"]
    prm = wl["params"]
    op = orc.Params(epsilon=prm.epsilon, tau=prm.tau, use_log_sum_exp=prm.use_log_sum_exp_trick)
    full = orc.Problem(src["x"], src["jxw"], src["density"], off, src["cell_centers"], wl["y"], wl["nu"])
    psi = np.zeros(wl["y"].shape[0])
    r = full.distance_threshold(psi, op)

    def subproblem(cells):
        qpc = int(off[1] - off[0])
        qidx = (cells[:, None] * qpc + np.arange(qpc)[None, :]).ravel()
        return orc.Problem(src["x"][qidx], src["jxw"][qidx], src["density"][qidx],
                           np.arange(cells.size + 1, dtype=np.int64) * qpc,
                           np.asarray(src["cell_centers"]).reshape(ncell, dim)[cells], wl["y"], wl["nu"])

    ncores = os.cpu_count() or 1
    nthr = threads if threads > 0 else ncores
    probe = np.linspace(0, ncell - 1, min(ncell, 4 * nthr)).astype(np.int64)
    P = subproblem(probe)
    t0 = time.perf_counter()
    P.evaluate_cells(psi, op, r, 0, probe.size, faithful=True, threads=nthr)
    dt = max(time.perf_counter() - t0, 1e-6)
    n = int(min(ncell, max(probe.size, probe.size * seconds / dt)))
    cells = np.linspace(0, ncell - 1, n).astype(np.int64)
    P = subproblem(cells)
    t0 = time.perf_counter()
    _, _, _, pairs = P.evaluate_cells(psi, op, r, 0, cells.size, faithful=True, threads=nthr)
    dt = time.perf_counter() - t0
    desc = (f"{cells.size} of {ncell} cells (evenly spaced), full target set, psi=0, threshold r={r:.6g}; "
            f"{pairs} pairs in {dt:.2f}s; reference-faithful FP64 (per-cell O(N) CopyData zeroing + "
            f"serialised in-order merge), OpenMP {nthr} threads")
    return pairs / dt, nthr, desc, dt


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    def __init__(self, index: int):
        self.index = index
        self.lines = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for k, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(k)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def read_traffic(kernel: str, workload: str):
    """DRAM bytes per launch of a kernel from the committed ncu summary
    profiles/<kernel>_<workload>.md (line 'traffic_bytes_per_launch: X')."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.md")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


# ---------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------

def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    wl = make_workload(args.workload, args.scale)
    per_step = max(1.0, args.cpu_seconds / 2)
    for _ in range(args.warmup):
        cpu_sample(wl, per_step / 4)
    vals, descs, cores = [], [], 0
    t_total = 0.0
    for _ in range(args.steps):
        v, cores, d, dt = cpu_sample(wl, per_step)
        vals.append(v)
        descs.append(d)
        t_total += dt
    value = float(np.mean(vals))
    line = {"impl": "reference", "metric": "LSE dual-gradient pairs/s", "value": value, "unit": "pairs/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * t_total / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded; no published dataset)",
            "config": workload_config(wl, args, 1),
            "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": cores, "kind": "port",
                             "sample": descs[-1]},
            "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_ours(args):
    import torch
    from semidiscreteot_b200 import SotSolver
    from semidiscreteot_b200.distributed import DistributedSotSolver

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.gpus > 1 and world == 1:
        print("bench.py: --gpus > 1 must be launched with torchrun (one process per GPU)", file=sys.stderr)
        return 2
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    wl = make_workload(args.workload, args.scale)
    src, y, nu, prm, dim = wl["source"], wl["y"], wl["nu"], wl["params"], wl["dim"]
    N = y.shape[0]
    if world > 1:
        solver = DistributedSotSolver(dim, rank, world, device=local, precision=args.precision)
        solver.setup_source(src)
        solver.setup_target(y, nu)
        solver.configure(prm)
        lib = solver.local
    else:
        solver = SotSolver(dim=dim, device=local, precision=args.precision)
        solver.setup_source_measure(src)
        solver.setup_target(y, nu)
        solver.configure(prm)
        lib = solver
    stream = torch.cuda.ExternalStream(lib.stream_handle, device=dev)
    psi = torch.zeros(N, dtype=torch.float64, device=dev)
    grad = torch.empty(N, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step():
        if world > 1:
            J, g, C, pairs = solver.evaluate(psi)
            return pairs
        solver.evaluate_functional_device(psi.data_ptr(), grad.data_ptr())
        return solver.last_eval_info["n_pairs"]

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    lib.set_profiling(True)
    lib.kernel_times(reset=True)
    times, pairs = [], 0.0
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            pairs = step()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        torch.cuda.synchronize()
    kt = lib.kernel_times(reset=True)
    lib.set_profiling(False)
    t_ms = float(np.mean(times))
    if world > 1:
        t = torch.tensor([t_ms], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        t_ms = float(t.item())
        torch.distributed.barrier()
    value = pairs / (t_ms * 1e-3)

    # e2e through the public host API (pinned host psi in, host gradient out)
    e2e = None
    if world == 1:
        hpsi = torch.zeros(N, dtype=torch.float64).pin_memory()
        hgrad = torch.empty(N, dtype=torch.float64).pin_memory()
        psi_np, grad_np = hpsi.numpy(), hgrad.numpy()
        for _ in range(2):
            solver.evaluate_functional(psi_np, grad_np)
        et = []
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            solver.evaluate_functional(psi_np, grad_np)
            e1.record(stream)
            e1.synchronize()
            et.append(e0.elapsed_time(e1))
        e2e = {"value": pairs / (float(np.mean(et)) * 1e-3), "unit": "pairs/s",
               "h2d_bytes_per_step": int(N * 8), "d2h_bytes_per_step": int(N * 8 + 8),
               "ms_per_step": float(np.mean(et))}

    if rank != 0:
        if world > 1:
            solver.close()
            torch.distributed.destroy_process_group()
        return 0

    # roofline of the dominant kernel (device time per launch from CUDA events)
    peaks = SotSolver.measure_peaks(local)
    nsteps = args.steps
    tv = kt["value_sweep"]["ms"] / max(1, kt["value_sweep"]["launches"])
    tg = kt["gradient_sweep"]["ms"] / max(1, kt["gradient_sweep"]["launches"])
    local_pairs = lib.last_eval_info["n_pairs"]
    if tv >= tg:
        ach = VALUE_FLOPS_PER_PAIR[dim] * local_pairs / (tv * 1e-3) / 1e12
        kname = ("k_value_dense (FP64 exp2 value sweep)" if prm.tau <= 0 else
                 "k_fused (FP64 exp2 value sweep + FP32 ex2 gradient sweep, one kernel)")
        roof = {"kernel": kname,
                "bound": "fp64", "achieved": ach, "peak": peaks["fp64_tflops"], "unit": "TFLOP/s",
                "frac": ach / peaks["fp64_tflops"],
                "traffic": read_traffic("value_sweep", wl["name"]),
                "flops_per_pair": VALUE_FLOPS_PER_PAIR[dim], "ms_per_launch": tv,
                "peak_source": "measured on this GPU by sdot_measure_peaks (FP64 FMA chains); "
                               "MEASURED_PEAKS.json has no FP64 figure"}
    else:
        ach = local_pairs / (tg * 1e-3) / 1e9
        roof = {"kernel": "gradient sweep (FP32 ex2)", "bound": "mufu", "achieved": ach,
                "peak": peaks["ex2_gops"], "unit": "Gex2/s", "frac": ach / peaks["ex2_gops"],
                "traffic": read_traffic("gradient_sweep", wl["name"]), "ms_per_launch": tg,
                "peak_source": "measured on this GPU by sdot_measure_peaks (ex2.approx chains)"}
    launches = sum(v["launches"] for v in kt.values())
    line = {"metric": "LSE dual-gradient pairs/s", "value": value, "unit": "pairs/s", "n_gpus": world,
            "steps": nsteps, "warmup": max(3, args.warmup), "ms_per_step": t_ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f64 value sweep + f32 exp gradient sweep",
            "data": "synthetic (seeded; no published dataset)", "config": workload_config(wl, args, world),
            "pairs_per_step": pairs, "roofline": roof,
            "kernel_ms_per_step": {k: v["ms"] / nsteps for k, v in kt.items()},
            "gpu_launches": int(launches), "clocks": clk.summary(), "peaks_measured": peaks}
    if e2e is not None:
        line["e2e"] = e2e
    if not args.no_cpu_baseline and world == 1:
        v, cores, desc, _ = cpu_sample(wl, args.cpu_seconds)
        line["cpu_baseline"] = {"value": v, "unit": "pairs/s", "cores": cores, "kind": "port", "sample": desc}
    print(json.dumps(line))
    if world > 1:
        solver.close()
        torch.distributed.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# solve-level workloads (the Newton / batched / served configurations)
# ---------------------------------------------------------------------------

def _fp64_lbfgs_baseline(problems, seconds):
    """One-at-a-time plain FP64 GPU solves (sdot_solve, L-BFGS, no epsilon
    scaling) on the problems in order until the wall budget is spent."""
    from semidiscreteot_b200 import SotSolver
    t_all, done, conv, iters = 0.0, 0, 0, []
    for p in problems:
        if t_all >= seconds:
            break
        src = p["source"]
        s = SotSolver(dim=p["y"].shape[1], device=0, precision="fp64")
        s.setup_source_measure(src)
        s.setup_target(p["y"], p["nu"])
        t0 = time.perf_counter()
        try:
            s.solve(np.zeros(len(p["nu"])), p["params"])
            ok = bool(s.get_convergence_status())
        except RuntimeError:
            ok = False
        t_all += time.perf_counter() - t0
        iters.append(int(s.get_last_iteration_count()))
        done += 1
        conv += ok
        s.close()
    return {"solves_per_s": conv / t_all if t_all > 0 else 0.0, "attempted": done, "converged": conv,
            "seconds": t_all, "iterations": iters,
            "method": "sdot_solve (L-BFGS, FP64 sweeps), one problem at a time, psi0 = 0, no epsilon scaling"}


def run_hessian_3d(args):
    """Config 3: tensor-core Hessian (roofline) and the Newton solve to gradient
    linf 1e-8, against the FP64 L-BFGS solve of the same problem."""
    import torch
    from semidiscreteot_b200 import SotSolver
    wl = make_workload("newton_3d", args.scale)
    src, y, nu, prm = wl["source"], wl["y"], wl["nu"], wl["params"]
    N, Q = y.shape[0], src["jxw"].size
    s = SotSolver(dim=3, device=0, precision="fp64")
    s.setup_source_measure(src)
    s.setup_target(y, nu)
    s.configure(prm)
    s.set_profiling(True)
    psi = torch.tensor(0.2 * prm.epsilon * np.random.default_rng(0).standard_normal(N), dtype=torch.float64,
                       device="cuda")
    H = torch.empty((N, N), dtype=torch.float32, device="cuda")
    for _ in range(max(3, args.warmup)):
        s.compute_hessian_device(psi.data_ptr(), H.data_ptr(), method="tensor", out_f32=True)
    with ClockSampler(0) as clk:
        ks = []
        for _ in range(args.steps):
            info = s.compute_hessian_device(psi.data_ptr(), H.data_ptr(), method="tensor", out_f32=True)
            ks.append(info["kernel_ms"])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        psi_n = s.solve_newton(np.zeros(N), prm, hessian="tensor")
        t_newton = time.perf_counter() - t0
        ninfo = dict(s.last_solve_info)
    conv = s.get_convergence_status()
    g = np.zeros(N)
    s.evaluate_functional(psi_n, g)   # FP64 sweeps
    ninfo["final_grad_linf_fp64"] = float(np.max(np.abs(g)))
    s.close()
    kms = float(np.mean(ks))
    flops = 3.0 * Q * N * N  # three BF16 products x 2 Q N^2 / 2 (upper triangle)
    ach = flops / (kms * 1e-3) / 1e12
    mp = _measured_peaks()
    peak = mp.get("bf16_tflops")
    import dataclasses
    prm_b = dataclasses.replace(prm, max_iterations=int(args.baseline_seconds * 20))  # ~50 ms per iteration
    base = _fp64_lbfgs_baseline([{"source": src, "y": y, "nu": nu, "params": prm_b}], args.baseline_seconds)
    line = {"metric": "Newton solves/s at grad linf 1e-8", "value": (1.0 / t_newton) if conv else 0.0,
            "unit": "solves/s", "n_gpus": 1, "steps": args.steps, "warmup": max(3, args.warmup),
            "ms_per_step": 1000 * t_newton, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16 hi+lo tensor-core Hessian (fp32 accumulation, fp64 drains), fp64 value/gradient/CG/line search",
            "data": "synthetic (seeded; no published dataset)",
            "config": {"workload": "hessian_3d", "n_quadrature": int(Q), "n_targets": int(N), "epsilon": prm.epsilon,
                       "tau": 0.0, "tolerance": prm.tolerance},
            "newton": ninfo, "converged": bool(conv),
            "roofline": {"kernel": "k_hessian_tc (tcgen05 BF16 hi+lo, TMEM accumulators)", "bound": "tensor",
                         "achieved": ach, "peak": peak, "unit": "TFLOP/s",
                         "frac": (ach / peak) if peak else None, "traffic": None, "ms_per_launch": kms,
                         "flops_per_launch": flops, "peak_source": mp["source"] + ": bf16_tflops (burst)"},
            "fp64_lbfgs_baseline": base, "clocks": clk.summary()}
    print(json.dumps(line))
    return 0


def _measured_peaks():
    """Roofline denominators: MEASURED_PEAKS.json when present, else the pool's
    earlier measurement (6.65 TB/s copy, 1.59 PFLOP/s bf16 burst); "source" says which."""
    try:
        d = dict(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))))
        d["source"] = "MEASURED_PEAKS.json"
        return d
    except (OSError, ValueError, TypeError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback (MEASURED_PEAKS.json absent)"}


def _submit(srv, p):
    return srv.submit(p["source"], p["y"], p["nu"], p["params"], method=p.get("method", "auto"),
                      precision="fp64", epsilon_scaling_factor=p.get("eps_factor", 10.0),
                      epsilon_scaling_steps=p.get("eps_steps", 1),
                      intermediate_tolerance=p.get("inter_tol", 0.0))


def _solve_requests_through_server(problems, slots, rate, seed, warmup=()):
    """Untimed warm-up requests (all at once, so that every slot has run one),
    then `problems` with Poisson arrivals at `rate` (0: all at once).  Returns
    the timed requests' results, the wall time and their latency statistics."""
    from semidiscreteot_b200 import SolveServer
    rng = np.random.default_rng(seed)
    srv = SolveServer(n_slots=slots)
    for t in [_submit(srv, p) for p in warmup]:
        srv.wait(t, raise_on_error=False)
    srv.reset_stats()   # latencies and peak concurrency of the timed requests only
    tickets = []
    t0 = time.perf_counter()
    next_t = t0
    for p in problems:
        if rate > 0:
            next_t += rng.exponential(1.0 / rate)
            while time.perf_counter() < next_t:
                time.sleep(min(0.005, max(0.0, next_t - time.perf_counter())))
        tickets.append(_submit(srv, p))
    res = [srv.wait(t, raise_on_error=False)[1] for t in tickets]
    wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    return res, wall, st


def run_batched_2d(args):
    """Config 4: the batched problems solved through the solve service (Newton
    with the tensor-core Hessian, epsilon scaling, all submitted at once),
    against one-at-a-time plain FP64 L-BFGS solves."""
    from semidiscreteot_b200 import workloads as W
    probs = W.batched_2d(seed=0, n_problems=args.problems)
    nw = max(args.warmup, args.slots)
    warm = W.batched_2d(seed=1, n_problems=nw)   # other problems of the same distribution
    for p in probs + warm:
        p.update(method="newton", eps_factor=10.0, eps_steps=2, inter_tol=1e-6)
    with ClockSampler(0) as clk:
        res, wall, st = _solve_requests_through_server(probs, args.slots, 0.0, 0, warm)
    conv = sum(r["converged"] for r in res)
    base = _fp64_lbfgs_baseline(probs, args.baseline_seconds)
    line = {"metric": "batched solves/s at grad linf 1e-8", "value": conv / wall, "unit": "solves/s", "n_gpus": 1,
            "steps": 1, "warmup": nw, "ms_per_step": 1000 * wall, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "bf16 hi+lo tensor-core Hessian, fp64 value/gradient/CG/line search",
            "data": "synthetic (seeded; no published dataset)",
            "config": {"workload": "batched_2d", "problems": len(probs), "slots": args.slots,
                       "method": "Newton (tensor-core Hessian), epsilon scaling 2 levels x10, all submitted at once"},
            "converged": conv, "latency_p50_ms": st["p50_ms"], "latency_p99_ms": st["p99_ms"],
            "peak_concurrent": st["peak_running"], "iterations": [r["iterations"] for r in res],
            "fp64_lbfgs_baseline": base,
            "speedup_vs_fp64_lbfgs": (conv / wall) / base["solves_per_s"] if base["solves_per_s"] > 0 else None,
            "clocks": clk.summary()}
    print(json.dumps(line))
    return 0


def serve_requests(n, seed=0, scale=1.0):
    """Config 5's request mix: 80% config-3-like (uniform density cube, uniform
    targets, eps 5e-3), 20% 3D cubes with Gaussian-mixture targets and eps in
    [1e-3, 1e-2]; sizes scaled by `scale` (cells per axis and targets)."""
    from semidiscreteot_b200 import SolverParameters, structured_source
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        if rng.random() < 0.8:
            cells = max(4, int(round(32 * scale)))
            nt = max(64, int(20_000 * scale ** 3))
            src = structured_source(3, cells, 2)
            y = rng.random((nt, 3))
            nu = np.full(nt, 1.0 / nt)
            eps = 5e-3
        else:
            cells = max(4, int(round(np.exp(rng.uniform(np.log(16), np.log(64))) * scale)))
            nt = max(64, int(np.exp(rng.uniform(np.log(5_000), np.log(50_000))) * scale ** 3))
            src = structured_source(3, cells, 2)
            k = 5
            means = rng.uniform(0.2, 0.8, (k, 3))
            comp = rng.integers(0, k, nt)
            y = np.clip(means[comp] + 0.1 * rng.standard_normal((nt, 3)), 0, 1)
            nu = rng.dirichlet(np.ones(nt))
            eps = float(np.exp(rng.uniform(np.log(1e-3), np.log(1e-2))))
        prm = SolverParameters(epsilon=eps, tau=0.0, use_log_sum_exp_trick=True, tolerance=1e-8,
                               solver_control_type="linf", max_iterations=2000)
        out.append({"source": src, "y": y, "nu": nu, "params": prm, "method": "auto",
                    "eps_factor": 4.0, "eps_steps": 2 if eps < 5e-3 else 1, "inter_tol": 1e-6})
    return out


def run_serve_3d(args):
    """Config 5: Poisson arrivals into the solve service; solves/s and p50/p99
    latency at gradient tolerance 1e-8."""
    reqs = serve_requests(args.problems, 0, args.scale)
    nw = max(args.warmup, 2 * args.slots)
    warm = serve_requests(nw, 12345, args.scale)   # other requests of the same mix
    with ClockSampler(0) as clk:
        res, wall, st = _solve_requests_through_server(reqs, args.slots, args.rate, 1, warm)
    conv = sum(r["converged"] for r in res)
    line = {"metric": "served solves/s at grad linf 1e-8 (p50/p99 latency)", "value": conv / wall,
            "unit": "solves/s", "n_gpus": 1, "steps": 1, "warmup": nw, "ms_per_step": 1000 * wall,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16 hi+lo tensor-core Hessian, fp64 value/gradient/CG/line search",
            "data": "synthetic (seeded; no published dataset)",
            "config": {"workload": "serve_3d", "requests": len(reqs), "rate_per_s": args.rate, "slots": args.slots,
                       "scale": args.scale},
            "converged": conv, "latency_p50_ms": st["p50_ms"], "latency_p99_ms": st["p99_ms"],
            "latency_mean_ms": st["mean_ms"], "peak_concurrent": st["peak_running"],
            "methods": [r["method"] for r in res], "clocks": clk.summary()}
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "hessian_3d":
        return run_hessian_3d(args)
    if args.workload == "batched_2d":
        return run_batched_2d(args)
    if args.workload == "serve_3d":
        return run_serve_3d(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
