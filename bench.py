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
    ap.add_argument("--workload", default="trunc_3d", choices=["trunc_3d", "dense_2d", "newton_3d"])
    ap.add_argument("--precision", default="hybrid", choices=["hybrid", "fp64", "mixed"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--scale", type=float, default=1.0, help="shrink the workload (tests only)")
    return ap.parse_args()


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


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
