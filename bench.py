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

With the default workload the line also carries (unless --no-extra):
  precision_fp64 : the same evaluation with FP64 exponentials in both sweeps;
  config1        : the dense 2D configuration (64 x 64 cells x 3 x 3 Gauss
                   points = 36,864 points, 1,000 uniform targets, eps = 1e-2,
                   no truncation) with its own value, e2e, roofline, the
                   reference-faithful CPU evaluation over every cell, and the
                   full L-BFGS solve to |g|_inf <= 1e-8 on the GPU and on the
                   CPU (time, iterations).
Clocks are sampled through NVML every 2 ms during every timed region.
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
    ap.add_argument("--like-for-like", type=int, default=16,
                    help="batched_2d: problems of the common subset for the like-for-like arms (0: skip)")
    ap.add_argument("--batched-eval", type=int, default=1,
                    help="batched_2d: time one batched evaluation with default and autotuned shapes (0: skip)")
    ap.add_argument("--precision", default="hybrid", choices=["hybrid", "fp64", "mixed"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="trunc_3d: skip the other-precision figure and the dense 2D (config1) sub-object")
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
# clocks during the timed regions
# ---------------------------------------------------------------------------

class ClockSampler:
    """SM clock, its maximum and the clock-event reasons, sampled every 2 ms
    through NVML while a timed region is open (``with clk.region(): ...``);
    nvidia-smi at 100 ms when NVML is unavailable.  Read-only: no setting of
    the GPU is changed."""

    PERIOD_S = 0.002

    def __init__(self, index: int):
        self.index = index
        self.samples = []          # (sm_mhz, max_mhz, reasons set)
        self._active = threading.Event()
        self._stop = threading.Event()
        self._th = None
        self._smi = None
        self._smi_lines = []
        self._nvml = None

    def _handle(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            try:
                import torch
                uuid = str(torch.cuda.get_device_properties(self.index).uuid)
                h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            return pynvml, h
        except Exception:
            return None

    def __enter__(self):
        self._nvml = self._handle()
        if self._nvml is not None:
            self._th = threading.Thread(target=self._run_nvml, daemon=True)
            self._th.start()
        else:
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            try:
                self._smi = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                              "--format=csv,noheader,nounits", "-lms", "100"],
                                             stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self._th = threading.Thread(target=self._run_smi, daemon=True)
                self._th.start()
            except (OSError, ValueError):
                self._smi = None
        return self

    def _run_nvml(self):
        nv, h = self._nvml
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        while not self._stop.is_set():
            if self._active.is_set():
                try:
                    sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                    mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                    r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((float(sm), float(mx), {k for k, b in bits.items() if r & b}))
                except Exception:
                    pass
                time.sleep(self.PERIOD_S)
            else:
                self._active.wait(0.05)

    def _run_smi(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self._smi.stdout:
            if not self._active.is_set():
                continue
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                self.samples.append((float(f[1]), float(f[2]),
                                     {k for k, v in zip(names, f[5:9]) if v.lower().startswith("active")}))
            except ValueError:
                continue

    class _Region:
        def __init__(self, owner):
            self.owner = owner

        def __enter__(self):
            self.owner._active.set()

        def __exit__(self, *exc):
            self.owner._active.clear()

    def region(self):
        return ClockSampler._Region(self)

    def __exit__(self, *exc):
        self._active.clear()
        self._stop.set()
        if self._smi is not None:
            self._smi.terminate()
            try:
                self._smi.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._smi.kill()
        if self._th is not None:
            self._th.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm = [s[0] for s in self.samples]
        reasons = set().union(*[s[2] for s in self.samples])
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(s[1] for s in self.samples),
                "reasons": sorted(reasons), "samples": len(sm),
                "source": "NVML every 2 ms" if self._nvml is not None else "nvidia-smi every 100 ms"}


# DRAM traffic per launch of the dominant kernels (dram__bytes_read.sum +
# dram__bytes_write.sum), from one ncu capture each:
#   k_fused, trunc_3d (2,097,152 points x 100,000 targets), HYBRID (FP32
#   gradient partials): 130,609,408 read + 167,453,952 written, from
#     ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum,gpu__time_duration.sum
#         --clock-control none -k regex:k_fused -s 3 -c 1 --csv
#         python bench.py --steps 1 --warmup 3 --no-cpu-baseline --no-extra
#   dense sweeps (k_value_dense_tensor, k_grad_dense_tensor, ...), dense_2d: the inputs (0.9 MB) stay in L2, so
#     DRAM traffic is not a meaningful bound there (null).
TRAFFIC_BYTES = {
    ("trunc_3d", "hybrid"): 298063360.0,
}


# ---------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------

def cpu_full(wl, seconds: float, threads: int = 0):
    """The reference-faithful evaluation over every cell of a (small) workload,
    repeated for about `seconds`; returns (pairs/s, cores, description)."""
    from oracle import oracle as orc
    src = wl["source"]
    prm = wl["params"]
    op = orc.Params(epsilon=prm.epsilon, tau=prm.tau, use_log_sum_exp=prm.use_log_sum_exp_trick)
    P = orc.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"], wl["y"], wl["nu"])
    psi = np.zeros(wl["y"].shape[0])
    nthr = threads if threads > 0 else (os.cpu_count() or 1)
    r = P.distance_threshold(psi, op)
    ncell = P.ctr.shape[0]
    reps, pairs, t_all = 0, 0, 0.0
    while t_all < seconds or reps < 2:
        t0 = time.perf_counter()
        _, _, _, pp = P.evaluate_cells(psi, op, r, 0, ncell, faithful=True, threads=nthr)
        t_all += time.perf_counter() - t0
        pairs += pp
        reps += 1
    desc = (f"all {ncell} cells x {reps} evaluations, full target set, psi=0; {pairs} pairs in {t_all:.2f}s; "
            f"reference-faithful FP64 (per-cell O(N) CopyData zeroing + serialised in-order merge), "
            f"OpenMP {nthr} threads")
    return pairs / t_all, nthr, desc


def cpu_solve(wl, threads: int = 0):
    """The oracle's reference-faithful L-BFGS solve (SotSolver::solve with
    deal.II SolverBFGS) from psi = 0 to the workload's tolerance."""
    from oracle import oracle as orc
    src = wl["source"]
    prm = wl["params"]
    op = orc.Params(epsilon=prm.epsilon, tau=prm.tau, use_log_sum_exp=prm.use_log_sum_exp_trick,
                    tolerance=prm.tolerance, solver_control_type=prm.solver_control_type,
                    max_iterations=prm.max_iterations)
    P = orc.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"], wl["y"], wl["nu"])
    nthr = threads if threads > 0 else (os.cpu_count() or 1)
    t0 = time.perf_counter()
    psi, info = P.solve(np.zeros(wl["y"].shape[0]), op, threads=nthr, faithful=True)
    dt = time.perf_counter() - t0
    return {"seconds": dt, "iterations": info["iterations"], "evaluations": info["n_evaluations"],
            "converged": info["converged"], "final_grad_linf": info["last_check_value"], "cores": nthr,
            "kind": "port", "method": "reference-faithful FP64 L-BFGS (deal.II SolverBFGS rules), psi0 = 0"}


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
    if args.workload == "trunc_3d" and not args.no_extra:
        c1 = make_workload("dense_2d", 1.0)
        v1, cores1, desc1 = cpu_full(c1, max(2.0, args.cpu_seconds / 4))
        line["config1"] = {"workload": "dense_2d", "value": v1, "unit": "pairs/s", "cores": cores1, "kind": "port",
                           "sample": desc1, "solve": cpu_solve(c1)}
    print(json.dumps(line))
    return 0


def _make_single(wl, precision, local):
    from semidiscreteot_b200 import SotSolver
    s = SotSolver(dim=wl["dim"], device=local, precision=precision)
    s.setup_source_measure(wl["source"])
    s.setup_target(wl["y"], wl["nu"])
    s.configure(wl["params"])
    return s


def measure_single(wl, precision, steps, warmup, local, clk, flush, e2e=True):
    """Device-timed evaluations of one workload on one GPU (inputs resident,
    L2 flushed before each step, CUDA events on the library's stream), then
    the same through the host API with pinned host buffers (e2e)."""
    import torch
    dev = torch.device("cuda", local)
    solver = _make_single(wl, precision, local)
    stream = torch.cuda.ExternalStream(solver.stream_handle, device=dev)
    N = wl["y"].shape[0]
    psi = torch.zeros(N, dtype=torch.float64, device=dev)
    grad = torch.empty(N, dtype=torch.float64, device=dev)
    for _ in range(max(3, warmup)):
        solver.evaluate_functional_device(psi.data_ptr(), grad.data_ptr())
    torch.cuda.synchronize()

    def timed(profiled):
        solver.set_profiling(profiled)
        solver.kernel_times(reset=True)
        ts = []
        torch.cuda.synchronize()
        with clk.region():
            for _ in range(steps):
                with torch.cuda.stream(stream):
                    flush.fill_(1.0)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                solver.evaluate_functional_device(psi.data_ptr(), grad.data_ptr())
                e1.record(stream)
                e1.synchronize()
                ts.append(e0.elapsed_time(e1))
            torch.cuda.synchronize()
        k = solver.kernel_times(reset=True)
        solver.set_profiling(False)
        return ts, k

    # the step time without the library's per-phase events (which add a few
    # microseconds per evaluation), then the same steps with them: the
    # per-kernel CUDA-event times of the roofline and the launch count
    times, _ = timed(False)
    _, kt = timed(True)
    pairs = solver.last_eval_info["n_pairs"]
    ms = float(np.mean(times))
    out = {"value": pairs / (ms * 1e-3), "ms_per_step": ms, "pairs_per_step": pairs, "kt": kt,
           "gpu_launches": int(sum(v["launches"] for v in kt.values()))}
    if e2e:
        hpsi = torch.zeros(N, dtype=torch.float64).pin_memory()
        hgrad = torch.empty(N, dtype=torch.float64).pin_memory()
        psi_np, grad_np = hpsi.numpy(), hgrad.numpy()
        for _ in range(2):
            solver.evaluate_functional(psi_np, grad_np)
        et = []
        with clk.region():
            for _ in range(steps):
                with torch.cuda.stream(stream):
                    flush.fill_(1.0)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                solver.evaluate_functional(psi_np, grad_np)
                e1.record(stream)
                e1.synchronize()
                et.append(e0.elapsed_time(e1))
        out["e2e"] = {"value": pairs / (float(np.mean(et)) * 1e-3), "unit": "pairs/s",
                      "h2d_bytes_per_step": int(N * 8), "d2h_bytes_per_step": int(N * 8 + 8),
                      "ms_per_step": float(np.mean(et))}
    solver.close()
    return out


def roofline_of(m, wl, peaks, precision):
    """Roofline of the dominant kernel from the per-phase CUDA-event times."""
    kt = m["kt"]
    dim = wl["dim"]
    tv = kt["value_sweep"]["ms"] / max(1, kt["value_sweep"]["launches"])
    tg = kt["gradient_sweep"]["ms"] / max(1, kt["gradient_sweep"]["launches"])
    pairs = m["pairs_per_step"]
    truncated = wl["params"].tau > 0
    if tv >= tg or truncated:
        ach = VALUE_FLOPS_PER_PAIR[dim] * pairs / (tv * 1e-3) / 1e12
        kname = ("k_fused (FP64 exp2 value sweep + FP32 ex2 gradient sweep, one kernel)" if truncated else
                 "dense FP64 value sweep: k_value_dense_tensor (per tensor-grid cell and target slice; one "
                 "exponential per cell and target on uniform grids) + k_value_dense_merge, or per point; flops "
                 "counted for the unfactored form")
        return {"kernel": kname, "bound": "fp64", "achieved": ach, "peak": peaks["fp64_tflops"], "unit": "TFLOP/s",
                "frac": ach / peaks["fp64_tflops"], "traffic": TRAFFIC_BYTES.get((wl["name"], precision)),
                "flops_per_pair": VALUE_FLOPS_PER_PAIR[dim], "ms_per_launch": tv,
                "peak_source": "measured on this GPU by sdot_measure_peaks (FP64 FMA chains); "
                               "MEASURED_PEAKS.json has no FP64 figure"}
    ach = pairs / (tg * 1e-3) / 1e9
    return {"kernel": "k_grad_dense_tensor / k_grad_dense (FP32 ex2 gradient sweep)" if precision != "fp64" else
            "k_grad_dense_tensor / k_grad_dense (FP64 exp2 gradient sweep)", "bound": "mufu", "achieved": ach,
            "peak": peaks["ex2_gops"], "unit": "Gex2/s", "frac": ach / peaks["ex2_gops"],
            "traffic": TRAFFIC_BYTES.get((wl["name"], precision)), "ms_per_launch": tg,
            "peak_source": "measured on this GPU by sdot_measure_peaks (ex2.approx chains)"}


def measure_config1(args, local, clk, flush, peaks):
    """The dense 2D configuration (64 x 64 cells x 3 x 3 Gauss points, 1,000
    targets, eps = 1e-2, untruncated): evaluation throughput (device and e2e),
    its roofline, the reference-faithful CPU evaluation over every cell, and
    the full L-BFGS solve to |g|_inf <= 1e-8 on the GPU and on the CPU."""
    import torch
    wl = make_workload("dense_2d", 1.0)
    steps = max(args.steps, 200)   # 0.3 ms steps: enough of them for a timed region the clocks cover
    m = measure_single(wl, args.precision, steps, args.warmup, local, clk, flush)
    out = {"workload": "dense_2d", "n_quadrature": int(wl["source"]["jxw"].size), "n_targets": int(wl["y"].shape[0]),
           "epsilon": wl["params"].epsilon, "tau": 0.0, "precision": args.precision, "steps": steps,
           "value": m["value"], "unit": "pairs/s", "ms_per_step": m["ms_per_step"],
           "pairs_per_step": m["pairs_per_step"], "e2e": m["e2e"], "roofline": roofline_of(m, wl, peaks, args.precision),
           "kernel_ms_per_step": {k: v["ms"] / steps for k, v in m["kt"].items()},
           "gpu_launches": m["gpu_launches"]}
    # full solve on the GPU (FP64 sweeps, L-BFGS like the reference)
    s = _make_single(wl, "fp64", local)
    N = wl["y"].shape[0]
    s.solve(np.zeros(N), wl["params"])   # warm-up (first-use costs)
    torch.cuda.synchronize()
    with clk.region():
        t0 = time.perf_counter()
        psi = s.solve(np.zeros(N), wl["params"])
        t_gpu = time.perf_counter() - t0
    gpu = {"seconds": t_gpu, "iterations": int(s.get_last_iteration_count()),
           "evaluations": int(s.last_solve_info.get("n_evaluations", 0)), "converged": bool(s.get_convergence_status()),
           "final_grad_linf": float(s.last_solve_info.get("last_check_value", float("nan"))),
           "method": "sdot_solve (L-BFGS, FP64 sweeps), psi0 = 0, host wall clock"}
    s.close()
    if not args.no_cpu_baseline:
        from oracle import oracle as orc
        src = wl["source"]
        P = orc.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"],
                        wl["y"], wl["nu"])
        op = orc.Params(epsilon=wl["params"].epsilon, tau=0.0, use_log_sum_exp=True)
        _, go, _ = P.evaluate(psi, op)
        gpu["oracle_grad_linf_at_gpu_psi"] = float(np.max(np.abs(go)))
        v, cores, desc = cpu_full(wl, max(2.0, args.cpu_seconds / 4))
        out["cpu_baseline"] = {"value": v, "unit": "pairs/s", "cores": cores, "kind": "port", "sample": desc}
        cpu = cpu_solve(wl)
        out["solve"] = {"gpu": gpu, "cpu": cpu, "speedup": cpu["seconds"] / t_gpu if t_gpu > 0 else None}
    else:
        out["solve"] = {"gpu": gpu}
    return out


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
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    wl = make_workload(args.workload, args.scale)
    dim = wl["dim"]

    if world == 1:
        with ClockSampler(local) as clk:
            m = measure_single(wl, args.precision, args.steps, args.warmup, local, clk, flush)
            peaks = SotSolver.measure_peaks(local)
            extra = {}
            if args.workload == "trunc_3d" and not args.no_extra:
                other = "fp64" if args.precision != "fp64" else "hybrid"
                mo = measure_single(wl, other, args.steps, args.warmup, local, clk, flush, e2e=False)
                extra[f"precision_{other}"] = {"value": mo["value"], "unit": "pairs/s",
                                               "ms_per_step": mo["ms_per_step"],
                                               "pairs_per_step": mo["pairs_per_step"],
                                               "kernel_ms_per_step": {k: v["ms"] / args.steps
                                                                      for k, v in mo["kt"].items()}}
                extra["config1"] = measure_config1(args, local, clk, flush, peaks)
        t_ms = m["ms_per_step"]
        pairs = m["pairs_per_step"]
        line = {"metric": "LSE dual-gradient pairs/s", "value": m["value"], "unit": "pairs/s", "n_gpus": 1,
                "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": t_ms, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "f64 value sweep + f32 exp gradient sweep",
                "data": "synthetic (seeded; no published dataset)", "config": workload_config(wl, args, 1),
                "pairs_per_step": pairs, "roofline": roofline_of(m, wl, peaks, args.precision),
                "kernel_ms_per_step": {k: v["ms"] / args.steps for k, v in m["kt"].items()},
                "gpu_launches": m["gpu_launches"], "clocks": clk.summary(), "peaks_measured": peaks,
                "e2e": m["e2e"]}
        if not args.no_cpu_baseline:
            v, cores, desc, _ = cpu_sample(wl, args.cpu_seconds)
            line["cpu_baseline"] = {"value": v, "unit": "pairs/s", "cores": cores, "kind": "port", "sample": desc}
        line.update(extra)
        print(json.dumps(line))
        return 0

    # N > 1: source cells sharded over the ranks, one all-reduce of n_targets + 3 doubles per step
    import datetime
    import torch.distributed as dist
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    N = wl["y"].shape[0]
    solver = DistributedSotSolver(dim, rank, world, device=local, precision=args.precision)
    solver.setup_source(wl["source"])
    solver.setup_target(wl["y"], wl["nu"])
    solver.configure(wl["params"])
    lib = solver.local
    stream = torch.cuda.ExternalStream(lib.stream_handle, device=dev)
    psi = torch.zeros(N, dtype=torch.float64, device=dev)
    for _ in range(max(3, args.warmup)):
        solver.evaluate(psi)
    torch.cuda.synchronize()
    lib.set_profiling(True)
    lib.kernel_times(reset=True)
    times, pairs = [], 0.0
    dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        with clk.region():
            for _ in range(args.steps):
                with torch.cuda.stream(stream):
                    flush.fill_(1.0)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                _, _, _, pairs = solver.evaluate(psi)
                e1.record(stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
            torch.cuda.synchronize()
    kt = lib.kernel_times(reset=True)
    lib.set_profiling(False)
    t = torch.tensor([float(np.mean(times))], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    t_ms = float(t.item())
    dist.barrier()
    if rank == 0:
        value = pairs / (t_ms * 1e-3)
        peaks = SotSolver.measure_peaks(local)
        m = {"kt": kt, "pairs_per_step": lib.last_eval_info["n_pairs"]}
        line = {"metric": "LSE dual-gradient pairs/s", "value": value, "unit": "pairs/s", "n_gpus": world,
                "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": t_ms, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "f64 value sweep + f32 exp gradient sweep",
                "data": "synthetic (seeded; no published dataset)", "config": workload_config(wl, args, world),
                "pairs_per_step": pairs, "roofline": roofline_of(m, wl, peaks, args.precision),
                "kernel_ms_per_step": {k: v["ms"] / args.steps for k, v in kt.items()},
                "gpu_launches": int(sum(v["launches"] for v in kt.values())), "clocks": clk.summary(),
                "peaks_measured": peaks}
        print(json.dumps(line))
    solver.close()
    dist.destroy_process_group()
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
    with ClockSampler(0) as clk, clk.region():
        ks = []
        for _ in range(args.steps):
            info = s.compute_hessian_device(psi.data_ptr(), H.data_ptr(), method="tensor", out_f32=True)
            ks.append(info["kernel_ms"])
        factored = s.set_hessian_generation(None)
        # the per-point operand generation on the same problem, for comparison
        s.set_hessian_generation(False)
        kp = [s.compute_hessian_device(psi.data_ptr(), H.data_ptr(), method="tensor", out_f32=True)["kernel_ms"]
              for _ in range(2)]
        s.set_hessian_generation(True)
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
                         "flops_per_launch": flops, "peak_source": mp["source"] + ": bf16_tflops (burst)",
                         "operand_generation": "factored per 2x2x2 cell" if factored else "per point",
                         "per_point_generation_ms_per_launch": float(np.mean(kp))},
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


def _one_at_a_time(problems, seconds, method, hessian="fp64"):
    """Each problem alone (one context, no concurrency), in order, until the
    wall budget is spent: method "newton" (sdot_solve_newton with the given
    Hessian method) or "lbfgs" (sdot_solve); FP64 evaluations; the problem's
    epsilon scaling (levels eps f^(s-1), ..., eps, warm started, intermediate
    tolerance), as the solve service applies it.  Convergence is the FP64
    gradient's linf norm at the final epsilon."""
    import dataclasses
    from semidiscreteot_b200 import SotSolver
    t_all, done, conv, iters = 0.0, 0, 0, []
    for p in problems:
        if t_all >= seconds:
            break
        s = SotSolver(dim=p["y"].shape[1], device=0, precision="fp64")
        s.setup_source_measure(p["source"])
        s.setup_target(p["y"], p["nu"])
        prm = p["params"]
        f, steps, inter = p.get("eps_factor", 10.0), max(1, p.get("eps_steps", 1)), p.get("inter_tol", 0.0)
        psi = np.zeros(len(p["nu"]))
        it = 0
        t0 = time.perf_counter()
        try:
            for lvl in range(steps):
                last = lvl == steps - 1
                pl = dataclasses.replace(prm, epsilon=prm.epsilon * f ** (steps - 1 - lvl),
                                         tolerance=prm.tolerance if (last or inter <= 0) else inter)
                psi = s.solve_newton(psi, pl, hessian=hessian) if method == "newton" else s.solve(psi, pl)
                it += int(s.get_last_iteration_count())
            ok = bool(s.get_convergence_status())
        except RuntimeError:
            ok = False
        t_all += time.perf_counter() - t0
        iters.append(it)
        done += 1
        conv += ok
        s.close()
    return {"solves_per_s": conv / t_all if t_all > 0 else 0.0, "attempted": done, "converged": conv,
            "seconds": t_all, "iterations": iters}


def _batched_evaluation(probs, reps=5):
    """One batched evaluation of every problem in one persistent launch
    (sdot_batch, FP32-exponential gradient sweep): device time with the
    default launch shape and with the shape the batch's autotuner picks."""
    from semidiscreteot_b200 import BatchSolver
    b = BatchSolver(dim=2)
    for p in probs:
        b.add_source(p["source"], p["y"], p["nu"], p["params"])
    psis = [np.zeros(len(p["nu"])) for p in probs]
    pairs = float(sum(p["source"]["jxw"].size * len(p["nu"]) for p in probs))

    def timed():
        b.evaluate(psis, fp32=True)   # warm-up
        ms = []
        for _ in range(reps):
            b.evaluate(psis, fp32=True)
            ms.append(b.last_eval_ms())
        return float(np.median(ms))

    default_shape = b.shape
    t_default = timed()
    t0 = time.perf_counter()
    shape, cached = b.autotune(psis, fp32=True, reps=3)
    tune_s = time.perf_counter() - t0
    t_tuned = timed()
    b.close()
    return {"problems": len(probs), "pairs": pairs, "default_shape": default_shape, "default_ms": t_default,
            "default_pairs_per_s": pairs / (t_default * 1e-3), "tuned_shape": shape, "tuned_ms": t_tuned,
            "tuned_pairs_per_s": pairs / (t_tuned * 1e-3), "tuning_seconds": tune_s, "cached": cached,
            "shape_fields": "[value CTAs/SM, gradient CTAs/SM, gradient slice target per SM]"}


def run_batched_2d(args):
    """Config 4: the batched problems solved through the solve service (Newton
    with the tensor-core Hessian, epsilon scaling, all submitted at once),
    against one-at-a-time plain FP64 L-BFGS solves; like-for-like comparisons
    on a common subset; the batched evaluation with autotuned launch shapes."""
    from semidiscreteot_b200 import workloads as W
    probs = W.batched_2d(seed=0, n_problems=args.problems)
    nw = max(args.warmup, args.slots)
    warm = W.batched_2d(seed=1, n_problems=nw)   # other problems of the same distribution
    for p in probs + warm:
        p.update(method="newton", eps_factor=10.0, eps_steps=2, inter_tol=1e-6)
    with ClockSampler(0) as clk, clk.region():
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
    if args.like_for_like > 0:
        # the same problems (the first K), the same epsilon scaling and FP64 convergence test in every arm
        sub = probs[:args.like_for_like]
        with clk.region():
            rs, wall_s, _ = _solve_requests_through_server(sub, args.slots, 0.0, 0)
        served = sum(r["converged"] for r in rs) / wall_s
        arms = {"service_tc_newton": {"solves_per_s": served, "converged": sum(r["converged"] for r in rs),
                                      "attempted": len(sub), "seconds": wall_s},
                "one_at_a_time_tc_newton": _one_at_a_time(sub, args.baseline_seconds, "newton", "tensor"),
                "one_at_a_time_fp64_newton": _one_at_a_time(sub, args.baseline_seconds, "newton", "fp64"),
                "one_at_a_time_fp64_lbfgs": _one_at_a_time(sub, args.baseline_seconds, "lbfgs")}
        ref = arms["one_at_a_time_fp64_newton"]["solves_per_s"]
        line["like_for_like"] = {
            "problems": len(sub), "arms": arms,
            "service_vs_fp64_newton": served / ref if ref > 0 else None,
            "note": "service = mixed precision (BF16 tensor-core Hessian) + concurrency; one_at_a_time_tc_newton "
                    "isolates the precision; one_at_a_time_fp64_newton is the plain FP64 path of the same method"}
    if args.batched_eval:
        line["batched_evaluation"] = _batched_evaluation(probs)
    print(json.dumps(line))
    return 0


def serve_requests(n, seed=0, scale=1.0):
    """Config 5's request mix: 80% config-3-like (uniform density cube, uniform
    targets, eps 5e-3), 20% 3D cubes with Gaussian-mixture targets and eps in
    [1e-3, 1e-2]; all untruncated (Newton with the tensor-core Hessian up to
    46,340 targets); sizes scaled by `scale` (cells per axis and targets)."""
    from semidiscreteot_b200 import SolverParameters, structured_source
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        tau, maxit, kind = 0.0, 2000, "config3"
        if rng.random() < 0.8:
            cells = max(4, int(round(32 * scale)))
            nt = max(64, int(20_000 * scale ** 3))
            src = structured_source(3, cells, 2)
            y = rng.random((nt, 3))
            nu = np.full(nt, 1.0 / nt)
            eps = 5e-3
        else:
            kind = "mixture_cube"
            cells = max(4, int(round(np.exp(rng.uniform(np.log(16), np.log(64))) * scale)))
            nt = max(64, int(np.exp(rng.uniform(np.log(5_000), np.log(50_000))) * scale ** 3))
            src = structured_source(3, cells, 2)
            k = 5
            means = rng.uniform(0.2, 0.8, (k, 3))
            comp = rng.integers(0, k, nt)
            y = np.clip(means[comp] + 0.1 * rng.standard_normal((nt, 3)), 0, 1)
            nu = rng.dirichlet(np.ones(nt))
            eps = float(np.exp(rng.uniform(np.log(1e-3), np.log(1e-2))))
        prm = SolverParameters(epsilon=eps, tau=tau, use_log_sum_exp_trick=True, tolerance=1e-8,
                               solver_control_type="linf", max_iterations=maxit)
        out.append({"source": src, "y": y, "nu": nu, "params": prm, "method": "auto", "kind": kind,
                    "eps_factor": 4.0, "eps_steps": 2 if eps < 5e-3 else 1, "inter_tol": 1e-6})
    return out


def run_serve_3d(args):
    """Config 5: Poisson arrivals into the solve service; solves/s and p50/p99
    latency at gradient tolerance 1e-8."""
    reqs = serve_requests(args.problems, 0, args.scale)
    nw = max(args.warmup, 2 * args.slots)
    warm = serve_requests(nw, 12345, args.scale)   # other requests of the same mix
    with ClockSampler(0) as clk, clk.region():
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
            "methods": [r["method"] for r in res], "clocks": clk.summary(),
            "requests_detail": [{"kind": p["kind"], "n_q": int(p["source"]["jxw"].size), "n_t": int(len(p["nu"])),
                                 "epsilon": p["params"].epsilon, "tau": p["params"].tau, "method": r["method"],
                                 "iterations": int(r["iterations"]), "converged": bool(r["converged"]),
                                 "queue_ms": round(r["queue_ms"], 1), "run_ms": round(r["run_ms"], 1)}
                                for p, r in zip(reqs, res)]}
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
