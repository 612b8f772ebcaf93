"""The bench line's arithmetic, on CPU (no GPU run): the roofline of the dominant kernel from per-phase times, the
peak fallback, and the workload description.

- roofline_of: the value sweep when it dominates (or on the truncated path): achieved = FP64 flops per pair x pairs
  / its time; the gradient sweep otherwise: pairs / its time against the ex2 rate; frac = achieved / peak.
- _measured_peaks: MEASURED_PEAKS.json when present, else the stated fallback, and it says which.
- workload_config: the configuration keys of the line, from the workload's own arrays.
"""
import json
import os
import sys
import types

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _times(value_ms, grad_ms, launches=2):
    return {"kt": {"value_sweep": {"ms": value_ms * launches, "launches": launches},
                   "gradient_sweep": {"ms": grad_ms * launches, "launches": launches}},
            "pairs_per_step": 1.0e9}


def _wl(name, dim, tau):
    return {"name": name, "dim": dim, "params": types.SimpleNamespace(tau=tau)}


PEAKS = {"fp64_tflops": 30.0, "ex2_gops": 4000.0}


def test_roofline_value_sweep_truncated():
    r = bench.roofline_of(_times(4.0, 0.1), _wl("trunc_3d", 3, 1e-12), PEAKS, "hybrid")
    ach = bench.VALUE_FLOPS_PER_PAIR[3] * 1.0e9 / 4.0e-3 / 1e12
    assert r["bound"] == "fp64" and r["unit"] == "TFLOP/s"
    assert r["achieved"] == pytest.approx(ach) and r["frac"] == pytest.approx(ach / 30.0)
    assert r["ms_per_launch"] == pytest.approx(4.0)
    assert r["traffic"] == bench.TRAFFIC_BYTES[("trunc_3d", "hybrid")]


def test_roofline_gradient_sweep_when_it_dominates_untruncated():
    # untruncated and the gradient sweep slower than the value sweep: the gradient sweep is the kernel
    r = bench.roofline_of(_times(0.02, 0.05), _wl("dense_2d", 2, 0.0), PEAKS, "fp64")
    assert r["bound"] == "mufu" and r["unit"] == "Gex2/s"
    assert r["achieved"] == pytest.approx(1.0e9 / 0.05e-3 / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / 4000.0)
    assert "FP64" in r["kernel"] and r["traffic"] is None
    r = bench.roofline_of(_times(0.05, 0.02), _wl("dense_2d", 2, 0.0), PEAKS, "hybrid")
    assert r["bound"] == "fp64" and r["flops_per_pair"] == bench.VALUE_FLOPS_PER_PAIR[2]


def test_measured_peaks_file_and_fallback(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    p = bench._measured_peaks()
    assert p["source"].startswith("fallback") and p["hbm_gbs"] == 6650.0 and p["bf16_tflops"] == 1590.0
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 7000.0, "bf16_tflops": 1600.0}))
    p = bench._measured_peaks()
    assert p["source"] == "MEASURED_PEAKS.json" and p["hbm_gbs"] == 7000.0


def test_workload_config_keys():
    wl = bench.make_workload("dense_2d", 0.25)
    args = types.SimpleNamespace(precision="hybrid")
    cfg = bench.workload_config(wl, args, 1)
    assert cfg["workload"] == "dense_2d" and cfg["dim"] == 2
    assert cfg["n_cells"] == 16 * 16 and cfg["n_quadrature"] == 16 * 16 * 9 and cfg["n_targets"] == 62
    assert cfg["parallelism"] == "single GPU" and cfg["tau"] == 0.0
    assert bench.workload_config(wl, args, 4)["parallelism"] == "source-sharded x4"
