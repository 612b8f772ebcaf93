"""``BatchSolver``: many untruncated semi-discrete OT problems solved together on one GPU.

Each problem is what one ``SotSolver`` would solve (SotSolver::solve,
src/solvers/SotSolver.cc:105-215, optionally over the epsilon-scaling
sequence of SemiDiscreteOT.cc:878-922); the batch advances all of them with
one batched evaluation per round (see sdot_batch_* in include/sdot.h).
Sources are given in the flattened quadrature layout of
``SotSolver.setup_source`` without cells (the untruncated path never queries
them).
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional

import numpy as np

from . import _lib
from .parameters import SolverParameters
from .solver import SotSolver


class BatchSolver:
    def __init__(self, dim: int = 2, device: int = 0):
        self.dim = int(dim)
        self._L = _lib.load()
        h = C.c_void_p()
        st = self._L.sdot_batch_create(C.byref(h), int(device), self.dim)
        if st != _lib.SDOT_OK:
            raise _lib.SdotError(st, "sdot_batch_create failed (no CUDA device?)")
        self._h = h
        self.sizes: List[int] = []
        self.last_info: dict = {}

    def set_verbose(self, verbose: bool = True):
        self._check(self._L.sdot_batch_set_verbose(self._h, int(bool(verbose))))

    def _check(self, st: int):
        if st != _lib.SDOT_OK:
            raise _lib.SdotError(st, self._L.sdot_batch_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._L.sdot_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add(self, x, jxw, density, y, nu, params: SolverParameters) -> int:
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, self.dim)
        jxw = np.ascontiguousarray(jxw, dtype=np.float64)
        density = np.ascontiguousarray(density, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64).reshape(-1, self.dim)
        nu = np.ascontiguousarray(nu, dtype=np.float64)
        if not (x.shape[0] == jxw.size == density.size) or y.shape[0] != nu.size:
            raise ValueError("inconsistent problem sizes")
        idx = C.c_int(-1)
        cp = SotSolver._cparams(params)
        self._check(self._L.sdot_batch_add(self._h, x.shape[0], x.ctypes.data, jxw.ctypes.data,
                                           density.ctypes.data, y.shape[0], y.ctypes.data, nu.ctypes.data,
                                           C.byref(cp), C.byref(idx)))
        self.sizes.append(int(y.shape[0]))
        return idx.value

    def add_source(self, src: dict, y, nu, params: SolverParameters) -> int:
        return self.add(src["x"], src["jxw"], src["density"], y, nu, params)

    def split(self, flat: np.ndarray) -> List[np.ndarray]:
        return np.split(flat, np.cumsum(self.sizes)[:-1])

    def evaluate(self, psis, fp32: bool = False):
        """One batched evaluation; returns (values[n], list of gradients)."""
        flat = np.ascontiguousarray(np.concatenate([np.asarray(p, dtype=np.float64) for p in psis]))
        g = np.empty_like(flat)
        vals = np.empty(len(self.sizes))
        self._check(self._L.sdot_batch_evaluate(self._h, flat.ctypes.data, g.ctypes.data, vals.ctypes.data,
                                                int(bool(fp32))))
        return vals, self.split(g)

    def solve(self, psis=None, epsilon_scaling_factor: float = 10.0, epsilon_scaling_steps: int = 1,
              intermediate_tolerance: float = 0.0, mixed_precision: bool = True,
              raise_on_line_search: bool = True) -> List[np.ndarray]:
        """Solves every problem and returns the potentials.  A line-search
        failure of some problem (SDOT_ELINESEARCH, reported after all other
        problems have finished) raises, unless raise_on_line_search is False:
        then the potentials are returned all the same, the failed problems
        report converged = False in problem_info, and last_info["status"]
        holds the status."""
        if psis is None:
            flat = np.zeros(sum(self.sizes))
        else:
            flat = np.ascontiguousarray(np.concatenate([np.asarray(p, dtype=np.float64) for p in psis]))
        opts = _lib.BatchOptions(float(epsilon_scaling_factor), int(epsilon_scaling_steps),
                                 float(intermediate_tolerance), int(bool(mixed_precision)))
        info = _lib.BatchInfo()
        st = self._L.sdot_batch_solve(self._h, flat.ctypes.data, C.byref(opts), C.byref(info))
        self.last_info = {"n_problems": info.n_problems, "converged": info.converged, "rounds": info.rounds,
                          "evaluations": info.evaluations, "total_pairs": info.total_pairs,
                          "eval_ms": info.eval_ms, "solve_ms": info.solve_ms, "status": int(st)}
        if st == _lib.SDOT_ELINESEARCH and not raise_on_line_search:
            return self.split(flat)
        self._check(st)
        return self.split(flat)

    @property
    def shape(self) -> List[int]:
        """Launch shape of the batched sweeps: [value CTAs/SM, gradient CTAs/SM, gradient slice target]."""
        out = np.zeros(3, dtype=np.int32)
        self._check(self._L.sdot_batch_get_shape(self._h, out.ctypes.data))
        return [int(v) for v in out]

    def set_shape(self, shape):
        arr = np.ascontiguousarray(shape, dtype=np.int32)
        self._check(self._L.sdot_batch_set_shape(self._h, arr.ctypes.data))

    def last_eval_ms(self) -> float:
        """Device milliseconds of the last batched evaluation."""
        return float(self._L.sdot_batch_last_eval_ms(self._h))

    def autotune(self, psis=None, fp32: bool = True, reps: int = 3):
        """The batch's autotuner (sdot_batch_autotune): returns (shape, cached)."""
        if psis is None:
            flat = np.zeros(sum(self.sizes))
        else:
            flat = np.ascontiguousarray(np.concatenate([np.asarray(p, dtype=np.float64) for p in psis]))
        out = np.zeros(3, dtype=np.int32)
        cached = C.c_int(0)
        self._check(self._L.sdot_batch_autotune(self._h, flat.ctypes.data, int(bool(fp32)), int(reps),
                                                out.ctypes.data, C.byref(cached)))
        return [int(v) for v in out], bool(cached.value)

    def problem_info(self, index: int) -> dict:
        r = _lib.SolveInfo()
        self._check(self._L.sdot_batch_problem_info(self._h, int(index), C.byref(r)))
        return {"iterations": r.iterations, "converged": bool(r.converged), "n_evaluations": r.n_evaluations,
                "last_value": r.last_value, "last_check_value": r.last_check_value, "total_pairs": r.total_pairs}
