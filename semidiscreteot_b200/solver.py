"""``SotSolver``: the reference's solver interface on top of ``libsdot_cuda``.

Mirrors ``SotSolver<dim, spacedim>`` (include/SemiDiscreteOT/solvers/SotSolver.h
:54-525): the same method names, argument meaning and error behaviour, with
numpy arrays in place of deal.II types.  deal.II ``DoFHandler``/``Mapping``
objects cannot cross the C ABI, so ``setup_source`` takes the flattened
quadrature data that ``SemiDiscreteOT::save_discrete_measures`` writes
(src/core/SemiDiscreteOT.cc:2489-2558); ``source.structured_source`` builds it
for structured Q1 meshes.

Errors raise ``RuntimeError`` (``SdotError``) like the reference's exceptions,
except non-convergence of ``solve``, which the reference swallows
(SotSolver.cc:207-211) and reports through ``get_convergence_status()``.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from .parameters import SolverParameters


def _f64(a, shape=None) -> np.ndarray:
    out = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        out = out.reshape(shape)
    return out


class SotSolver:
    """Entropic semi-discrete OT dual solver on one GPU (one CUDA stream)."""

    def __init__(self, dim: int = 3, device: int = 0, precision: str = "hybrid",
                 memory_budget: int = 0, verbose: bool = False):
        self.dim = int(dim)
        self._L = _lib.load()
        opts = _lib.Options(int(device), _lib.PRECISION[precision], int(memory_budget), int(verbose))
        h = C.c_void_p()
        st = self._L.sdot_create(C.byref(h), C.byref(opts))
        if st != _lib.SDOT_OK:
            raise _lib.SdotError(st, "sdot_create failed (no CUDA device?)")
        self._h = h
        self.device = int(device)
        self.precision = precision
        self.current_params = SolverParameters()
        self._n_targets = 0
        self.last_eval_info: dict = {}
        self.last_solve_info: dict = {}

    # ------------------------------------------------------------------ utils
    def _check(self, st: int):
        if st != _lib.SDOT_OK:
            msg = self._L.sdot_last_error(self._h).decode()
            raise _lib.SdotError(st, msg)

    def close(self):
        if getattr(self, "_h", None):
            self._L.sdot_destroy(self._h)
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

    @staticmethod
    def _cparams(p: SolverParameters) -> _lib.SolverParams:
        return _lib.SolverParams(int(p.max_iterations), float(p.tolerance),
                                 _lib.CONTROL[p.solver_control_type], float(p.epsilon), float(p.tau),
                                 _lib.THRESHOLD[p.distance_threshold_type], int(bool(p.use_log_sum_exp_trick)),
                                 _lib.LINE_SEARCH[p.line_search])

    # ------------------------------------------------------------- measures
    def setup_source(self, x, jxw, density, cell_offsets, cell_centers):
        """SotSolver::setup_source (SotSolver.cc:43-51) on flattened quadrature data."""
        x = _f64(x).reshape(-1, self.dim)
        jxw = _f64(jxw)
        density = _f64(density)
        off = np.ascontiguousarray(cell_offsets, dtype=np.int64)
        ctr = _f64(cell_centers).reshape(-1, self.dim)
        if not (x.shape[0] == jxw.size == density.size):
            raise ValueError("x, jxw and density must have one entry per quadrature point")
        if off.size != ctr.shape[0] + 1:
            raise ValueError("cell_offsets must have n_cells + 1 entries")
        self._check(self._L.sdot_set_source(self._h, self.dim, x.shape[0], x.ctypes.data, jxw.ctypes.data,
                                            density.ctypes.data, ctr.shape[0], off.ctypes.data, ctr.ctypes.data))
        self._src = (x, jxw, density, off, ctr)

    def setup_source_measure(self, src: dict):
        self.setup_source(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"])

    def setup_target(self, target_points, target_density):
        """SotSolver::setup_target (SotSolver.cc:53-60); weights are not normalised."""
        y = _f64(target_points).reshape(-1, self.dim)
        nu = _f64(target_density)
        if y.shape[0] != nu.size:
            raise ValueError(f"Dimension mismatch: {y.shape[0]} != {nu.size}")
        self._check(self._L.sdot_set_target(self._h, y.shape[0], y.ctypes.data, nu.ctypes.data))
        self._n_targets = y.shape[0]

    def configure(self, params: SolverParameters):
        """SotSolver::configure (SotSolver.cc:62-69)."""
        self.current_params = params
        cp = self._cparams(params)
        self._check(self._L.sdot_configure(self._h, C.byref(cp)))

    def set_distance_function(self, name: str):
        """SotSolver::set_distance_function: "euclidean" or "spherical"."""
        self._check(self._L.sdot_set_distance_function(self._h, name.encode()))
        self.distance = name

    # ------------------------------------------------------------- hot path
    def evaluate_functional(self, potential, gradient_out: Optional[np.ndarray] = None) -> float:
        """SotSolver::evaluate_functional (SotSolver.cc:217-377): returns J(psi);
        the gradient sum_q w_q pi_qj - nu_j is written into gradient_out."""
        psi = _f64(potential)
        if psi.size != self._n_targets:
            raise ValueError("potential size differs from the number of targets")
        g = gradient_out if (gradient_out is not None and gradient_out.dtype == np.float64
                             and gradient_out.flags.c_contiguous) else np.empty(self._n_targets)
        val = C.c_double(0.0)
        info = _lib.EvalInfo()
        self._check(self._L.sdot_evaluate(self._h, psi.ctypes.data, g.ctypes.data, C.byref(val), C.byref(info)))
        if gradient_out is not None and g is not gradient_out:
            gradient_out[...] = g
        self.last_eval_info = {"value": info.value, "C_global": info.C_global, "threshold": info.threshold,
                               "n_pairs": info.n_pairs, "device_ms": info.device_ms}
        self._last_grad = g
        return val.value

    def evaluate_functional_device(self, psi_ptr: int, grad_ptr: int) -> float:
        """Evaluation on device pointers (caller ordering, context's device)."""
        val = C.c_double(0.0)
        info = _lib.EvalInfo()
        self._check(self._L.sdot_evaluate_device(self._h, C.c_void_p(psi_ptr), C.c_void_p(grad_ptr),
                                                 C.byref(val), C.byref(info)))
        self.last_eval_info = {"value": info.value, "C_global": info.C_global, "threshold": info.threshold,
                               "n_pairs": info.n_pairs, "device_ms": info.device_ms}
        return val.value

    def evaluate_functional_device_noalloc(self, psi_ptr: int, grad_ptr: int) -> float:
        """Untruncated evaluation on device pointers that allocates no device
        memory (scratch in a static device array of NOALLOC_SCRATCH_BYTES per
        device; overlapping calls on one device race).  Same results as
        evaluate_functional_device."""
        val = C.c_double(0.0)
        self._check(self._L.sdot_evaluate_device_noalloc(self._h, C.c_void_p(psi_ptr), C.c_void_p(grad_ptr),
                                                         C.byref(val)))
        return val.value

    def solve(self, potential: np.ndarray, params: Optional[SolverParameters] = None) -> np.ndarray:
        """SotSolver::solve (SotSolver.cc:105-215): L-BFGS on the device.
        ``potential`` is updated in place when it is a float64 C-contiguous array."""
        if params is not None:
            self.current_params = params
        if potential is None or np.asarray(potential).size != self._n_targets:
            psi = np.zeros(self._n_targets)   # potentials.reinit(n) (SotSolver.cc:151-153)
        else:
            psi = potential if (isinstance(potential, np.ndarray) and potential.dtype == np.float64
                                and potential.flags.c_contiguous) else _f64(potential).copy()
        cp = self._cparams(self.current_params)
        info = _lib.SolveInfo()
        st = self._L.sdot_solve(self._h, psi.ctypes.data, C.byref(cp), C.byref(info))
        self.last_solve_info = {"iterations": info.iterations, "converged": bool(info.converged),
                                "n_evaluations": info.n_evaluations, "last_value": info.last_value,
                                "last_check_value": info.last_check_value, "total_pairs": info.total_pairs,
                                "device_ms": info.device_ms}
        self._check(st)
        if isinstance(potential, np.ndarray) and potential is not psi and potential.size == psi.size:
            potential[...] = psi
        return psi

    def solve_newton(self, potential: np.ndarray, params: Optional[SolverParameters] = None,
                     hessian: str = "auto") -> np.ndarray:
        """Newton solve with the tensor-core Hessian (sdot_solve_newton): same
        parameters, convergence control and in-place update as ``solve``."""
        psi = _f64(potential).copy()
        if psi.size != self._n_targets:
            raise ValueError("potential size does not match the number of targets")
        if params is not None:
            self.current_params = params
        cp = self._cparams(self.current_params)
        info = _lib.NewtonInfo()
        st = self._L.sdot_solve_newton(self._h, psi.ctypes.data, C.byref(cp), _lib.HESSIAN_METHOD[hessian],
                                       C.byref(info))
        names = {v: k for k, v in _lib.HESSIAN_METHOD.items()}
        self.last_solve_info = {"iterations": info.iterations, "converged": bool(info.converged),
                                "n_evaluations": info.n_evaluations, "cg_iterations": info.cg_iterations,
                                "last_value": info.last_value, "last_check_value": info.last_check_value,
                                "total_pairs": info.total_pairs, "eval_ms": info.eval_ms,
                                "hessian_ms": info.hessian_ms, "cg_ms": info.cg_ms,
                                "hessian_method": names.get(info.hessian_method, info.hessian_method),
                                "n_hessians": info.n_hessians}
        # in place also after a failure, like solve (the library writes the last iterate back)
        if isinstance(potential, np.ndarray) and potential is not psi and potential.size == psi.size:
            potential[...] = psi
        self._check(st)
        return psi

    def set_newton_hessian_reuse(self, contraction: float):
        """Lagged Hessians in solve_newton (sdot_set_newton_hessian_reuse): keep the
        previous Hessian after a full step that reduced |g|_2 by `contraction`;
        0 recomputes it every step."""
        self._check(self._L.sdot_set_newton_hessian_reuse(self._h, float(contraction)))

    def softmax_refinement(self, potential_coarse, epsilon: float, threshold: float, y_fine, child_offsets,
                           child_indices, use_log_sum_exp: Optional[bool] = None) -> np.ndarray:
        """SoftmaxRefinement::compute_refinement (SoftmaxRefinement.cc:61-280): fine-level
        potentials from this solver's targets (the coarse level) and their potentials.
        child_offsets / child_indices: CSR children of each coarse target."""
        psi = _f64(potential_coarse)
        yf = _f64(y_fine).reshape(-1, self.dim)
        co = np.ascontiguousarray(child_offsets, dtype=np.int64)
        ci = np.ascontiguousarray(child_indices, dtype=np.int64)
        if psi.size != self._n_targets or co.size != self._n_targets + 1:
            raise ValueError("coarse potentials / child offsets do not match the coarse targets")
        lse = self.current_params.use_log_sum_exp_trick if use_log_sum_exp is None else use_log_sum_exp
        out = np.zeros(yf.shape[0])
        self._check(self._L.sdot_softmax_refinement(self._h, psi.ctypes.data, float(epsilon), float(threshold),
                                                    int(bool(lse)), yf.shape[0], yf.ctypes.data, co.ctypes.data,
                                                    ci.ctypes.data, out.ctypes.data))
        return out

    def evaluate_weighted_barycenters(self, potential, params: Optional[SolverParameters] = None,
                                      barycenters=None) -> np.ndarray:
        """SotSolver::evaluate_weighted_barycenters (SotSolver.cc:584-660).  Euclidean distance
        (:871-971): barycenter_j = sum_q rho_q JxW_q pi_qj x_q / nu_j at the given potentials,
        threshold recomputed there.  Spherical distance (:612-650, 662-767): Riemannian gradient
        steps from `barycenters` (the starting points, as the reference's barycenters_out) with
        the parameters' tolerance and max_iterations; the iterations run and the last gradient
        norm are left in last_barycenter_info.  Returns (n_targets, dim).  `params` configures
        the solver first; the computation reads the configured epsilon as the reference's
        current_params does."""
        if params is not None:
            self.configure(params)
        psi = _f64(potential)
        if psi.size != self._n_targets:
            raise ValueError("potential size differs from the number of targets")
        if getattr(self, "distance", "euclidean") == "spherical":
            if barycenters is None:
                raise ValueError("the spherical barycenter iteration needs starting points")
            b = np.array(barycenters, dtype=np.float64, copy=True).reshape(self._n_targets, self.dim)
            it = C.c_uint(0)
            nrm = C.c_double(0.0)
            p = self.current_params
            self._check(self._L.sdot_weighted_barycenters_spherical(self._h, psi.ctypes.data, b.ctypes.data,
                                                                     int(p.max_iterations), float(p.tolerance),
                                                                     C.byref(it), C.byref(nrm)))
            self.last_barycenter_info = {"iterations": int(it.value), "grad_norm": float(nrm.value)}
            return b
        out = np.empty((self._n_targets, self.dim))
        self._check(self._L.sdot_weighted_barycenters(self._h, psi.ctypes.data, out.ctypes.data))
        return out

    def get_potential_conditioned_density(self, points, density_at_points, potential, potential_indices,
                                          epsilon: Optional[float] = None,
                                          threshold: Optional[float] = None) -> np.ndarray:
        """SotSolver::get_potential_conditioned_density (SotSolver.cc:973-1046) at the given
        support points: row i is density(p) e^(t_k - m) / sum_j nu_j e^(t_j - m) for target
        k = potential_indices[i] where k is within the threshold of p, else 0.  epsilon and
        threshold default to the configured epsilon and the last distance threshold."""
        P = _f64(points).reshape(-1, self.dim)
        rho = _f64(density_at_points)
        psi = _f64(potential)
        idx = np.ascontiguousarray(potential_indices, dtype=np.int64)
        if rho.size != P.shape[0]:
            raise ValueError("one density value per support point expected")
        if psi.size != self._n_targets:
            raise ValueError("potential size differs from the number of targets")
        eps = self.current_params.epsilon if epsilon is None else float(epsilon)
        thr = self.get_last_distance_threshold() if threshold is None else float(threshold)
        out = np.zeros((idx.size, P.shape[0]))
        self._check(self._L.sdot_conditioned_densities(self._h, psi.ctypes.data, eps, thr, P.shape[0],
                                                       P.ctypes.data, rho.ctypes.data, idx.size,
                                                       idx.ctypes.data, out.ctypes.data))
        return out

    def compute_hessian(self, potential, hessian_out: Optional[np.ndarray] = None) -> np.ndarray:
        """Dense Hessian H = (1/eps) sum_q w_q (diag(pi_q) - pi_q pi_q^T) (declared at SotSolver.h:343-344)."""
        psi = _f64(potential)
        n = self._n_targets
        H = hessian_out if (hessian_out is not None and hessian_out.shape == (n, n) and
                            hessian_out.dtype == np.float64 and hessian_out.flags.c_contiguous) else np.empty((n, n))
        self._check(self._L.sdot_hessian(self._h, psi.ctypes.data, H.ctypes.data))
        if hessian_out is not None and H is not hessian_out:
            hessian_out[...] = H
        return H

    def compute_hessian_device(self, psi_ptr: int, hessian_ptr: int, method: str = "auto",
                               out_f32: bool = False) -> dict:
        """Hessian into device memory (n x n row-major, caller order) by
        ``method`` "fp64" | "tensor" (tcgen05, BF16 hi+lo) | "auto" (see
        sdot_hessian_device); returns the method used and device times."""
        info = _lib.HessianInfo()
        self._check(self._L.sdot_hessian_device(self._h, C.c_void_p(psi_ptr), C.c_void_p(hessian_ptr),
                                                _lib.HESSIAN_METHOD[method], int(bool(out_f32)),
                                                C.byref(info)))
        names = {v: k for k, v in _lib.HESSIAN_METHOD.items()}
        return {"method": names.get(info.method, info.method), "eval_ms": info.eval_ms,
                "hessian_ms": info.hessian_ms, "kernel_ms": info.kernel_ms, "tiles": info.tiles}

    def hessian_tile_count(self) -> int:
        """Number of 128 x 256 upper-triangle tiles of the tensor-core Hessian (sdot_hessian_tile_count)."""
        k = C.c_int64(0)
        self._check(self._L.sdot_hessian_tile_count(self._h, C.byref(k)))
        return k.value

    def compute_hessian_tiles_device(self, psi_ptr: int, hessian_ptr: int, tile_begin: int, tile_end: int,
                                     out_f32: bool = True) -> dict:
        """Tiles [tile_begin, tile_end) of the tensor-core Hessian at psi (sdot_hessian_tiles_device):
        their entries and mirrors are written, every other entry of the n x n buffer is left as it is."""
        info = _lib.HessianInfo()
        self._check(self._L.sdot_hessian_tiles_device(self._h, C.c_void_p(psi_ptr), C.c_void_p(hessian_ptr),
                                                      int(bool(out_f32)), int(tile_begin), int(tile_end),
                                                      C.byref(info)))
        return {"eval_ms": info.eval_ms, "hessian_ms": info.hessian_ms, "kernel_ms": info.kernel_ms,
                "tiles": info.tiles}

    def hessian_matvec_device(self, hessian_ptr: int, x_ptr: int, y_ptr: int, f32: bool = True):
        """y = H x with FP64 accumulation (sdot_hessian_matvec_device); returns when y is complete."""
        self._check(self._L.sdot_hessian_matvec_device(self._h, C.c_void_p(hessian_ptr), int(bool(f32)),
                                                       C.c_void_p(x_ptr), C.c_void_p(y_ptr)))

    def set_hessian_chunk(self, stages: int):
        """Stages of 64 points accumulated in FP32 between FP64 drains (tensor Hessian)."""
        self._check(self._L.sdot_set_hessian_chunk(self._h, int(stages)))

    def set_hessian_generation(self, factored: Optional[bool] = None) -> bool:
        """Factored operand generation of the tensor Hessian on 2x2x2 Gauss cells
        (True: where it applies, the default; False: never; None: unchanged).
        Returns whether the last tensor Hessian used it."""
        last = C.c_int(0)
        self._check(self._L.sdot_set_hessian_generation(self._h, -1 if factored is None else int(bool(factored)),
                                                        C.byref(last)))
        return bool(last.value)

    def set_hessian_pairs(self, mode: Optional[int] = None) -> int:
        """Whole tensor Hessians on SM pairs (tcgen05 cta_group::2 over 256 x 256
        tiles): 2 (default) with two generation groups and an MMA warp per CTA,
        1 with one group, 0 on single SMs; None leaves the setting (True / False
        mean 2 / 0).  Returns the mode the last tensor Hessian ran in."""
        last = C.c_int(0)
        m = -1 if mode is None else (2 if mode is True else (0 if mode is False else int(mode)))
        self._check(self._L.sdot_set_hessian_pairs(self._h, m, C.byref(last)))
        return int(last.value)

    def set_hessian_wait_limit(self, clocks: int):
        """SM clocks a device-side wait of the tensor Hessian may take before the
        call fails with SDOT_ETIMEOUT (<= 0: the default, about 1 s)."""
        self._check(self._L.sdot_set_hessian_wait_limit(self._h, int(clocks)))

    def evaluate_partial_device(self, psi_ptr: int, out_ptr: int) -> dict:
        """Source-shard evaluation into out[n_targets + 3] on the device (see
        sdot_evaluate_partial_device); the caller all-reduces and finishes."""
        info = _lib.EvalInfo()
        self._check(self._L.sdot_evaluate_partial_device(self._h, C.c_void_p(psi_ptr), C.c_void_p(out_ptr),
                                                         C.byref(info)))
        self.last_eval_info = {"value": info.value, "C_global": info.C_global, "threshold": info.threshold,
                               "n_pairs": info.n_pairs, "device_ms": info.device_ms}
        return self.last_eval_info

    def set_state(self, global_functional: float, C_global: float):
        self._check(self._L.sdot_set_state(self._h, float(global_functional), float(C_global)))

    # ------------------------------------------------------------ measurement
    @property
    def stream_handle(self) -> int:
        return int(self._L.sdot_get_stream(self._h) or 0)

    def set_profiling(self, enable: bool = True):
        self._check(self._L.sdot_set_profiling(self._h, int(enable)))

    PHASES = ("threshold", "target_prep", "value_sweep", "gradient_sweep", "finalize", "layout", "pair_lists")

    def kernel_times(self, reset: bool = False) -> dict:
        """Device ms and launches per phase.  Truncated path: value_sweep is the
        fused kernel (both exponential sweeps), gradient_sweep the partial
        reduction, pair_lists the block-pair list build."""
        ms = np.zeros(7)
        ln = np.zeros(7, dtype=np.int64)
        self._check(self._L.sdot_get_kernel_times(self._h, ms.ctypes.data, ln.ctypes.data, 7, int(reset)))
        return {k: {"ms": float(ms[i]), "launches": int(ln[i])} for i, k in enumerate(self.PHASES)}

    # ---------------------------------------------------------------- getters
    def get_last_functional_value(self) -> float:
        return self._L.sdot_get_last_functional_value(self._h)

    def get_last_iteration_count(self) -> int:
        return self._L.sdot_get_last_iteration_count(self._h)

    def get_convergence_status(self) -> bool:
        return bool(self._L.sdot_get_convergence_status(self._h))

    def get_last_distance_threshold(self) -> float:
        return self._L.sdot_get_last_distance_threshold(self._h)

    def get_C_global(self) -> float:
        return self._L.sdot_get_C_global(self._h)

    def set_distance_threshold(self, threshold: float):
        self._check(self._L.sdot_set_distance_threshold(self._h, float(threshold)))

    def compute_covering_radius(self) -> float:
        r = C.c_double(0.0)
        self._check(self._L.sdot_compute_covering_radius(self._h, C.byref(r)))
        return r.value

    @staticmethod
    def measure_peaks(device: int = 0) -> dict:
        """Own microbenchmarks: FP64/FP32 FMA TFLOP/s, MUFU ex2 Gop/s, SM clock."""
        L = _lib.load()
        out = np.zeros(4)
        st = L.sdot_measure_peaks(int(device), out.ctypes.data)
        if st != _lib.SDOT_OK:
            raise _lib.SdotError(st, "sdot_measure_peaks failed")
        return {"fp64_tflops": float(out[0]), "fp32_tflops": float(out[1]), "ex2_gops": float(out[2]),
                "sm_clock_mhz": float(out[3])}

    def compute_geometric_radius_bound(self, potentials, epsilon: float, tolerance: float) -> float:
        psi = _f64(potentials)
        r = C.c_double(0.0)
        self._check(self._L.sdot_compute_geometric_radius_bound(self._h, psi.ctypes.data, float(epsilon),
                                                                float(tolerance), C.byref(r)))
        return r.value
