"""ctypes front end of the FP64 CPU oracle (``oracle/sdot_oracle.c``).

TEST INFRASTRUCTURE ONLY.  This module is the checker for the CUDA path: it
may be imported by ``tests/``, by ``__graft_entry__.smoke()`` and by the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``, never by the
product package ``semidiscreteot_b200``.

Parity status: unpinned.  The reference (SemiDiscreteOT, C++ on deal.II 9.5,
Boost.Geometry, MPI) cannot be built here and ships no golden vectors; the
restatement is validated by first-principles known-answer tests instead.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libsdot_oracle.so")

THRESH = {"pointwise": 0, "integral": 1, "geometric": 2}
CONTROL = {"l1norm": 0, "componentwise": 1, "linf": 2}
LINE_SEARCH = {"upstream": 0, "vendored": 1}
DISTANCE = {"euclidean": 0, "spherical": 1}


def build(force: bool = False) -> str:
    """Compile the oracle shared library with its Makefile (gcc, OpenMP)."""
    src = os.path.join(_HERE, "sdot_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class _Problem(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("n_q", C.c_int64), ("n_cells", C.c_int64), ("n_targets", C.c_int64),
        ("xq", C.c_void_p), ("jxw", C.c_void_p), ("rho", C.c_void_p),
        ("cell_offsets", C.c_void_p), ("cell_centers", C.c_void_p),
        ("y", C.c_void_p), ("nu", C.c_void_p), ("distance", C.c_int),
    ]


class _Params(C.Structure):
    _fields_ = [
        ("epsilon", C.c_double), ("tau", C.c_double), ("use_log_sum_exp", C.c_int),
        ("threshold_type", C.c_int), ("control_type", C.c_int), ("tolerance", C.c_double),
        ("max_iterations", C.c_uint), ("line_search_variant", C.c_int),
    ]


class _State(C.Structure):
    _fields_ = [
        ("global_functional", C.c_double), ("C_global", C.c_double),
        ("covering_radius", C.c_double), ("min_target_density", C.c_double),
        ("current_distance_threshold", C.c_double),
    ]


class _Stats(C.Structure):
    _fields_ = [("threshold", C.c_double), ("n_pairs", C.c_int64),
                ("n_active_cells", C.c_int64), ("n_skipped_q", C.c_int64)]


class _SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_uint), ("converged", C.c_int), ("status", C.c_int),
                ("n_evaluations", C.c_int64), ("last_value", C.c_double),
                ("last_check_value", C.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        d, i64, vp, ip = C.c_double, C.c_int64, C.c_void_p, C.c_int
        _lib.orc_gauss_legendre.argtypes = [ip, vp, vp]
        _lib.orc_structured_source.argtypes = [ip, ip, d, d, ip, vp, ip, vp, vp, vp, vp, vp]
        _lib.orc_structured_source.restype = i64
        _lib.orc_covering_radius.argtypes = [vp]
        _lib.orc_covering_radius.restype = d
        _lib.orc_distance_threshold.argtypes = [vp, vp, vp, vp]
        _lib.orc_distance_threshold.restype = d
        _lib.orc_integral_radius_bound.argtypes = [vp, vp, d, d, d, d]
        _lib.orc_integral_radius_bound.restype = d
        _lib.orc_geometric_radius_bound.argtypes = [vp, vp, vp, d, d]
        _lib.orc_geometric_radius_bound.restype = d
        _lib.orc_candidates.argtypes = [vp, vp, d, vp]
        _lib.orc_candidates.restype = i64
        _lib.orc_evaluate.argtypes = [vp, vp, vp, vp, vp, vp, ip, ip]
        _lib.orc_evaluate.restype = d
        _lib.orc_evaluate_cells.argtypes = [vp, vp, d, vp, i64, i64, vp, vp, vp, ip, ip]
        _lib.orc_evaluate_cells.restype = d
        _lib.orc_solve.argtypes = [vp, vp, vp, vp, vp, vp, i64, ip]
        _lib.orc_solve.restype = ip
        _lib.orc_solve_ex.argtypes = [vp, vp, vp, vp, vp, vp, i64, ip, ip]
        _lib.orc_solve_ex.restype = ip
        _lib.orc_hessian.argtypes = [vp, vp, d, vp, vp, ip]
        _lib.orc_softmax_refinement.argtypes = [vp, vp, d, d, ip, i64, vp, vp, vp, vp, ip]
        _lib.orc_weighted_barycenters.argtypes = [vp, vp, d, vp, vp, ip]
        _lib.orc_conditioned_densities.argtypes = [vp, vp, d, d, i64, vp, vp, i64, vp, vp]
        _lib.orc_spherical_barycenters.argtypes = [vp, vp, d, vp, vp, C.c_uint, d, vp]
        _lib.orc_spherical_barycenters.restype = ip
        _lib.orc_epsilon_sequence.argtypes = [d, d, C.c_uint, vp]
        _lib.orc_epsilon_sequence.restype = ip
    return _lib


def _p(a):
    return a.ctypes.data if a is not None else None


def gauss_legendre(n: int):
    x = np.zeros(n)
    w = np.zeros(n)
    lib().orc_gauss_legendre(n, _p(x), _p(w))
    return x, w


def structured_source(dim, n, lo=0.0, hi=1.0, order=2, nodal=None, normalize=True):
    """Oracle's own structured Q1 source flattening (x_q, JxW_q, rho_q, offsets, centres)."""
    ncell = n ** dim
    qpc = order ** dim
    Q = ncell * qpc
    xq = np.zeros((Q, dim))
    jxw = np.zeros(Q)
    rho = np.zeros(Q)
    off = np.zeros(ncell + 1, dtype=np.int64)
    ctr = np.zeros((ncell, dim))
    nod = None if nodal is None else np.ascontiguousarray(nodal, dtype=np.float64)
    got = lib().orc_structured_source(dim, n, lo, hi, order, _p(nod), int(normalize),
                                      _p(xq), _p(jxw), _p(rho), _p(off), _p(ctr))
    assert got == Q
    return xq, jxw, rho, off, ctr


@dataclass
class Params:
    epsilon: float = 1e-3
    tau: float = 1e-8
    use_log_sum_exp: bool = False
    distance_threshold_type: str = "pointwise"
    solver_control_type: str = "l1norm"
    tolerance: float = 1.0
    max_iterations: int = 1000
    line_search: str = "upstream"

    def c(self) -> _Params:
        return _Params(self.epsilon, self.tau, int(self.use_log_sum_exp),
                       THRESH[self.distance_threshold_type], CONTROL[self.solver_control_type],
                       self.tolerance, self.max_iterations, LINE_SEARCH[self.line_search])


class Problem:
    """Holds contiguous FP64 copies of a problem and the reference-like solver state."""

    def __init__(self, xq, jxw, rho, cell_offsets, cell_centers, y, nu, distance="euclidean"):
        self.xq = np.ascontiguousarray(xq, dtype=np.float64)
        self.dim = self.xq.shape[1]
        self.jxw = np.ascontiguousarray(jxw, dtype=np.float64)
        self.rho = np.ascontiguousarray(rho, dtype=np.float64)
        self.off = np.ascontiguousarray(cell_offsets, dtype=np.int64)
        self.ctr = np.ascontiguousarray(cell_centers, dtype=np.float64).reshape(-1, self.dim)
        self.y = np.ascontiguousarray(y, dtype=np.float64).reshape(-1, self.dim)
        self.nu = np.ascontiguousarray(nu, dtype=np.float64)
        self._c = _Problem(self.dim, self.xq.shape[0], self.ctr.shape[0], self.y.shape[0],
                           _p(self.xq), _p(self.jxw), _p(self.rho), _p(self.off), _p(self.ctr),
                           _p(self.y), _p(self.nu), DISTANCE[distance])
        self.state = _State(0.0, 0.0, 0.0, 0.0, 1e-1)

    @property
    def N(self):
        return self.y.shape[0]

    def reset_state(self):
        self.state = _State(0.0, 0.0, 0.0, 0.0, 1e-1)

    def covering_radius(self) -> float:
        return lib().orc_covering_radius(C.byref(self._c))

    def distance_threshold(self, psi, prm: Params) -> float:
        psi = np.ascontiguousarray(psi, dtype=np.float64)
        pc = prm.c()
        return lib().orc_distance_threshold(C.byref(self._c), C.byref(pc), C.byref(self.state), _p(psi))

    def geometric_radius_bound(self, psi, eps, tol) -> float:
        psi = np.ascontiguousarray(psi, dtype=np.float64)
        return lib().orc_geometric_radius_bound(C.byref(self._c), C.byref(self.state), _p(psi), eps, tol)

    def integral_radius_bound(self, psi, eps, tol, C_value, J_value) -> float:
        psi = np.ascontiguousarray(psi, dtype=np.float64)
        return lib().orc_integral_radius_bound(C.byref(self._c), _p(psi), eps, tol, C_value, J_value)

    def candidates(self, center, r):
        out = np.zeros(self.N + 1, dtype=np.int64)
        c = np.ascontiguousarray(center, dtype=np.float64)
        k = lib().orc_candidates(C.byref(self._c), _p(c), r, _p(out))
        return out[:k]

    def evaluate(self, psi, prm: Params, faithful=False, threads=0):
        """Returns (J, grad, stats dict) and updates the persistent state."""
        psi = np.ascontiguousarray(psi, dtype=np.float64)
        g = np.zeros(self.N)
        st = _Stats()
        pc = prm.c()
        J = lib().orc_evaluate(C.byref(self._c), C.byref(pc), C.byref(self.state), _p(psi),
                               _p(g), C.byref(st), int(faithful), threads)
        return J, g, {"threshold": st.threshold, "n_pairs": st.n_pairs,
                      "C_global": self.state.C_global}

    def evaluate_cells(self, psi, prm: Params, r, c0, c1, faithful=False, threads=0, grad=True):
        psi = np.ascontiguousarray(psi, dtype=np.float64)
        g = np.zeros(self.N) if grad else None
        Cv = C.c_double(0.0)
        npairs = C.c_int64(0)
        pc = prm.c()
        J = lib().orc_evaluate_cells(C.byref(self._c), C.byref(pc), r, _p(psi), c0, c1, _p(g),
                                     C.byref(Cv), C.byref(npairs), int(faithful), threads)
        return J, g, Cv.value, npairs.value

    def solve(self, psi0, prm: Params, threads=0, trace_cap=100000, faithful=False):
        psi = np.array(psi0, dtype=np.float64, copy=True)
        info = _SolveInfo()
        trace = np.zeros((trace_cap, 3))
        pc = prm.c()
        lib().orc_solve_ex(C.byref(self._c), C.byref(pc), C.byref(self.state), _p(psi),
                           C.byref(info), _p(trace), trace_cap, threads, int(bool(faithful)))
        n = info.iterations + 1
        return psi, {"iterations": info.iterations, "converged": bool(info.converged),
                     "status": info.status, "n_evaluations": info.n_evaluations,
                     "last_value": info.last_value, "last_check_value": info.last_check_value,
                     "trace": trace[: min(n, trace_cap)]}

    def hessian(self, psi, prm: Params, r, threads=0):
        psi = np.ascontiguousarray(psi, dtype=np.float64)
        H = np.zeros((self.N, self.N))
        pc = prm.c()
        lib().orc_hessian(C.byref(self._c), C.byref(pc), r, _p(psi), _p(H), threads)
        return H

    def softmax_refinement(self, psi_coarse, eps, r, use_lse, y_fine, child_offsets,
                           child_indices, threads=0):
        psi_coarse = np.ascontiguousarray(psi_coarse, dtype=np.float64)
        yf = np.ascontiguousarray(y_fine, dtype=np.float64).reshape(-1, self.dim)
        co = np.ascontiguousarray(child_offsets, dtype=np.int64)
        ci = np.ascontiguousarray(child_indices, dtype=np.int64)
        out = np.zeros(yf.shape[0])
        lib().orc_softmax_refinement(C.byref(self._c), _p(psi_coarse), eps, r, int(use_lse),
                                     yf.shape[0], _p(yf), _p(co), _p(ci), _p(out), threads)
        return out


    def weighted_barycenters(self, psi, prm: Params, r, threads=0):
        psi = np.ascontiguousarray(psi, dtype=np.float64)
        out = np.zeros((self.N, self.dim))
        pc = prm.c()
        lib().orc_weighted_barycenters(C.byref(self._c), C.byref(pc), r, _p(psi), _p(out), threads)
        return out

    def spherical_barycenters(self, psi, prm: Params, r, bary0, max_iterations, tolerance):
        """Spherical weighted-barycenter iteration; returns (barycenters, iterations, last gradient norm)."""
        psi = np.ascontiguousarray(psi, dtype=np.float64)
        b = np.array(bary0, dtype=np.float64, copy=True).reshape(self.N, self.dim)
        nrm = C.c_double(0.0)
        pc = prm.c()
        it = lib().orc_spherical_barycenters(C.byref(self._c), C.byref(pc), r, _p(psi), _p(b),
                                             int(max_iterations), float(tolerance), C.byref(nrm))
        return b, it, nrm.value

    def conditioned_densities(self, psi, eps, r, points, density, indices):
        psi = np.ascontiguousarray(psi, dtype=np.float64)
        P = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, self.dim)
        rho = np.ascontiguousarray(density, dtype=np.float64)
        idx = np.ascontiguousarray(indices, dtype=np.int64)
        out = np.zeros((idx.size, P.shape[0]))
        lib().orc_conditioned_densities(C.byref(self._c), _p(psi), eps, r, P.shape[0], _p(P), _p(rho),
                                        idx.size, _p(idx), _p(out))
        return out

def epsilon_sequence(eps, factor, steps):
    out = np.zeros(max(int(steps), 1))
    n = lib().orc_epsilon_sequence(eps, factor, int(steps), _p(out))
    return out[:n]
