"""Lloyd iterations with regularised semi-discrete OT.

Mirrors Lloyd::run_lloyd (src/core/Lloyd.cc:14-61) on a ``SotSolver`` whose
source is set:
- each iteration solves from zero potentials (``potential.reinit``,
  run_sot_iteration :180-283), over the epsilon-scaling sequence when the
  parameters ask for it, else at params.epsilon;
- the targets then move to the weighted barycenters of their cells
  (run_centroid_iteration :83-178).  The reference evaluates them once per
  epsilon of the sequence but always at the last solve's epsilon (the
  solver's current parameters), so one evaluation gives the same points;
- the step norm is the RMS distance between successive barycenters
  (compute_step_norm :64-81); the loop stops once it is below
  ``absolute_threshold`` and otherwise re-targets the solver at the new points
  with the same densities.
``output_dir`` receives barycenters_<n>.ply as the reference writes them.
A solve or barycenter evaluation that fails (a line-search failure) is
recorded and the loop goes on, as the reference catches std::exception there
(:273-276, :143-145): the potentials keep the last iterate, which the solver
writes back in place.
"""
from __future__ import annotations

import dataclasses
import os
from typing import List, Optional

import numpy as np

from ._lib import SdotError
from .io import write_ply
from .parameters import SolverParameters, epsilon_sequence


def step_norm(b_next: np.ndarray, b_prev: np.ndarray) -> float:
    d = np.asarray(b_next, dtype=np.float64) - np.asarray(b_prev, dtype=np.float64)
    return float(np.sqrt(np.sum(d * d) / d.shape[0]))


def run_lloyd(solver, target_points, target_density, params: SolverParameters, absolute_threshold: float = 1e-8,
              max_iterations: int = 100, output_dir: Optional[str] = None, method: str = "lbfgs") -> dict:
    """Returns the final barycenters, the potentials of the last solve, the
    step norms and the number of iterations run."""
    y = np.array(target_points, dtype=np.float64).reshape(-1, solver.dim)
    nu = np.ascontiguousarray(target_density, dtype=np.float64)
    solver.setup_target(y, nu)
    bary = y.copy()
    prev = y.copy()
    norms: List[float] = []
    eps_list = (epsilon_sequence(params.epsilon, params.epsilon_scaling_factor, params.epsilon_scaling_steps)
                if params.use_epsilon_scaling else [params.epsilon])
    psi = np.zeros(y.shape[0])
    failures: List[tuple] = []
    it = 0
    for it in range(max_iterations):
        psi = np.zeros(y.shape[0])
        for eps in eps_list:
            p = dataclasses.replace(params, epsilon=float(eps))
            try:
                if method == "newton":
                    solver.solve_newton(psi, p)
                else:
                    solver.solve(psi, p)
            except SdotError as e:
                failures.append((it, float(eps), str(e)))
        try:
            bary = solver.evaluate_weighted_barycenters(psi)
        except SdotError as e:
            failures.append((it, None, str(e)))
        if output_dir is not None:
            write_ply(bary, os.path.join(output_dir, f"barycenters_{it}.ply"))
        norms.append(step_norm(bary, prev))
        prev = bary.copy()
        if norms[-1] < absolute_threshold:
            break
        solver.setup_target(bary, nu)
    return {"barycenters": bary, "potentials": psi, "step_norms": norms, "iterations": it + 1,
            "failures": failures}
