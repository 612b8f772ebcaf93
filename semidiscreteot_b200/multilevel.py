"""Target-multilevel solves: coarse-to-fine with potential transfer.

Mirrors SemiDiscreteOT::run_target_multilevel (src/core/SemiDiscreteOT.cc
:966-1323) on a ``SotSolver``:
- the levels run from the coarsest to the finest (level 0);
- each level's potentials start from the coarser level's solution, through
  ``SotSolver.softmax_refinement`` at the last solve's distance threshold
  (``use_softmax_potential_transfer``, SemiDiscreteOT.cc:768-801), or by giving
  every child its parent's potential (:803-823);
- each level then solves over its epsilon values (an epsilon distribution as
  EpsilonScalingHandler::compute_epsilon_distribution gives, or the
  parameters' epsilon).

``run_source_multilevel`` mirrors SemiDiscreteOT::run_source_multilevel
(SemiDiscreteOT.cc:1325-1522): the same targets are solved against a list of
source measures, coarsest first; each level starts from the previous level's
potentials (the first from ``initial_potential`` or zero) and runs its share
of the epsilon-scaling sequence (EpsilonScalingHandler distribution over the
source levels), or params.epsilon when there is none.  The levels are given as
flattened sources (``setup_source`` dicts); ``nearest_vertex_density`` moves a
nodal density to a coarser mesh's vertices.

``run_combined_multilevel`` mirrors SemiDiscreteOT::run_combined_multilevel
(SemiDiscreteOT.cc:1524-1766): max(source levels, target levels) combined
levels, coarsest first; the hierarchy with more levels advances every level,
the other starts once the remaining depths line up (both reach their finest
level together).  When the target level moves one level finer, the potentials
are transferred (softmax or parent copy, as in the target multilevel driver)
before the solver is re-targeted; when it does not change they are kept.

``build_hierarchy`` is a seeded k-means coarsening (k-means++ seeds, Lloyd
iterations) with the level sizes of PointCloudHierarchyManager::getPointsForLevel
(src/core/PointCloudHierarchy.cc:63-76): level 1 holds min(N, max_points) points,
each further level a quarter of it, at least min_points.  Its clusters are
not the reference's; load the reference's own files with ``io.load_hierarchy``.
"""
from __future__ import annotations

import dataclasses
from typing import Dict, List, Optional, Sequence

import numpy as np

from .io import child_csr_from_parents
from .parameters import SolverParameters


def points_for_level(base_points: int, level: int, min_points: int, max_points: int) -> int:
    if level == 0:
        return base_points
    l1 = min(base_points, max_points)
    if level == 1:
        return l1
    return max(int(l1 / 4.0 ** (level - 1)), min_points)


def _kmeans(pts: np.ndarray, w: np.ndarray, k: int, rng, iters: int = 20):
    n = pts.shape[0]
    k = min(k, n)
    centres = [pts[rng.integers(n)]]
    d2 = np.sum((pts - centres[0]) ** 2, axis=1)
    for _ in range(1, k):
        p = d2 / d2.sum() if d2.sum() > 0 else None
        c = pts[rng.choice(n, p=p)]
        centres.append(c)
        d2 = np.minimum(d2, np.sum((pts - c) ** 2, axis=1))
    C = np.array(centres)
    for _ in range(iters):
        a = np.argmin(((pts[:, None, :] - C[None, :, :]) ** 2).sum(-1), axis=1) if n * k <= 4_000_000 else \
            np.array([np.argmin(np.sum((C - x) ** 2, axis=1)) for x in pts])
        for j in range(k):
            m = a == j
            if m.any():
                C[j] = np.average(pts[m], axis=0, weights=w[m])
    a = np.argmin(((pts[:, None, :] - C[None, :, :]) ** 2).sum(-1), axis=1) if n * k <= 4_000_000 else \
        np.array([np.argmin(np.sum((C - x) ** 2, axis=1)) for x in pts])
    used = np.unique(a)
    remap = -np.ones(k, dtype=np.int64)
    remap[used] = np.arange(used.size)
    a = remap[a]
    C = C[used]
    dens = np.bincount(a, weights=w, minlength=used.size)
    return C, dens, a


def build_hierarchy(points, densities=None, min_points: int = 100, max_points: int = 1000, seed: int = 0,
                    num_levels: Optional[int] = None) -> Dict[str, list]:
    """Levels (0 = the input) with points, densities and children CSR (children
    of a level-L point are level L-1 indices), like ``io.load_hierarchy``."""
    P = np.asarray(points, dtype=np.float64)
    w = np.full(P.shape[0], 1.0 / P.shape[0]) if densities is None else np.asarray(densities, dtype=np.float64)
    n = P.shape[0]
    l1 = min(n, max_points)
    if num_levels is None:
        num_levels = min(5, int(np.log(l1 / min_points) / np.log(4.0)) + 2) if l1 > min_points else 1
    rng = np.random.default_rng(seed)
    pts, dens, ch = [P], [w], []
    for L in range(1, num_levels):
        k = points_for_level(n, L, min_points, max_points)
        C, d, a = _kmeans(pts[-1], dens[-1], k, rng)
        ch.append(child_csr_from_parents(a, C.shape[0]))
        pts.append(C)
        dens.append(d)
    return {"points": pts, "densities": dens, "children": ch}


def run_target_multilevel(solver, hierarchy: Dict[str, list], params: SolverParameters,
                          use_softmax: bool = True, epsilon_distribution: Optional[Sequence[Sequence[float]]] = None,
                          initial_potential: Optional[np.ndarray] = None, method: str = "lbfgs") -> List[dict]:
    """Solves every level, coarsest first; returns per level (coarsest first)
    its level number, potentials, iterations and the threshold of its last solve.

    epsilon_distribution[i]: the epsilon values of the i-th level solved
    (coarsest first), e.g. ``distribute_epsilon_values``; default: params.epsilon."""
    pts, dens, ch = hierarchy["points"], hierarchy["densities"], hierarchy["children"]
    nl = len(pts)
    out: List[dict] = []
    psi = None
    for i, L in enumerate(range(nl - 1, -1, -1)):
        if i == 0:
            solver.setup_target(pts[L], dens[L])
            psi = np.zeros(len(dens[L])) if initial_potential is None else np.array(initial_potential, dtype=np.float64)
            if psi.size != len(dens[L]):
                raise ValueError("initial potential does not match the coarsest level")
        else:
            off, idx = ch[L]  # children (level L) of the level L+1 points now set as targets
            if use_softmax:
                psi = solver.softmax_refinement(psi, params.epsilon, solver.get_last_distance_threshold(), pts[L],
                                                off, idx, use_log_sum_exp=params.use_log_sum_exp_trick)
            else:
                fine = np.zeros(len(dens[L]))
                for j in range(len(off) - 1):
                    fine[idx[off[j]:off[j + 1]]] = psi[j]
                psi = fine
            solver.setup_target(pts[L], dens[L])
        eps_list = list(epsilon_distribution[i]) if epsilon_distribution is not None else [params.epsilon]
        its = 0
        for eps in eps_list:
            p = dataclasses.replace(params, epsilon=float(eps))
            if method == "newton":
                psi = solver.solve_newton(psi, p)
            else:
                psi = solver.solve(psi, p)
            its += solver.get_last_iteration_count()
        out.append({"level": L, "potentials": psi.copy(), "iterations": its,
                    "converged": bool(solver.get_convergence_status()),
                    "threshold": solver.get_last_distance_threshold()})
    return out


def nearest_vertex_density(fine_vertices, fine_density, coarse_vertices) -> np.ndarray:
    """Nodal density on a coarse mesh: each coarse vertex takes the value of the
    nearest fine vertex (a nearest-neighbour transfer in the spirit of
    Utils::interpolate_non_conforming_nearest, utils.h:504-600; ties go to the
    lowest fine index)."""
    F = np.asarray(fine_vertices, dtype=np.float64)
    d = np.asarray(fine_density, dtype=np.float64)
    Cv = np.asarray(coarse_vertices, dtype=np.float64)
    out = np.empty(Cv.shape[0])
    for k0 in range(0, Cv.shape[0], 2048):
        blk = Cv[k0:k0 + 2048]
        d2 = ((blk[:, None, :] - F[None, :, :]) ** 2).sum(-1) if F.shape[0] * blk.shape[0] <= 2 ** 26 else None
        if d2 is None:
            idx = np.array([int(np.argmin(np.sum((F - x) ** 2, axis=1))) for x in blk])
        else:
            idx = np.argmin(d2, axis=1)
        out[k0:k0 + blk.shape[0]] = d[idx]
    return out


def run_source_multilevel(solver, sources: Sequence[dict], target_points, target_density, params: SolverParameters,
                          epsilon_distribution: Optional[Sequence[Sequence[float]]] = None,
                          initial_potential: Optional[np.ndarray] = None, method: str = "lbfgs") -> List[dict]:
    """sources: flattened source measures, coarsest first.  Returns per level
    (coarsest first) its index, potentials, iterations, convergence and last
    threshold; the last entry holds the finest level's potentials."""
    y = np.asarray(target_points, dtype=np.float64)
    nu = np.asarray(target_density, dtype=np.float64)
    psi = np.zeros(len(nu)) if initial_potential is None else np.array(initial_potential, dtype=np.float64)
    if psi.size != len(nu):
        raise ValueError("initial potential does not match the target points")
    out: List[dict] = []
    for i, src in enumerate(sources):
        solver.setup_source(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"])
        solver.setup_target(y, nu)
        eps_list = list(epsilon_distribution[i]) if epsilon_distribution is not None and \
            i < len(epsilon_distribution) and len(epsilon_distribution[i]) else [params.epsilon]
        its = 0
        for eps in eps_list:
            p = dataclasses.replace(params, epsilon=float(eps))
            if method == "newton":
                psi = solver.solve_newton(psi, p)
            else:
                psi = solver.solve(psi, p)
            its += solver.get_last_iteration_count()
        out.append({"level": len(sources) - 1 - i, "potentials": psi.copy(), "iterations": its,
                    "converged": bool(solver.get_convergence_status()),
                    "threshold": solver.get_last_distance_threshold()})
    return out


def combined_level_indices(n_source: int, n_target: int):
    """(source index, target index) per combined level, coarsest first, indices
    counted from the coarsest level of each hierarchy (SemiDiscreteOT.cc:1598-1607)."""
    out = []
    for i in range(max(n_source, n_target)):
        if n_source >= n_target:
            out.append((i, i - (n_source - n_target) if i >= n_source - n_target else 0))
        else:
            out.append((i - (n_target - n_source) if i >= n_target - n_source else 0, i))
    return out


def run_combined_multilevel(solver, sources: Sequence[dict], hierarchy: Dict[str, list], params: SolverParameters,
                            use_softmax: bool = True,
                            epsilon_distribution: Optional[Sequence[Sequence[float]]] = None,
                            initial_potential: Optional[np.ndarray] = None, method: str = "lbfgs") -> List[dict]:
    """sources: flattened source measures, coarsest first; hierarchy: target
    levels as from build_hierarchy / io.load_hierarchy (level 0 finest).
    Returns per combined level its source and target levels, potentials,
    iterations, convergence and last threshold."""
    pts, dens, ch = hierarchy["points"], hierarchy["densities"], hierarchy["children"]
    nt_levels = len(pts)
    out: List[dict] = []
    psi = None
    prev_tl = None
    for i, (si, ti) in enumerate(combined_level_indices(len(sources), nt_levels)):
        tl = nt_levels - 1 - ti                       # actual target level (0 = finest)
        if i == 0:
            psi = np.zeros(len(dens[tl])) if initial_potential is None else np.array(initial_potential, dtype=np.float64)
            if psi.size != len(dens[tl]):
                raise ValueError("initial potential does not match the coarsest target level")
        elif tl != prev_tl:
            if prev_tl != tl + 1:
                raise ValueError("target levels must advance one at a time")
            off, idx = ch[tl]                         # children (level tl) of the level tl+1 points
            if use_softmax:
                psi = solver.softmax_refinement(psi, params.epsilon, solver.get_last_distance_threshold(), pts[tl],
                                                off, idx, use_log_sum_exp=params.use_log_sum_exp_trick)
            else:
                fine = np.zeros(len(dens[tl]))
                for j in range(len(off) - 1):
                    fine[idx[off[j]:off[j + 1]]] = psi[j]
                psi = fine
        src = sources[si]
        solver.setup_source(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"])
        solver.setup_target(pts[tl], dens[tl])
        eps_list = list(epsilon_distribution[i]) if epsilon_distribution is not None and \
            i < len(epsilon_distribution) and len(epsilon_distribution[i]) else [params.epsilon]
        its = 0
        for eps in eps_list:
            p = dataclasses.replace(params, epsilon=float(eps))
            psi = solver.solve_newton(psi, p) if method == "newton" else solver.solve(psi, p)
            its += solver.get_last_iteration_count()
        out.append({"source_level": len(sources) - 1 - si, "target_level": tl, "potentials": psi.copy(),
                    "iterations": its, "converged": bool(solver.get_convergence_status()),
                    "threshold": solver.get_last_distance_threshold()})
        prev_tl = tl
    return out
