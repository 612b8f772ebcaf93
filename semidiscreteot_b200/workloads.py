"""Seeded synthetic workloads with the shapes of the benchmark configurations.

The reference publishes no dataset for this path; these generators stand in
for it with the stated sizes and distributions:

  dense_2d    : [0,1]^2, 64x64 Q1 cells, QGauss(3) (36,864 points), uniform
                density; N = 1,000 uniform targets, nu = 1/N; eps = 1e-2,
                no truncation (tau = 0), log-sum-exp on.
  trunc_3d    : [0,1]^3, 64^3 hex cells, QGauss(2) (2,097,152 points), density a
                4-component isotropic Gaussian mixture (sigma in [0.05, 0.2]),
                Q1-interpolated and renormalised on the mesh; N = 100,000
                targets from a 6-component mixture clipped to the cube,
                nu ~ Dirichlet(1); eps = 1e-3, tau = 1e-12.
  newton_3d   : [0,1]^3, 32^3 hex cells, QGauss(2) (262,144 points), uniform
                density; N = 20,000 uniform targets, nu = 1/N; eps = 5e-3.

  batched_2d  : n problems (256 at full size): square meshes of side
                log-uniform in [16, 128] cells, QGauss(3), density a sum of
                random Gaussian bumps, renormalised on the mesh; N log-uniform
                in [256, 16,384] uniform targets, nu ~ Dirichlet(1); eps drawn
                from {1e-1, 1e-2, 1e-3}; gradient tolerance 1e-8 (linf).

``scale`` shrinks the mesh (cells per axis) and the target count for tests.
"""
from __future__ import annotations

import numpy as np

from .parameters import SolverParameters
from .source import structured_source


def _mixture_pdf(pts, means, sigmas, weights):
    d = pts.shape[1]
    out = np.zeros(pts.shape[0])
    for m, s, w in zip(means, sigmas, weights):
        r2 = np.sum((pts - m) ** 2, axis=1)
        out += w * np.exp(-0.5 * r2 / s ** 2) / ((2 * np.pi) ** (d / 2) * s ** d)
    return out


def dense_2d(seed: int = 0, n_cells: int = 64, n_targets: int = 1000, order: int = 3):
    rng = np.random.default_rng(seed)
    src = structured_source(2, n_cells, order)
    y = rng.random((n_targets, 2))
    nu = np.full(n_targets, 1.0 / n_targets)
    prm = SolverParameters(epsilon=1e-2, tau=0.0, use_log_sum_exp_trick=True, tolerance=1e-8,
                           solver_control_type="linf", max_iterations=10000, verbose_output=False)
    return {"name": "dense_2d", "source": src, "y": y, "nu": nu, "params": prm, "dim": 2}


def trunc_3d(seed: int = 0, n_cells: int = 64, n_targets: int = 100_000, order: int = 2,
             epsilon: float = 1e-3, tau: float = 1e-12):
    rng = np.random.default_rng(seed)
    means = rng.uniform(0.2, 0.8, size=(4, 3))
    sigmas = rng.uniform(0.05, 0.2, size=4)
    weights = rng.dirichlet(np.ones(4))
    src = structured_source(3, n_cells, order, nodal_density=lambda p: _mixture_pdf(p, means, sigmas, weights))
    tm = rng.uniform(0.1, 0.9, size=(6, 3))
    ts = rng.uniform(0.05, 0.2, size=6)
    tw = rng.dirichlet(np.ones(6))
    comp = rng.choice(6, size=n_targets, p=tw)
    y = np.clip(tm[comp] + rng.standard_normal((n_targets, 3)) * ts[comp, None], 0.0, 1.0)
    nu = rng.dirichlet(np.ones(n_targets))
    prm = SolverParameters(epsilon=epsilon, tau=tau, use_log_sum_exp_trick=True, tolerance=1e-8,
                           solver_control_type="linf", max_iterations=10000, verbose_output=False)
    return {"name": "trunc_3d", "source": src, "y": y, "nu": nu, "params": prm, "dim": 3}


def newton_3d(seed: int = 0, n_cells: int = 32, n_targets: int = 20_000, order: int = 2):
    rng = np.random.default_rng(seed)
    src = structured_source(3, n_cells, order)
    y = rng.random((n_targets, 3))
    nu = np.full(n_targets, 1.0 / n_targets)
    prm = SolverParameters(epsilon=5e-3, tau=0.0, use_log_sum_exp_trick=True, tolerance=1e-8,
                           solver_control_type="linf", max_iterations=10000, verbose_output=False)
    return {"name": "newton_3d", "source": src, "y": y, "nu": nu, "params": prm, "dim": 3}


def batched_2d(seed: int = 0, n_problems: int = 256, side_range=(16, 128), target_range=(256, 16_384),
               eps_choices=(1e-1, 1e-2, 1e-3), order: int = 3, tolerance: float = 1e-8):
    """Problems of the batched configuration: list of dicts with source, y, nu, params."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_problems):
        side = int(round(np.exp(rng.uniform(np.log(side_range[0]), np.log(side_range[1])))))
        nt = int(round(np.exp(rng.uniform(np.log(target_range[0]), np.log(target_range[1])))))
        nb = int(rng.integers(1, 5))
        means = rng.uniform(0.15, 0.85, size=(nb, 2))
        sig = rng.uniform(0.08, 0.3, size=nb)
        amp = rng.uniform(0.5, 2.0, size=nb)

        def dens(p, means=means, sig=sig, amp=amp):
            out_ = np.full(p.shape[0], 0.05)
            for m, s_, a in zip(means, sig, amp):
                out_ += a * np.exp(-0.5 * np.sum((p - m) ** 2, axis=1) / s_ ** 2)
            return out_

        src = structured_source(2, side, order, nodal_density=dens)
        y = rng.random((nt, 2))
        nu = rng.dirichlet(np.ones(nt))
        eps = float(eps_choices[int(rng.integers(0, len(eps_choices)))])
        prm = SolverParameters(epsilon=eps, tau=0.0, use_log_sum_exp_trick=True, tolerance=tolerance,
                               solver_control_type="linf", max_iterations=20000, verbose_output=False)
        out.append({"source": src, "y": y, "nu": nu, "params": prm, "side": side})
    return out


WORKLOADS = {"dense_2d": dense_2d, "trunc_3d": trunc_3d, "newton_3d": newton_3d}
