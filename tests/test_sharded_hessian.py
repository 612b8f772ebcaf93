"""The tensor-core Hessian computed by tile ranges (sdot_hessian_tiles_device),
the way GPUs share it in a sharded Newton solve, on one GPU.

Every entry of the upper triangle lies in exactly one 128 x 256 tile and a
tile's arithmetic does not depend on which launch computes it, so the
matrices of disjoint tile ranges, each written into a zeroed buffer, add up to
the full tensor-core Hessian exactly.  The sharded Newton driver
(ShardedHessianNewton, here with one rank) converges to solve_newton's
potential.
"""
import numpy as np
import pytest
import torch

from semidiscreteot_b200 import SolverParameters, SotSolver, structured_source
from semidiscreteot_b200.distributed import ShardedHessianNewton, hessian_tiles, tile_range

pytestmark = pytest.mark.gpu


def _solver():
    rng = np.random.default_rng(17)
    src = structured_source(2, 24, 3, nodal_density=lambda p: 0.5 + np.exp(-np.sum((p - 0.4) ** 2, axis=1) / 0.1))
    n = 700                                   # 12 tiles
    y = rng.random((n, 2))
    nu = rng.dirichlet(np.ones(n) * 4)
    prm = SolverParameters(epsilon=2e-2, tau=0.0, use_log_sum_exp_trick=True, tolerance=1e-9,
                           solver_control_type="linf", max_iterations=200)
    s = SotSolver(dim=2, device=0, precision="fp64")
    s.setup_source(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"])
    s.setup_target(y, nu)
    s.configure(prm)
    return s, n, prm, rng


def test_tile_ranges_sum_to_the_full_hessian():
    s, n, prm, rng = _solver()
    assert s.hessian_tile_count() == len(hessian_tiles(n)) == 12
    psi = torch.tensor(0.3 * prm.epsilon * rng.standard_normal(n), dtype=torch.float64, device="cuda")
    full = torch.empty(n * n, dtype=torch.float32, device="cuda")
    s.compute_hessian_device(psi.data_ptr(), full.data_ptr(), method="tensor", out_f32=True)
    for world in (2, 3):
        total = torch.zeros(n * n, dtype=torch.float32, device="cuda")
        for r in range(world):
            part = torch.zeros(n * n, dtype=torch.float32, device="cuda")
            t0, t1 = tile_range(12, r, world)
            info = s.compute_hessian_tiles_device(psi.data_ptr(), part.data_ptr(), t0, t1)
            assert info["tiles"] == t1 - t0
            total += part
        assert torch.equal(total, full), world
    with pytest.raises(RuntimeError):
        s.compute_hessian_tiles_device(psi.data_ptr(), full.data_ptr(), 5, 13)
    # the library's matvec of a share: its part of H x
    x = torch.tensor(rng.standard_normal(n), dtype=torch.float64, device="cuda")
    y = torch.empty(n, dtype=torch.float64, device="cuda")
    s.hessian_matvec_device(full.data_ptr(), x.data_ptr(), y.data_ptr(), f32=True)
    ref = full.view(n, n).double() @ x
    assert torch.max(torch.abs(y - ref)).item() <= 1e-12 * torch.max(torch.abs(ref)).item()
    s.close()


def test_sharded_newton_one_rank_matches_solve_newton():
    s, n, prm, _ = _solver()
    sh = ShardedHessianNewton(s, rank=0, world=1)
    psi, info = sh.solve(np.zeros(n), prm)
    assert info["converged"] and info["n_hessians"] >= 1
    g = np.zeros(n)
    s.evaluate_functional(psi, g)
    assert np.max(np.abs(g)) <= 1e-9
    ref = s.solve_newton(np.zeros(n), prm)
    assert s.get_convergence_status()
    d = (psi - psi.mean()) - (ref - ref.mean())
    assert np.max(np.abs(d)) <= 1e-7
    s.close()
