"""Lloyd iterations (Lloyd::run_lloyd) on the device against the same loop on the oracle.

Each iteration solves from zero potentials to a 1e-9 gradient tolerance, so the
two loops' potentials agree to about 1e-7 and the barycenters to 1e-5
(absolute, unit square); within one loop the barycenters conserve the source's
first moment, sum_j nu_j B_j = sum_q w_q x_q, to 1e-10.
"""
import numpy as np
import pytest

from semidiscreteot_b200 import SolverParameters, SotSolver, run_lloyd, structured_source
from semidiscreteot_b200.io import read_ply

pytestmark = pytest.mark.gpu


def setup(rng):
    src = structured_source(2, 12, 3, nodal_density=lambda p: 0.5 + np.exp(-np.sum((p - 0.4) ** 2, axis=1) / 0.05))
    y = rng.random((30, 2))
    nu = np.full(30, 1.0 / 30)
    return src, y, nu


def test_lloyd_matches_oracle_loop(oracle_mod, tmp_path):
    rng = np.random.default_rng(8)
    src, y, nu = setup(rng)
    prm = SolverParameters(epsilon=2e-2, tau=0.0, tolerance=1e-9, solver_control_type="linf", max_iterations=3000)
    s = SotSolver(dim=2, device=0, precision="fp64")
    s.setup_source(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"])
    out = run_lloyd(s, y, nu, prm, absolute_threshold=0.0, max_iterations=3, output_dir=str(tmp_path))
    assert out["iterations"] == 3 and len(out["step_norms"]) == 3
    moment = (src["density"] * src["jxw"]) @ src["x"].reshape(-1, 2)
    np.testing.assert_allclose(nu @ out["barycenters"], moment, rtol=1e-10)
    op = oracle_mod.Params(epsilon=2e-2, tau=0.0, tolerance=1e-9, solver_control_type="linf", max_iterations=3000)
    yo = y.copy()
    norms = []
    for it in range(3):
        P = oracle_mod.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"], yo, nu)
        psi, info = P.solve(np.zeros(30), op)
        assert info["converged"]
        B = P.weighted_barycenters(psi, op, 1e300)
        norms.append(np.sqrt(np.sum((B - yo) ** 2) / 30))
        np.testing.assert_allclose(read_ply(str(tmp_path / f"barycenters_{it}.ply")), B, atol=2e-5)
        yo = B
    np.testing.assert_allclose(out["barycenters"], yo, atol=1e-5)
    np.testing.assert_allclose(out["step_norms"], norms, rtol=1e-4, atol=1e-7)
    s.close()


@pytest.mark.parametrize("method", ["lbfgs", "newton"])
def test_lloyd_converges(method):
    """Runs to a 1.5e-3 step norm with epsilon scaling (the oracle's loop gets
    there in about 20 iterations on this case and then slows to ~4e-5 by 400)."""
    rng = np.random.default_rng(9)
    src, y, nu = setup(rng)
    prm = SolverParameters(epsilon=1e-2, tau=0.0, tolerance=1e-8, solver_control_type="linf", max_iterations=3000,
                           use_epsilon_scaling=True, epsilon_scaling_factor=4.0, epsilon_scaling_steps=2)
    s = SotSolver(dim=2, device=0, precision="fp64")
    s.setup_source(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"])
    out = run_lloyd(s, y, nu, prm, absolute_threshold=1.5e-3, max_iterations=60, method=method)
    assert out["step_norms"][-1] < 1.5e-3 and out["iterations"] < 60
    g = np.zeros(30)
    s.evaluate_functional(out["potentials"], g)
    assert np.max(np.abs(g)) < 1e-6
    s.close()


def test_lloyd_goes_on_after_solver_failures():
    """At a 1e-9 tolerance the deal.II line search fails on many of these solves
    (the oracle's loop: 319 of 800).  Like the reference's driver, the loop
    records the failure and goes on from the last iterate."""
    rng = np.random.default_rng(9)
    src, y, nu = setup(rng)
    prm = SolverParameters(epsilon=1e-2, tau=0.0, tolerance=1e-9, solver_control_type="linf", max_iterations=3000,
                           use_epsilon_scaling=True, epsilon_scaling_factor=4.0, epsilon_scaling_steps=2)
    s = SotSolver(dim=2, device=0, precision="fp64")
    s.setup_source(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"])
    out = run_lloyd(s, y, nu, prm, absolute_threshold=0.0, max_iterations=8)
    assert out["iterations"] == 8 and len(out["step_norms"]) == 8
    assert all(f[2].startswith("SDOT_ELINESEARCH") for f in out["failures"])
    assert np.all(np.isfinite(out["barycenters"]))
    s.close()
