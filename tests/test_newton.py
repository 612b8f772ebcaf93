"""Newton solve (tensor-core Hessian + PCG + Armijo) against the L-BFGS solve and the oracle.

Both solvers stop at the same control (linf gradient <= tol); the potentials
they reach must agree up to the constant shift (J is shift invariant) within
the error that a gradient of size tol allows, and the gradient the oracle
computes at Newton's potential must meet the tolerance too.
"""
import numpy as np
import pytest

from semidiscreteot_b200 import SolverParameters, SotSolver, structured_source

pytestmark = pytest.mark.gpu


def problem(kind, seed=0):
    rng = np.random.default_rng(seed)
    if kind == "dense2d":
        src = structured_source(2, 16, 3)
        N, eps = 400, 2e-2
        y = rng.random((N, 2))
        nu = np.full(N, 1.0 / N)
    elif kind == "dense3d":
        src = structured_source(3, 10, 2)
        N, eps = 700, 1e-2
        y = rng.random((N, 3))
        nu = rng.dirichlet(np.ones(N) * 4)
    else:
        raise KeyError(kind)
    return src, y, nu, eps


def make(src, y, nu, precision="fp64"):
    s = SotSolver(dim=y.shape[1], device=0, precision=precision)
    s.setup_source(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"])
    s.setup_target(y, nu)
    return s


@pytest.mark.parametrize("kind", ["dense2d", "dense3d"])
def test_newton_matches_lbfgs_and_oracle(oracle_mod, kind):
    src, y, nu, eps = problem(kind)
    N = len(nu)
    prm = SolverParameters(epsilon=eps, tau=0.0, use_log_sum_exp_trick=True, tolerance=1e-9,
                           solver_control_type="linf", max_iterations=5000)
    s = make(src, y, nu)
    psi_n = s.solve_newton(np.zeros(N), prm, hessian="tensor")
    info = s.last_solve_info
    assert s.get_convergence_status() and info["converged"], info
    assert info["hessian_method"] == "tensor"
    assert info["iterations"] <= 30, info
    g = np.zeros(N)
    s.evaluate_functional(psi_n, g)
    assert np.max(np.abs(g)) <= 1e-9
    psi_l = s.solve(np.zeros(N), prm)
    assert s.get_convergence_status()
    d = (psi_n - psi_n.mean()) - (psi_l - psi_l.mean())
    print(f"{kind}: Newton {info['iterations']} its ({info['cg_iterations']} CG), "
          f"L-BFGS {s.get_last_iteration_count()} its, |dpsi| {np.max(np.abs(d)):.2e}")
    assert np.max(np.abs(d)) <= 1e-5
    # the oracle's gradient at Newton's potential
    P = oracle_mod.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"], y, nu)
    op = oracle_mod.Params(epsilon=eps, tau=0.0, use_log_sum_exp=True)
    _, go, _ = P.evaluate(psi_n, op)
    assert np.max(np.abs(go)) <= 1.5e-9
    s.close()


def test_newton_fp64_hessian_and_truncated_fallback():
    src, y, nu, eps = problem("dense2d", seed=2)
    N = len(nu)
    prm = SolverParameters(epsilon=eps, tau=0.0, use_log_sum_exp_trick=True, tolerance=1e-9,
                           solver_control_type="linf", max_iterations=100)
    s = make(src, y, nu)
    psi_t = s.solve_newton(np.zeros(N), prm, hessian="tensor")
    psi_f = s.solve_newton(np.zeros(N), prm, hessian="fp64")
    assert s.last_solve_info["hessian_method"] == "fp64" and s.get_convergence_status()
    d = (psi_t - psi_t.mean()) - (psi_f - psi_f.mean())
    assert np.max(np.abs(d)) <= 1e-6
    # truncated problem: "auto" falls back to the FP64 Hessian, "tensor" is refused
    prm_t = SolverParameters(epsilon=5e-3, tau=1e-10, use_log_sum_exp_trick=True, tolerance=1e-8,
                             solver_control_type="linf", max_iterations=200)
    psi_a = s.solve_newton(np.zeros(N), prm_t, hessian="auto")
    assert s.get_convergence_status() and s.last_solve_info["hessian_method"] == "fp64"
    g = np.zeros(N)
    s.evaluate_functional(psi_a, g)
    assert np.max(np.abs(g)) <= 1e-8
    with pytest.raises(RuntimeError, match="untruncated"):
        s.solve_newton(np.zeros(N), prm_t, hessian="tensor")
    s.close()


def test_newton_nonconvergence_is_reported_not_raised():
    src, y, nu, eps = problem("dense2d", seed=4)
    prm = SolverParameters(epsilon=eps, tau=0.0, use_log_sum_exp_trick=True, tolerance=1e-14,
                           solver_control_type="linf", max_iterations=2)
    s = make(src, y, nu)
    s.solve_newton(np.zeros(len(nu)), prm)
    assert not s.get_convergence_status()
    assert s.get_last_iteration_count() == 2
    s.close()
