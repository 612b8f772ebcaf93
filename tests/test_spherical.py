"""The spherical distance (SotSolver::set_distance_function("spherical")).

CPU: the oracle's spherical restatement against first principles -- the
candidate predicate against a brute-force great-circle distance, mass
conservation sum_j (g_j + nu_j) = sum_q w_q, finite-difference gradients, and
the barycenter iteration on a cap symmetric about the pole (one target: the
pole is a fixed point; a point off the pole moves to the other side, the
step being twice the mean logarithm).
GPU: evaluations, an L-BFGS solve (to |g|_inf <= 1e-8, within 3 iterations
of the oracle's own solve) and the barycenter iteration through the C ABI
against the oracle (value 1e-10 relative, gradient 1e-12 absolute in FP64,
candidate pairs exact; barycenters 1e-10).
"""
import numpy as np
import pytest

from semidiscreteot_b200 import SolverParameters, SotSolver, sphere_source


def _targets(rng, n, cap=np.pi):
    t = np.arccos(1 - rng.random(n) * (1 - np.cos(cap)))
    p = 2 * np.pi * rng.random(n)
    return np.stack([np.sin(t) * np.cos(p), np.sin(t) * np.sin(p), np.cos(t)], axis=1)


def _problem(oracle_mod, seed=0, n_targets=60, cap=np.pi):
    rng = np.random.default_rng(seed)
    src = sphere_source(10, 20, 2, theta_max=cap, density=lambda x: 1.0 + 0.5 * x[:, 2])
    y = _targets(rng, n_targets, cap)
    nu = rng.dirichlet(np.ones(n_targets) * 4)
    P = oracle_mod.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"], y, nu,
                           distance="spherical")
    return src, y, nu, P


def _gc(a, b):
    c = np.clip(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)), -1, 1)
    return np.arccos(c)


def test_oracle_spherical_candidates_brute_force(oracle_mod):
    src, y, nu, P = _problem(oracle_mod)
    for c in src["cell_centers"][::17]:
        for r in (0.3, 0.9, 2.0):
            got = P.candidates(c, r)
            want = [j for j in range(len(nu)) if _gc(y[j], c) <= r]
            assert list(got) == want


def test_oracle_spherical_mass_and_fd(oracle_mod):
    src, y, nu, P = _problem(oracle_mod, seed=1)
    op = oracle_mod.Params(epsilon=0.05, tau=0.0, use_log_sum_exp=True)
    psi = 0.02 * np.random.default_rng(2).standard_normal(len(nu))
    J, g, st = P.evaluate(psi, op)
    assert abs(np.sum(g + nu) - np.sum(src["density"] * src["jxw"])) <= 1e-12
    h = 1e-6
    for j in (0, 7, 33):
        e = np.zeros(len(nu))
        e[j] = h
        Jp, _, _ = P.evaluate(psi + e, op)
        Jm, _, _ = P.evaluate(psi - e, op)
        assert abs((Jp - Jm) / (2 * h) - g[j]) <= 1e-7


def test_oracle_spherical_barycenter_symmetric_cap(oracle_mod):
    cap = 0.4
    src = sphere_source(8, 32, 3, theta_max=cap)
    y = np.array([[0.0, 0.0, 1.0]])
    nu = np.array([1.0])
    P = oracle_mod.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"], y, nu,
                           distance="spherical")
    op = oracle_mod.Params(epsilon=0.1, tau=0.0, use_log_sum_exp=True)
    b, it, nrm = P.spherical_barycenters(np.zeros(1), op, 1e300, y, 5, 1e-10)
    assert it == 1 and nrm < 1e-10 and np.allclose(b, y, atol=0)
    a = 0.01
    b0 = np.array([[np.sin(a), 0.0, np.cos(a)]])
    b1, it, nrm = P.spherical_barycenters(np.zeros(1), op, 1e300, b0, 1, 0.0)
    assert it == 1
    # one step: twice the mean logarithm, to first order the mirror image of b0
    ang = np.arctan2(b1[0, 0], b1[0, 2])
    assert abs(ang + a) <= 0.05 * a and abs(np.linalg.norm(b1) - 1.0) <= 1e-12


def _gpu_solver(src, y, nu, prm, precision="fp64"):
    s = SotSolver(dim=3, device=0, precision=precision)
    s.set_distance_function("spherical")
    s.setup_source(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"])
    s.setup_target(y, nu)
    s.configure(prm)
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("tau,lse", [(0.0, True), (1e-8, True), (1e-8, False)])
def test_spherical_evaluate_matches_oracle(oracle_mod, tau, lse):
    src, y, nu, P = _problem(oracle_mod, seed=3, n_targets=80)
    eps = 0.05
    prm = SolverParameters(epsilon=eps, tau=tau, use_log_sum_exp_trick=lse)
    op = oracle_mod.Params(epsilon=eps, tau=tau, use_log_sum_exp=lse)
    psi = 0.02 * np.random.default_rng(4).standard_normal(len(nu))
    for precision in ("fp64", "hybrid"):
        s = _gpu_solver(src, y, nu, prm, precision)
        g = np.zeros(len(nu))
        J = s.evaluate_functional(psi, g)
        P.reset_state()
        Jo, go, st = P.evaluate(psi, op)
        assert s.get_last_distance_threshold() == st["threshold"]
        assert s.last_eval_info["n_pairs"] == st["n_pairs"]
        assert abs(J - Jo) <= 1e-10 * abs(Jo)
        assert np.max(np.abs(g - go)) <= 1e-12
        assert abs(s.get_C_global() - st["C_global"]) <= 1e-10 * abs(st["C_global"])
        s.close()


@pytest.mark.gpu
def test_spherical_solve_and_barycenters(oracle_mod):
    src, y, nu, P = _problem(oracle_mod, seed=5, n_targets=50)
    eps = 0.05
    # |g|_inf <= 1e-8: the reference's line search itself stops at 1.3e-9 on
    # this problem when asked for 1e-9 (the oracle's solve reports it)
    prm = SolverParameters(epsilon=eps, tau=0.0, use_log_sum_exp_trick=True, tolerance=1e-8,
                           solver_control_type="linf", max_iterations=3000)
    s = _gpu_solver(src, y, nu, prm)
    psi = s.solve(np.zeros(len(nu)), prm)
    assert s.get_convergence_status()
    op = oracle_mod.Params(epsilon=eps, tau=0.0, use_log_sum_exp=True, tolerance=1e-8, solver_control_type="linf",
                           max_iterations=3000)
    P.reset_state()
    _, oinfo = P.solve(np.zeros(len(nu)), op)
    assert oinfo["converged"]
    assert abs(s.get_last_iteration_count() - oinfo["iterations"]) <= 3
    P.reset_state()
    _, go, _ = P.evaluate(psi, op)
    assert np.max(np.abs(go)) <= 1.5e-8
    # barycenter iteration from the targets themselves, a few steps
    bprm = SolverParameters(epsilon=eps, tau=0.0, use_log_sum_exp_trick=True, tolerance=1e-12, max_iterations=4)
    b = s.evaluate_weighted_barycenters(psi, bprm, barycenters=y)
    info = s.last_barycenter_info
    bo, ito, nrmo = P.spherical_barycenters(psi, op, 1e300, y, 4, 1e-12)
    assert info["iterations"] == ito
    assert abs(info["grad_norm"] - nrmo) <= 1e-10 * max(nrmo, 1e-300)
    assert np.max(np.abs(b - bo)) <= 1e-10
    assert np.allclose(np.linalg.norm(b, axis=1), 1.0, atol=1e-12)
    with pytest.raises(RuntimeError):
        s.compute_hessian(psi)
    s.close()
