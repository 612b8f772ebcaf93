"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py).

CPU: the oracle still reproduces its frozen outputs (pins the oracle against
changes).  GPU: the CUDA path, through the C ABI, reproduces them with the
parity tolerances: value 1e-10 relative, gradient 1e-12 absolute in FP64 mode
(max(1e-8, 5e-6 max nu) in the hybrid mode), pair counts and pointwise radii
exact, C_global 1e-10 relative, Hessian 1e-9 of its largest entry.  Each case
runs three evaluations in a row (pointwise at psi1, then the case's threshold
type at psi1 and psi2, which read the state the previous evaluation left).
"""
import glob
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
NAMES = [os.path.splitext(os.path.basename(f))[0] for f in FIXTURES]


def load(name):
    return np.load(os.path.join(HERE, "golden", name + ".npz"))


def case_params(d):
    dim, n, order, N, eps, tau, lse, seed = d["meta"]
    return int(dim), float(eps), float(tau), bool(lse), str(d["threshold_type"])


def test_fixtures_present():
    assert len(FIXTURES) >= 7


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_golden(oracle_mod, name):
    d = load(name)
    dim, eps, tau, lse, ttype = case_params(d)
    P = oracle_mod.Problem(d["x"], d["jxw"], d["rho"], d["cell_offsets"], d["cell_centers"], d["y"], d["nu"])
    pw = oracle_mod.Params(epsilon=eps, tau=tau, use_log_sum_exp=lse)
    pc = oracle_mod.Params(epsilon=eps, tau=tau, use_log_sum_exp=lse, distance_threshold_type=ttype)
    for k, (psi, p) in enumerate(((d["psi1"], pw), (d["psi1"], pc), (d["psi2"], pc))):
        J, g, st = P.evaluate(psi, p)
        assert st["n_pairs"] == int(d[f"pairs{k}"])
        assert st["threshold"] == pytest.approx(float(d[f"r{k}"]), rel=1e-14)
        assert J == pytest.approx(float(d[f"J{k}"]), rel=1e-13)
        assert np.max(np.abs(g - d[f"g{k}"])) <= 1e-15
        assert st["C_global"] == pytest.approx(float(d[f"C{k}"]), rel=1e-13)
    assert P.covering_radius() == float(d["covering_radius"])
    P.reset_state()
    r1 = P.distance_threshold(d["psi1"], pw)
    assert r1 == float(d["H_r"])
    H = P.hessian(d["psi1"], pw, r1)
    assert np.max(np.abs(H - d["H"])) <= 1e-13 * np.max(np.abs(d["H"]))


def _solver(d, precision):
    from semidiscreteot_b200 import SotSolver
    dim = int(d["meta"][0])
    s = SotSolver(dim=dim, device=0, precision=precision)
    s.setup_source(d["x"], d["jxw"], d["rho"], d["cell_offsets"], d["cell_centers"])
    s.setup_target(d["y"], d["nu"])
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "hybrid"])
@pytest.mark.parametrize("name", NAMES)
def test_cuda_matches_golden(name, precision):
    from semidiscreteot_b200 import SolverParameters
    d = load(name)
    dim, eps, tau, lse, ttype = case_params(d)
    nu = d["nu"]
    gtol = 1e-12 if precision == "fp64" else max(1e-8, 5e-6 * float(np.max(nu)))
    s = _solver(d, precision)
    pw = SolverParameters(epsilon=eps, tau=tau, use_log_sum_exp_trick=lse)
    pc = SolverParameters(epsilon=eps, tau=tau, use_log_sum_exp_trick=lse, distance_threshold_type=ttype)
    for k, (psi, p) in enumerate(((d["psi1"], pw), (d["psi1"], pc), (d["psi2"], pc))):
        s.configure(p)
        g = np.zeros(len(nu))
        J = s.evaluate_functional(psi, g)
        r = s.get_last_distance_threshold()
        if ttype == "pointwise" or k == 0:
            assert r == float(d[f"r{k}"])
        else:
            # the stateful radii read J of the previous evaluation (1e-16 level)
            assert r == pytest.approx(float(d[f"r{k}"]), rel=1e-13)
        assert s.last_eval_info["n_pairs"] == int(d[f"pairs{k}"])
        assert abs(J - float(d[f"J{k}"])) <= 1e-10 * abs(float(d[f"J{k}"]))
        assert np.max(np.abs(g - d[f"g{k}"])) <= gtol
        assert s.get_C_global() == pytest.approx(float(d[f"C{k}"]), rel=1e-10)
    assert s.compute_covering_radius() == float(d["covering_radius"])
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_cuda_hessian_and_solve_match_golden(name):
    from semidiscreteot_b200 import SolverParameters
    d = load(name)
    dim, eps, tau, lse, ttype = case_params(d)
    s = _solver(d, "fp64")
    s.configure(SolverParameters(epsilon=eps, tau=tau, use_log_sum_exp_trick=lse))
    H = s.compute_hessian(d["psi1"])
    assert np.max(np.abs(H - d["H"])) <= 1e-9 * np.max(np.abs(d["H"]))
    prm = SolverParameters(epsilon=eps, tau=min(tau, 1e-14) if tau > 0 else 0.0, use_log_sum_exp_trick=lse,
                           solver_control_type="linf", tolerance=1e-8, max_iterations=2000)
    psi = s.solve(np.zeros(len(d["nu"])), prm)
    assert s.get_convergence_status()
    assert bool(d["solve_converged"])
    dd = (psi - psi.mean()) - (d["solve_psi"] - d["solve_psi"].mean())
    assert np.max(np.abs(dd)) <= 1e-5
    s.close()
