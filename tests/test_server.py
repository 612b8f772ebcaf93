"""Solve service (sdot_server_*): admission by budget, concurrency, determinism.

Continuous batching: requests submitted while others run are admitted as
slots and memory free up and their work overlaps on the device.  Solves are
deterministic (fixed-order reductions), so every request's potential must be
bitwise the one it gets when solved alone (tolerance 0), and each must meet its
FP64 gradient tolerance.
"""
import numpy as np
import pytest

from semidiscreteot_b200 import SolveServer, SolverParameters, SotSolver, structured_source

pytestmark = pytest.mark.gpu


def requests(seed=0, n=6):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        dim = 2 if i % 2 == 0 else 3
        if dim == 2:
            src = structured_source(2, int(rng.integers(8, 24)), 3,
                                    nodal_density=lambda p: 0.3 + np.exp(-np.sum((p - 0.5) ** 2, axis=1) / 0.1))
        else:
            src = structured_source(3, int(rng.integers(5, 9)), 2)
        nt = int(rng.integers(60, 900))
        y = rng.random((nt, dim))
        nu = rng.dirichlet(np.ones(nt) * 3)
        eps = [3e-2, 1e-2][i % 2]
        prm = SolverParameters(epsilon=eps, tau=0.0, use_log_sum_exp_trick=True, tolerance=1e-9,
                               solver_control_type="linf", max_iterations=3000)
        out.append((src, y, nu, prm))
    return out


def check_fp64(src, y, nu, prm, psi):
    s = SotSolver(dim=y.shape[1], device=0, precision="fp64")
    s.setup_source(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"])
    s.setup_target(y, nu)
    s.configure(prm)
    g = np.zeros(len(nu))
    s.evaluate_functional(psi, g)
    s.close()
    return float(np.max(np.abs(g)))


@pytest.mark.parametrize("method", ["newton", "lbfgs"])
def test_results_identical_alone_and_in_the_mix(method):
    reqs = requests(1)
    if method == "lbfgs":
        # the reference's line search stops short of 1e-9 on all six problems
        # (the oracle's own solves report it) and reaches 1e-8 on every one
        reqs = [(src, y, nu, SolverParameters(epsilon=prm.epsilon, tau=0.0, use_log_sum_exp_trick=True,
                                              tolerance=1e-8, solver_control_type="linf", max_iterations=3000))
                for src, y, nu, prm in reqs]
    alone = []
    with SolveServer(n_slots=1) as srv:
        for src, y, nu, prm in reqs:
            t = srv.submit(src, y, nu, prm, method=method, precision="fp64")
            alone.append(srv.wait(t))
    with SolveServer(n_slots=4) as srv:
        tickets = [srv.submit(src, y, nu, prm, method=method, precision="fp64") for src, y, nu, prm in reqs]
        mixed = [srv.wait(t) for t in tickets]
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["peak_running"] >= 2, st          # requests overlapped
    for (src, y, nu, prm), (pa, ra), (pm, rm) in zip(reqs, alone, mixed):
        assert ra["converged"] and rm["converged"], (ra, rm)
        assert ra["method"] == method
        assert np.array_equal(pa, pm)             # same alone and in the mix
        assert ra["iterations"] == rm["iterations"]
        assert check_fp64(src, y, nu, prm, pm) <= 1.5 * prm.tolerance


def test_budget_admission_and_rejection():
    reqs = requests(2, n=4)
    # every request fits alone, two do not fit together: no overlap
    with SolveServer(n_slots=4, memory_budget=150 << 20) as srv:
        tickets = [srv.submit(src, y, nu, prm, method="newton") for src, y, nu, prm in reqs]
        res = [srv.wait(t) for t in tickets]
        st = srv.stats()
    assert st["peak_running"] == 1, st
    assert all(r["converged"] for _, r in res)
    assert st["p99_ms"] >= st["p50_ms"] > 0
    with SolveServer(n_slots=2, memory_budget=1 << 20) as srv:
        src, y, nu, prm = reqs[0]
        with pytest.raises(RuntimeError, match="budget"):
            srv.submit(src, y, nu, prm)


def test_points_only_requests_and_warm_start():
    src, y, nu, prm = requests(3, n=1)[0]
    with SolveServer(n_slots=2) as srv:
        t1 = srv.submit(src, y, nu, prm, method="newton", with_cells=False)
        p1, r1 = srv.wait(t1)
        assert r1["converged"]
        srv.reset_stats()                          # statistics from here on
        assert srv.stats()["completed"] == 0
        t2 = srv.submit(src, y, nu, prm, method="newton", psi0=p1)
        p2, r2 = srv.wait(t2)
        assert r2["converged"] and r2["iterations"] <= 1
        t3 = srv.submit(src, y, nu, prm, method="newton", epsilon_scaling_factor=4.0, epsilon_scaling_steps=3,
                        intermediate_tolerance=1e-6)
        p3, r3 = srv.wait(t3)
        assert r3["converged"]
        st = srv.stats()
        assert st["completed"] == 2 and st["failed"] == 0, st
        assert st["p99_ms"] >= st["p50_ms"] > 0
    for p in (p1, p2, p3):
        assert check_fp64(src, y, nu, prm, p) <= 1e-9
