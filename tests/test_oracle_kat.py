"""Known-answer and property tests of the FP64 CPU oracle (no GPU).

The reference ships no golden vectors (parity unpinned), so the oracle's
restatement of SotSolver's evaluation is checked from first principles:
analytic single-target values, symmetry, mass conservation, shift invariance,
finite-difference gradient and Hessian, the candidate predicate against a
brute-force scan, the threshold formulas against a Python restatement, and
the solver/line-search semantics (control types, upstream vs vendored).
"""
import math

import numpy as np
import pytest


def unit_square(orc, n=8, order=3):
    return orc.structured_source(2, n, 0.0, 1.0, order)


def test_gauss_legendre(oracle_mod):
    for n in range(1, 8):
        x, w = oracle_mod.gauss_legendre(n)
        xr, wr = np.polynomial.legendre.leggauss(n)
        np.testing.assert_allclose(x, 0.5 * (xr + 1), atol=1e-15)
        np.testing.assert_allclose(w, 0.5 * wr, atol=1e-15)
        # exact for polynomials of degree 2n-1
        for k in range(2 * n):
            assert abs(np.sum(w * x ** k) - 1.0 / (k + 1)) < 1e-14


def test_structured_source_matches_product_generator(oracle_mod):
    from semidiscreteot_b200.source import structured_source
    for dim, n, order in [(2, 8, 3), (3, 4, 2), (2, 5, 2)]:
        rng = np.random.default_rng(dim * 10 + n)
        nodal = rng.random((n + 1) ** dim) + 0.5
        xq, jxw, rho, off, ctr = oracle_mod.structured_source(dim, n, 0.0, 1.0, order, nodal)
        p = structured_source(dim, n, order, nodal_density=nodal)
        np.testing.assert_allclose(p["x"], xq, atol=1e-15)
        np.testing.assert_allclose(p["jxw"], jxw, rtol=1e-14)
        np.testing.assert_allclose(p["density"], rho, rtol=1e-13)
        np.testing.assert_array_equal(p["cell_offsets"], off)
        np.testing.assert_allclose(p["cell_centers"], ctr, atol=0)
        # normalised: sum |rho| JxW = 1 (SemiDiscreteOT::normalize_density)
        assert abs(np.sum(np.abs(rho) * jxw) - 1.0) < 1e-13


def test_single_target_closed_form(oracle_mod):
    """N = 1, nu = 1: pi = 1 everywhere, grad = 0 for any psi and
    J = -1/2 int |x - y|^2 rho dx (independent of psi)."""
    xq, jxw, rho, off, ctr = unit_square(oracle_mod, 8, 3)
    y = np.array([[0.5, 0.5]])
    P = oracle_mod.Problem(xq, jxw, rho, off, ctr, y, [1.0])
    for lse in (True, False):
        prm = oracle_mod.Params(epsilon=0.05, tau=0.0, use_log_sum_exp=lse)
        for psi in (0.0, 0.37):
            J, g, _ = P.evaluate([psi], prm)
            assert abs(g[0]) < 1e-14
            # uniform density on [0,1]^2: int |x - c|^2 = 1/12 + 1/12
            assert abs(J - (-0.5 * (1.0 / 6.0))) < 1e-13


def test_symmetric_two_targets(oracle_mod):
    """Targets mirrored about x = 1/2 with equal weights: psi = 0 is optimal."""
    xq, jxw, rho, off, ctr = unit_square(oracle_mod, 8, 3)
    y = np.array([[0.25, 0.5], [0.75, 0.5]])
    P = oracle_mod.Problem(xq, jxw, rho, off, ctr, y, [0.5, 0.5])
    prm = oracle_mod.Params(epsilon=0.02, tau=0.0, use_log_sum_exp=True)
    J, g, _ = P.evaluate([0.0, 0.0], prm)
    assert np.max(np.abs(g)) < 1e-14


def random_problem(orc, seed=0, N=40, dim=2, n=8, order=3):
    rng = np.random.default_rng(seed)
    xq, jxw, rho, off, ctr = orc.structured_source(dim, n, 0.0, 1.0, order,
                                                   rng.random((n + 1) ** dim) + 0.2)
    y = rng.random((N, dim))
    nu = rng.dirichlet(np.ones(N) * 3)
    return orc.Problem(xq, jxw, rho, off, ctr, y, nu), rng


@pytest.mark.parametrize("lse", [True, False])
def test_mass_and_shift(oracle_mod, lse):
    P, rng = random_problem(oracle_mod, 1)
    prm = oracle_mod.Params(epsilon=0.03, tau=0.0, use_log_sum_exp=lse)
    psi = 0.01 * rng.standard_normal(P.N)
    J, g, st = P.evaluate(psi, prm)
    # mass conservation: sum_j (g_j + nu_j) = sum_q rho_q JxW_q = 1
    assert abs(np.sum(g + P.nu) - np.sum(P.rho * P.jxw)) < 1e-13
    # shift invariance J(psi + c) = J(psi) when sum nu = 1 (no truncation)
    J2, g2, _ = P.evaluate(psi + 0.123, prm)
    assert abs(J2 - J) < 1e-13
    np.testing.assert_allclose(g2, g, atol=1e-14)


def test_fd_gradient_and_hessian(oracle_mod):
    P, rng = random_problem(oracle_mod, 2, N=25)
    prm = oracle_mod.Params(epsilon=0.04, tau=0.0, use_log_sum_exp=True)
    psi = 0.01 * rng.standard_normal(P.N)
    J, g, _ = P.evaluate(psi, prm)
    H = P.hessian(psi, prm, 1e300)
    h = 1e-6
    for j in (0, 7, 19):
        e = np.zeros(P.N)
        e[j] = h
        Jp, gp, _ = P.evaluate(psi + e, prm)
        Jm, gm, _ = P.evaluate(psi - e, prm)
        assert abs((Jp - Jm) / (2 * h) - g[j]) < 1e-8
        np.testing.assert_allclose((gp - gm) / (2 * h), H[:, j], atol=1e-6)
    np.testing.assert_allclose(H, H.T, atol=1e-13)
    assert np.max(np.abs(H @ np.ones(P.N))) < 1e-11          # constant null vector
    assert np.min(np.linalg.eigvalsh(H)) > -1e-10              # positive semi-definite


def test_candidates_match_bruteforce(oracle_mod):
    P, rng = random_problem(oracle_mod, 3, N=300)
    for r in (0.05, 0.2, 0.5, 0.0, 2.0):
        for c in P.ctr[::7]:
            got = P.candidates(c, r)
            d = np.sqrt(np.sum((P.y - c) ** 2, axis=1))
            np.testing.assert_array_equal(got, np.nonzero(d <= r)[0])


def test_thresholds(oracle_mod):
    P, rng = random_problem(oracle_mod, 4, N=50)
    psi = 0.05 * rng.standard_normal(P.N)
    eps, tau = 0.01, 1e-8
    nu_min = P.nu.min()
    prm = oracle_mod.Params(epsilon=eps, tau=tau, distance_threshold_type="pointwise")
    r = P.distance_threshold(psi, prm)
    assert r == math.sqrt(max(0.0, -2.0 * eps * math.log(tau / nu_min) + 2.0 * psi.max()))
    # tau <= 0 -> no truncation (DBL_MAX)
    assert P.distance_threshold(psi, oracle_mod.Params(epsilon=eps, tau=0.0)) == np.finfo(float).max
    # integral bound with state C, J
    P.state.C_global, P.state.global_functional = 3.0, -0.02
    P.state.covering_radius = 0.01
    ri = P.distance_threshold(psi, oracle_mod.Params(epsilon=eps, tau=tau, distance_threshold_type="integral"))
    expect = math.sqrt(max(0.0, 2.0 * psi.max() + 2.0 * eps * math.log((eps * 3.0) / (tau * 0.02))))
    assert ri == max(expect, 0.01)
    # geometric bound
    P.state.covering_radius = 0.1
    rg = P.distance_threshold(psi, oracle_mod.Params(epsilon=eps, tau=tau, distance_threshold_type="geometric"))
    lt = math.log(eps / (nu_min * tau * 0.02))
    r2 = 0.1 * 0.1 + 2.0 * (psi.max() - psi.min()) + 2.0 * eps * lt
    assert rg == math.sqrt(max(r2, 0.01))


def test_covering_radius(oracle_mod):
    P, _ = random_problem(oracle_mod, 5, N=30)
    d = np.sqrt(((P.ctr[:, None, :] - P.y[None, :, :]) ** 2).sum(-1))
    assert P.covering_radius() == d.min(axis=1).max()


def test_truncated_evaluation_subset(oracle_mod):
    """With a threshold, each cell only sees its candidates: pair count and
    skipped cells behave like the reference (cells without candidates skip)."""
    P, rng = random_problem(oracle_mod, 6, N=200)
    prm = oracle_mod.Params(epsilon=0.01, tau=1e-3, use_log_sum_exp=True)
    psi = np.zeros(P.N)
    J, g, st = P.evaluate(psi, prm)
    r = st["threshold"]
    assert r < 1.0
    expect = 0
    qpc = int(P.off[1] - P.off[0])
    for c in P.ctr:
        expect += qpc * np.count_nonzero(np.sqrt(((P.y - c) ** 2).sum(1)) <= r)
    assert st["n_pairs"] == expect


def test_faithful_mode_same_numbers(oracle_mod):
    P, rng = random_problem(oracle_mod, 7, N=60)
    prm = oracle_mod.Params(epsilon=0.02, tau=1e-6, use_log_sum_exp=True)
    psi = 0.01 * rng.standard_normal(P.N)
    J1, g1, _ = P.evaluate(psi, prm, faithful=False)
    P.reset_state()
    J2, g2, _ = P.evaluate(psi, prm, faithful=True)
    assert abs(J1 - J2) < 1e-14
    np.testing.assert_allclose(g1, g2, atol=1e-15)


@pytest.mark.parametrize("control", ["l1norm", "componentwise", "linf"])
def test_solver_controls(oracle_mod, control):
    P, rng = random_problem(oracle_mod, 8, N=30)
    tol = {"l1norm": 1e-7, "componentwise": 1e-5, "linf": 1e-8}[control]
    prm = oracle_mod.Params(epsilon=0.05, tau=0.0, use_log_sum_exp=True, solver_control_type=control,
                            tolerance=tol, max_iterations=500)
    psi, info = P.solve(np.zeros(P.N), prm)
    assert info["converged"] and info["status"] == 0
    _, g, _ = P.evaluate(psi, prm)
    if control == "l1norm":
        assert np.sum(np.abs(g)) <= tol
    elif control == "componentwise":
        assert np.all(np.abs(g) <= P.nu * tol)
    else:
        assert np.max(np.abs(g)) <= tol


def test_solver_max_iterations(oracle_mod):
    """Non-convergence is reported, not raised (SotSolver.cc:207-211)."""
    P, _ = random_problem(oracle_mod, 9, N=30)
    prm = oracle_mod.Params(epsilon=0.05, tau=0.0, use_log_sum_exp=True, solver_control_type="linf",
                            tolerance=1e-14, max_iterations=3)
    psi, info = P.solve(np.zeros(P.N), prm)
    assert not info["converged"] and info["iterations"] == 3 and info["status"] == 1


def test_epsilon_sequence(oracle_mod):
    from semidiscreteot_b200.parameters import epsilon_sequence
    np.testing.assert_allclose(oracle_mod.epsilon_sequence(1e-3, 10.0, 3), [1e-1, 1e-2, 1e-3])
    assert list(oracle_mod.epsilon_sequence(1e-2, 0.5, 2)) == [2e-2, 1e-2]   # factor <= 1 -> 2
    assert list(oracle_mod.epsilon_sequence(1e-2, 3.0, 0)) == [1e-2]          # steps 0 -> 1
    for eps, f, s in [(1e-3, 10.0, 3), (1e-2, 0.5, 2), (5e-3, 2.0, 5)]:
        np.testing.assert_allclose(epsilon_sequence(eps, f, s), oracle_mod.epsilon_sequence(eps, f, s), rtol=1e-15)


def test_softmax_refinement_single_child(oracle_mod):
    """Coarse targets each with one child at the same position: the transfer
    returns -eps log sum_q w_q e^{-m_q}/S_q e^{-d^2/2eps}, and the fine
    potentials reproduce the coarse ones up to a common constant shift."""
    P, rng = random_problem(oracle_mod, 10, N=20)
    prm = oracle_mod.Params(epsilon=0.05, tau=0.0, use_log_sum_exp=True, solver_control_type="linf",
                            tolerance=1e-9, max_iterations=2000, line_search="vendored")
    psi, info = P.solve(np.zeros(P.N), prm)
    assert info["converged"], info
    co = np.arange(P.N + 1, dtype=np.int64)
    ci = np.arange(P.N, dtype=np.int64)
    fine = P.softmax_refinement(psi, 0.05, 1e300, True, P.y, co, ci)
    # psi_fine_j = psi_j - eps log((g_j + nu_j)/nu_j): equal up to eps*|g|/nu
    d = (fine - fine.mean()) - (psi - psi.mean())
    assert np.max(np.abs(d)) < 1e-6


def test_weighted_barycenters_known_answers(oracle_mod):
    """Single target: the barycenter is sum_q w_q x_q / nu.  Several targets,
    untruncated: sum_j nu_j B_j = sum_q w_q x_q (the plan's rows sum to w_q),
    for both log-sum-exp settings."""
    xq, jxw, rho, off, ctr = unit_square(oracle_mod, 8, 3)
    w = rho * jxw
    P1 = oracle_mod.Problem(xq, jxw, rho, off, ctr, np.array([[0.3, 0.6]]), [0.7])
    B1 = P1.weighted_barycenters([0.2], oracle_mod.Params(epsilon=0.05, tau=0.0), 1e300)
    np.testing.assert_allclose(B1[0], (w @ xq) / 0.7, rtol=1e-13)
    P, rng = random_problem(oracle_mod, 8, N=15)
    psi = 0.02 * rng.standard_normal(P.N)
    wsum = (P.rho * P.jxw) @ P.xq.reshape(-1, 2)
    for lse in (True, False):
        B = P.weighted_barycenters(psi, oracle_mod.Params(epsilon=0.03, tau=0.0, use_log_sum_exp=lse), 1e300)
        np.testing.assert_allclose(P.nu @ B, wsum, rtol=1e-12)


def test_conditioned_densities_known_answers(oracle_mod):
    """Untruncated: sum_k nu_k c_k(p) = density(p); a target outside the
    threshold of a point gets 0 there."""
    P, rng = random_problem(oracle_mod, 6, N=12)
    psi = 0.02 * rng.standard_normal(P.N)
    pts = rng.random((40, 2))
    dens = rng.random(40) + 0.5
    c = P.conditioned_densities(psi, 0.04, 1e300, pts, dens, np.arange(P.N))
    np.testing.assert_allclose(P.nu @ c, dens, rtol=1e-13)
    r = 0.3
    ct = P.conditioned_densities(psi, 0.04, r, pts, dens, np.arange(P.N))
    d = np.linalg.norm(P.y.reshape(-1, 2)[:, None, :] - pts[None, :, :], axis=2)
    assert np.all(ct[d > r] == 0.0)
    has = (d <= r).any(axis=0)
    np.testing.assert_allclose((P.nu @ ct)[has], dens[has], rtol=1e-13)
