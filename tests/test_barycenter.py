"""Weighted barycenters and potential-conditioned densities against the oracle.

Barycenters (compute_weighted_barycenters_euclidean) agree with the oracle's
restatement to 1e-10 relative + 1e-12 absolute: the plan entries come from the
FP64 evaluation's log-normalisers L_q instead of the reference's per-point
max/sum, and the sums run in a different fixed order; the candidate sets
(centre test) are bit-exact.  Conditioned densities agree to 1e-12 relative to
the largest value, with identical zero patterns (the per-point candidate test
is exact).
"""
import numpy as np
import pytest

from semidiscreteot_b200 import SolverParameters, SotSolver, structured_source

pytestmark = pytest.mark.gpu


def problem(rng, dim, n, order, N):
    src = structured_source(dim, n, order,
                            nodal_density=lambda p: 0.5 + np.exp(-np.sum((p - 0.5) ** 2, axis=1) / 0.1))
    y = rng.random((N, dim))
    nu = rng.dirichlet(np.ones(N) * 3)
    return src, y, nu


def solver_for(src, y, nu, dim, params):
    s = SotSolver(dim=dim, device=0, precision="fp64")
    s.setup_source(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"])
    s.setup_target(y, nu)
    s.configure(params)
    return s


@pytest.mark.parametrize("dim,lse,tau", [(2, True, 0.0), (2, False, 0.0), (2, True, 1e-4),
                                         (3, True, 0.0), (3, True, 1e-3)])
def test_barycenters_match_oracle(oracle_mod, dim, lse, tau):
    rng = np.random.default_rng(11 + dim)
    src, y, nu = problem(rng, dim, 12 if dim == 2 else 6, 3 if dim == 2 else 2, 150 if dim == 2 else 90)
    eps = 3e-2
    prm = SolverParameters(epsilon=eps, tau=tau, use_log_sum_exp_trick=lse)
    s = solver_for(src, y, nu, dim, prm)
    psi = 0.5 * eps * rng.standard_normal(len(nu))
    got = s.evaluate_weighted_barycenters(psi)
    r = s.get_last_distance_threshold()
    if tau > 0:
        assert r < 1.0                                   # the truncated path ran
    P = oracle_mod.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"], y, nu)
    want = P.weighted_barycenters(psi, oracle_mod.Params(epsilon=eps, tau=tau, use_log_sum_exp=lse), r)
    assert got.shape == (len(nu), dim)
    assert np.array_equal(got == 0.0, want == 0.0)
    np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-12)
    s.close()


def test_barycenters_keep_functional_state(oracle_mod):
    rng = np.random.default_rng(5)
    src, y, nu = problem(rng, 2, 8, 2, 40)
    s = solver_for(src, y, nu, 2, SolverParameters(epsilon=5e-2, tau=0.0))
    psi = 0.01 * rng.standard_normal(40)
    s.evaluate_functional(psi)
    f, C = s.get_last_functional_value(), s.get_C_global()
    s.evaluate_weighted_barycenters(np.zeros(40))
    assert s.get_last_functional_value() == f and s.get_C_global() == C
    s.close()


@pytest.mark.parametrize("dim", [2, 3])
def test_conditioned_densities_match_oracle(oracle_mod, dim):
    rng = np.random.default_rng(21 + dim)
    src, y, nu = problem(rng, dim, 6, 2, 300 if dim == 2 else 200)
    eps = 2e-2
    s = solver_for(src, y, nu, dim, SolverParameters(epsilon=eps, tau=0.0))
    P = oracle_mod.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"], y, nu)
    psi = 0.5 * eps * rng.standard_normal(len(nu))
    pts = rng.random((257, dim))
    dens = rng.random(257) + 0.25
    idx = np.concatenate([rng.choice(len(nu), 37, replace=False), [0, 0]])
    for r in (1e300, 0.25, 0.08):
        got = s.get_potential_conditioned_density(pts, dens, psi, idx, epsilon=eps, threshold=r)
        want = P.conditioned_densities(psi, eps, r, pts, dens, idx)
        assert np.array_equal(got == 0.0, want == 0.0), r
        assert np.max(np.abs(got - want)) <= 1e-12 * max(1.0, np.max(np.abs(want))), r
    # every target requested, untruncated: the values weighted by nu sum to the density
    allv = s.get_potential_conditioned_density(pts, dens, psi, np.arange(len(nu)), epsilon=eps, threshold=1e300)
    np.testing.assert_allclose(nu @ allv, dens, rtol=1e-12)
    with pytest.raises(RuntimeError):
        s.get_potential_conditioned_density(pts, dens, psi, [len(nu)], epsilon=eps, threshold=1e300)
    s.close()
