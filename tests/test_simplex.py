"""Simplex sources (FE_SimplexP(1) + a simplex rule, flattened per cell).

CPU: the rules integrate every monomial up to their degree exactly on the
reference simplex; the meshes tile their domain; P1 sources integrate linear
densities exactly; gmsh files round-trip (and the tutorial_0 mesh, when the
reference tree is present, reads as 98,304 tetrahedra over the same vertices
as ``tetra_cube_mesh(16)``).
GPU: value and gradient on triangle and tetrahedron sources against the
oracle (1e-10 relative / 1e-8 absolute, as for the hexahedral sources), and a
solve of the tutorial_0 settings (epsilon 1e-2, tau 1e-12, no log-sum-exp,
pointwise threshold) on a reduced tet mesh.
"""
import itertools
import math
import os

import numpy as np
import pytest

from semidiscreteot_b200.io import read_msh, write_msh
from semidiscreteot_b200.simplex import simplex_rule, simplex_source, tetra_cube_mesh, triangle_square_mesh

# The reference's tutorial_0 mesh (examples/tutorial_0/run/source.msh) is not
# committed; tests that read it run when SDOT_TUTORIAL_MESH names the file.
TUTORIAL_MESH = os.environ.get("SDOT_TUTORIAL_MESH", "")


def exact_monomial(alpha):
    """int over the unit reference simplex of prod x_d^alpha_d."""
    return math.prod(math.factorial(a) for a in alpha) / math.factorial(sum(alpha) + len(alpha))


@pytest.mark.parametrize("dim,n,degree", [(2, 1, 1), (2, 2, 2), (2, 3, 5), (3, 1, 1), (3, 2, 2), (3, 3, 3)])
def test_rule_exactness(dim, n, degree):
    B, w = simplex_rule(dim, n)
    assert np.all(w > 0) and np.all(B >= 0) and np.allclose(B.sum(axis=1), 1.0, atol=1e-15)
    X = B[:, :dim]                                   # Cartesian coordinates on the reference simplex
    for alpha in itertools.product(range(degree + 1), repeat=dim):
        if sum(alpha) > degree:
            continue
        got = np.sum(w * np.prod(X ** np.array(alpha), axis=1))
        assert abs(got - exact_monomial(alpha)) < 1e-15, (alpha, got)
    counts = {2: [1, 3, 7], 3: [1, 4, 10]}
    assert B.shape[0] == counts[dim][n - 1]


def test_meshes_tile_their_domain():
    V, T = triangle_square_mesh(9)
    C = V[T]
    d = np.linalg.det(C[:, :2] - C[:, 2:3])
    assert abs(np.abs(d).sum() / 2 - 1.0) < 1e-14 and np.all(np.abs(d) > 0)
    V3, T3 = tetra_cube_mesh(3, -1.0, 1.0)
    assert T3.shape == (27 * 24, 4) and V3.shape[0] == 4 ** 3 + 3 * 4 * 9
    C3 = V3[T3]
    d3 = np.linalg.det(C3[:, :3] - C3[:, 3:4])
    assert abs(np.abs(d3).sum() / 6 - 8.0) < 1e-13 and np.all(np.abs(d3) > 1e-12)


@pytest.mark.parametrize("dim", [2, 3])
def test_p1_source_integrates_linear_densities(dim):
    V, T = triangle_square_mesh(6) if dim == 2 else tetra_cube_mesh(2, 0.0, 1.0)
    lin = lambda P: 1.0 + P @ np.arange(1, dim + 1)   # noqa: E731
    src = simplex_source(V, T, lin, order=2, normalize=False)
    # int over the unit cube of 1 + sum (d+1) x_d = 1 + sum (d+1)/2
    assert abs(np.sum(src["density"] * src["jxw"]) - (1.0 + sum((d + 1) / 2 for d in range(dim)))) < 1e-13
    # first moments: int x_0 (1 + ...) exactly (degree 2 integrand, order-2 rule)
    want = 0.5 + sum((d + 1) * (1 / 3 if d == 0 else 1 / 4) for d in range(dim))
    assert abs(np.sum(src["density"] * src["jxw"] * src["x"][:, 0]) - want) < 1e-13
    nrm = simplex_source(V, T, lin, order=3)
    assert abs(np.sum(np.abs(nrm["density"]) * nrm["jxw"]) - 1.0) < 1e-13
    np.testing.assert_allclose(nrm["cell_centers"], V[T].mean(axis=1))
    assert np.all(np.diff(nrm["cell_offsets"]) == simplex_rule(dim, 3)[0].shape[0])


def test_msh_round_trip(tmp_path):
    V, T = tetra_cube_mesh(2)
    m = read_msh(write_msh(str(tmp_path / "m.msh"), V, T))
    assert m["dim"] == 3
    np.testing.assert_array_equal(m["nodes"], V)
    np.testing.assert_array_equal(m["cells"], T)
    V2, T2 = triangle_square_mesh(3)
    m2 = read_msh(write_msh(str(tmp_path / "t.msh"), V2, T2))
    assert m2["dim"] == 2 and np.array_equal(m2["cells"], T2) and np.array_equal(m2["nodes"][:, :2], V2)


@pytest.mark.skipif(not (TUTORIAL_MESH and os.path.exists(TUTORIAL_MESH)), reason="SDOT_TUTORIAL_MESH not set")
def test_reads_tutorial_mesh():
    m = read_msh(TUTORIAL_MESH)
    assert m["dim"] == 3 and m["cells"].shape == (98304, 4) and m["nodes"].shape == (17969, 3)
    V, _ = tetra_cube_mesh(16)
    assert set(map(tuple, np.round(m["nodes"], 12))) == set(map(tuple, np.round(V, 12)))
    C = m["nodes"][m["cells"]]
    assert abs(np.abs(np.linalg.det(C[:, :3] - C[:, 3:4])).sum() / 6 - 8.0) < 1e-12


def test_oracle_mass_on_simplex_source(oracle_mod):
    V, T = tetra_cube_mesh(2)
    src = simplex_source(V, T, lambda P: 1.5 + P[:, 0], order=3)
    rng = np.random.default_rng(0)
    y = rng.uniform(-1, 1, (20, 3))
    nu = np.full(20, 0.05)
    P = oracle_mod.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"], y, nu)
    _, g, _ = P.evaluate(0.01 * rng.standard_normal(20), oracle_mod.Params(epsilon=0.05, tau=0.0))
    assert abs(np.sum(g + nu) - 1.0) < 1e-13          # sum_j (grad_j + nu_j) = mass of the source


def _solver(src, y, nu, dim, prm):
    from semidiscreteot_b200 import SotSolver
    s = SotSolver(dim=dim, device=0, precision="fp64")
    s.setup_source(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"])
    s.setup_target(y, nu)
    s.configure(prm)
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("dim,lse,tau", [(2, True, 0.0), (2, False, 1e-8), (3, True, 0.0), (3, False, 1e-12)])
def test_simplex_evaluation_matches_oracle(oracle_mod, dim, lse, tau):
    from semidiscreteot_b200 import SolverParameters
    rng = np.random.default_rng(30 + dim)
    if dim == 2:
        V, T = triangle_square_mesh(14)
        src = simplex_source(V, T, lambda P: 0.5 + np.exp(-np.sum((P - 0.3) ** 2, axis=1) / 0.05), order=3)
        y, eps = rng.random((400, 2)), 5e-3
    else:
        V, T = tetra_cube_mesh(5)
        src = simplex_source(V, T, lambda P: 1.0 + 0.5 * P[:, 2], order=3)
        y, eps = rng.uniform(-1, 1, (300, 3)), 1e-2
    nu = rng.dirichlet(np.ones(len(y)) * 2)
    prm = SolverParameters(epsilon=eps, tau=tau, use_log_sum_exp_trick=lse)
    s = _solver(src, y, nu, dim, prm)
    P = oracle_mod.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"], y, nu)
    op = oracle_mod.Params(epsilon=eps, tau=tau, use_log_sum_exp=lse)
    for k in range(2):
        psi = 0.3 * eps * rng.standard_normal(len(y))
        g = np.zeros(len(y))
        J = s.evaluate_functional(psi, g)
        Jo, go, st = P.evaluate(psi, op)
        assert abs(J - Jo) <= 1e-10 * abs(Jo), (J, Jo)
        assert np.max(np.abs(g - go)) <= 1e-8
        assert s.get_last_distance_threshold() == st["threshold"]
    s.close()


@pytest.mark.gpu
def test_tutorial0_settings_solve(oracle_mod):
    """tutorial_0's solver settings on a 6^3-cube tet mesh of [-1, 1]^3 (5,184
    cells x 10 points) with 400 seeded targets of equal weight: both solvers
    reach the l1 tolerance 1e-2 and each solution meets it under the other."""
    from semidiscreteot_b200 import SolverParameters
    V, T = tetra_cube_mesh(6)
    src = simplex_source(V, T, None, order=3)
    rng = np.random.default_rng(4)
    y = rng.uniform(-0.9, 0.9, (400, 3))
    nu = np.full(400, 1.0 / 400)
    prm = SolverParameters(epsilon=1e-2, tau=1e-12, use_log_sum_exp_trick=False, tolerance=1e-2,
                           distance_threshold_type="pointwise")
    s = _solver(src, y, nu, 3, prm)
    psi = s.solve(np.zeros(400), prm)
    assert s.get_convergence_status()
    P = oracle_mod.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"], y, nu)
    op = oracle_mod.Params(epsilon=1e-2, tau=1e-12, use_log_sum_exp=False, tolerance=1e-2)
    psio, info = P.solve(np.zeros(400), op)
    assert info["converged"]
    P.reset_state()
    _, go, _ = P.evaluate(psi, op)
    assert np.sum(np.abs(go)) <= 1e-2
    g = np.zeros(400)
    s.evaluate_functional(psio, g)
    assert np.sum(np.abs(g)) <= 1e-2
    s.close()


def test_nearest_vertex_density():
    from semidiscreteot_b200.multilevel import nearest_vertex_density
    Vf, _ = tetra_cube_mesh(4)
    Vc, _ = tetra_cube_mesh(2)
    f = 1.0 + Vf[:, 0] ** 2
    got = nearest_vertex_density(Vf, f, Vc)
    np.testing.assert_array_equal(got, 1.0 + Vc[:, 0] ** 2)   # coarse vertices are fine vertices


@pytest.mark.gpu
def test_source_multilevel(oracle_mod):
    """Three tet levels of [-1, 1]^3 (2, 4 and 6 cubes per side) against 250
    targets, epsilon scaling spread over the levels: the finest level's
    potentials meet the tolerance under the oracle and agree with a direct
    solve on the finest source up to the constant shift."""
    from semidiscreteot_b200 import SolverParameters, SotSolver, distribute_epsilon_values, epsilon_sequence
    from semidiscreteot_b200.multilevel import run_source_multilevel
    dens = lambda P: 1.0 + 0.5 * np.sin(2 * P[:, 0]) * P[:, 1]   # noqa: E731
    levels = [simplex_source(*tetra_cube_mesh(n), dens, order=3) for n in (2, 4, 6)]
    rng = np.random.default_rng(12)
    y = rng.uniform(-0.9, 0.9, (250, 3))
    nu = np.full(250, 1.0 / 250)
    prm = SolverParameters(epsilon=2e-2, tau=0.0, use_log_sum_exp_trick=True, tolerance=1e-8,
                           solver_control_type="linf", max_iterations=3000)
    dist = distribute_epsilon_values(epsilon_sequence(2e-2, 2.0, 3), 3)
    s = SotSolver(dim=3, device=0, precision="fp64")
    res = run_source_multilevel(s, levels, y, nu, prm, epsilon_distribution=dist)
    assert [r["level"] for r in res] == [2, 1, 0] and all(r["converged"] for r in res)
    psi = res[-1]["potentials"]
    fine = levels[-1]
    P = oracle_mod.Problem(fine["x"], fine["jxw"], fine["density"], fine["cell_offsets"], fine["cell_centers"], y, nu)
    _, go, _ = P.evaluate(psi, oracle_mod.Params(epsilon=dist[-1][-1], tau=0.0, use_log_sum_exp=True))
    assert np.max(np.abs(go)) <= 1.5e-8
    s2 = SotSolver(dim=3, device=0, precision="fp64")
    s2.setup_source(fine["x"], fine["jxw"], fine["density"], fine["cell_offsets"], fine["cell_centers"])
    s2.setup_target(y, nu)
    import dataclasses
    direct = s2.solve(np.zeros(250), dataclasses.replace(prm, epsilon=dist[-1][-1]))
    d = (psi - psi.mean()) - (direct - direct.mean())
    assert np.max(np.abs(d)) <= 1e-5
    s.close()
    s2.close()
