"""The oracle on the sources of the tensor-grid cell tests (CPU): 2 x 2 Gauss points per cell and cell columns of
different widths, against a brute-force NumPy restatement of the untruncated dual (every point with every target):

    L_q = log sum_j nu_j exp((psi_j - |x_q - y_j|^2 / 2) / eps),
    J = sum_q w_q eps L_q - sum_j psi_j nu_j,
    g_j = sum_q w_q nu_j exp((psi_j - |x_q - y_j|^2 / 2) / eps - L_q) - nu_j,

with w_q = rho_q JxW_q.  Also checks that the graded source keeps every cell a tensor grid symmetric about its
centre while the spacing changes from column to column (the property the dense cell sweeps rely on, and the one the
graded case takes away from the uniform-grid form).
"""
import numpy as np
import pytest

from cell_sources import graded_source
from semidiscreteot_b200 import structured_source


def brute_force(src, y, nu, psi, eps):
    x = src["x"]
    w = src["density"] * src["jxw"]
    c = 0.5 * np.sum((x[:, None, :] - y[None, :, :]) ** 2, axis=2)
    a = (psi[None, :] - c) / eps + np.log(nu)[None, :]
    m = np.max(a, axis=1, keepdims=True)
    L = m[:, 0] + np.log(np.sum(np.exp(a - m), axis=1))
    J = np.sum(w * eps * L) - np.dot(psi, nu)
    g = np.sum(w[:, None] * np.exp(a - L[:, None]), axis=0) - nu
    return J, g


def cases():
    rng = np.random.default_rng(0)
    src_o2 = structured_source(2, 20, 2, nodal_density=lambda p: 1.0 + 0.5 * p[:, 1])
    y = rng.random((300, 2))
    nu = rng.dirichlet(np.ones(300) * 20)
    yield "order2", src_o2, y, nu, 2e-2
    src_gr = graded_source(np.random.default_rng(1), 2, 18, 3)
    y = rng.random((250, 2))
    nu = np.full(250, 1.0 / 250)
    yield "graded", src_gr, y, nu, 2e-2


@pytest.mark.parametrize("lse", [True, False])
def test_oracle_matches_brute_force_on_cell_sources(oracle_mod, lse):
    for name, src, y, nu, eps in cases():
        P = oracle_mod.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"], y, nu)
        psi = 0.05 * eps * np.random.default_rng(2).standard_normal(len(nu))
        op = oracle_mod.Params(epsilon=eps, tau=0.0, use_log_sum_exp=lse)
        J, g, st = P.evaluate(psi, op)
        Jb, gb = brute_force(src, y, nu, psi, eps)
        assert st["n_pairs"] == src["x"].shape[0] * len(nu), name
        assert abs(J - Jb) <= 1e-12 * abs(Jb), name
        assert np.max(np.abs(g - gb)) <= 1e-14, name
        assert abs(np.sum(g + nu) - np.sum(src["density"] * src["jxw"])) <= 1e-13, name


def test_graded_source_cells_are_tensor_grids_with_their_own_spacing():
    n, order, dim = 18, 3, 2
    src = graded_source(np.random.default_rng(1), dim, n, order)
    qpc = order ** dim
    x = src["x"].reshape(-1, qpc, dim)
    c = src["cell_centers"]
    off = x - c[:, None, :]
    # point i = i0 + order * i1: the x offset depends on i0 only, the y offset on i1 only, both symmetric
    ox = off[:, :, 0].reshape(-1, order, order)   # [cell, i1, i0]
    oy = off[:, :, 1].reshape(-1, order, order)
    np.testing.assert_allclose(ox, ox[:, :1, :].repeat(order, axis=1), atol=1e-15)
    np.testing.assert_allclose(oy, oy[:, :, :1].repeat(order, axis=2), atol=1e-15)
    np.testing.assert_allclose(ox[:, 0, :], -ox[:, 0, ::-1], atol=1e-15)
    np.testing.assert_allclose(oy[:, :, 0], -oy[:, ::-1, 0], atol=1e-15)
    # the spacing along x differs between columns; along y it is the same in every cell
    ax = ox[:, 0, -1]
    ay = oy[:, -1, 0]
    assert np.ptp(ax) > 0.1 * np.max(ax)
    assert np.ptp(ay) <= 1e-15
    # the measure still has unit mass on [0, 1]^2
    assert abs(np.sum(src["density"] * src["jxw"]) - 1.0) <= 1e-13
    assert np.all(x[:, :, 0] > 0) and np.all(x[:, :, 0] < 1)
