"""CUDA-graph replay of the untruncated evaluation.

An untruncated euclidean evaluation has no host step between its launches,
so the library captures it as one CUDA graph on the second consecutive
evaluation with the same launch key (sizes, parameters, buffer addresses) and
replays the graph afterwards.  These tests check that replays compute
bitwise what an eager evaluation computes, for new potentials, for the FP64
and hybrid sweeps, for the sliced and unsliced dense value sweeps, and after
the parameters change (a new key, so eager evaluations and a new capture);
and that the launch counters count the replayed kernels.
"""
import numpy as np
import pytest

from semidiscreteot_b200 import SolverParameters, SotSolver, structured_source

pytestmark = pytest.mark.gpu


def _problem(cells, nt, seed=0):
    rng = np.random.default_rng(seed)
    src = structured_source(2, cells, 3)
    y = rng.random((nt, 2))
    nu = rng.dirichlet(np.ones(nt) * 3)
    return src, y, nu


def _solver(src, y, nu, precision, eps):
    s = SotSolver(dim=2, device=0, precision=precision)
    s.setup_source(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"])
    s.setup_target(y, nu)
    s.configure(SolverParameters(epsilon=eps, tau=0.0, use_log_sum_exp_trick=True))
    return s


def _eval(s, psi):
    g = np.zeros(psi.size)
    J = s.evaluate_functional(psi, g)
    return J, g, s.get_C_global()


@pytest.mark.parametrize("precision", ["fp64", "hybrid"])
@pytest.mark.parametrize("cells,nt", [(64, 1000), (12, 100)])   # sliced / unsliced dense value sweep
def test_replay_matches_eager(precision, cells, nt):
    src, y, nu = _problem(cells, nt)
    rng = np.random.default_rng(1)
    psis = [0.01 * rng.standard_normal(nt) for _ in range(6)]
    a = _solver(src, y, nu, precision, 1e-2)
    got = [_eval(a, p) for p in psis]          # eager, eager + capture, replays
    for i, p in enumerate(psis):
        b = _solver(src, y, nu, precision, 1e-2)
        ref = _eval(b, p)                       # a fresh context: one eager evaluation
        b.close()
        assert got[i][0] == ref[0] and got[i][2] == ref[2], i
        assert np.array_equal(got[i][1], ref[1]), i
    # new parameters: a new key, so eager again, then a new capture
    a.configure(SolverParameters(epsilon=2e-2, tau=0.0, use_log_sum_exp_trick=True))
    got2 = [_eval(a, psis[0]) for _ in range(4)]
    b = _solver(src, y, nu, precision, 2e-2)
    ref2 = _eval(b, psis[0])
    b.close()
    for r in got2:
        assert r[0] == ref2[0] and np.array_equal(r[1], ref2[1])
    a.close()


def test_replayed_launches_are_counted():
    src, y, nu = _problem(16, 500)
    s = _solver(src, y, nu, "hybrid", 1e-2)
    psi = np.zeros(500)
    s.set_profiling(True)
    s.kernel_times(reset=True)
    _eval(s, psi)
    per_eval = sum(v["launches"] for v in s.kernel_times(reset=True).values())
    s.set_profiling(False)
    assert per_eval > 0
    for _ in range(5):
        _eval(s, psi)
    kt = s.kernel_times(reset=True)
    assert sum(v["launches"] for v in kt.values()) == 5 * per_eval
    s.close()
