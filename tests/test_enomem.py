"""Device allocation failures reach the caller as SDOT_ENOMEM.

sdot_debug_fail_allocation(k) makes the k-th following device allocation of
the library fail as if the device were out of memory (host-side: cudaMalloc
is not called, nothing faults).  The GPU test fails, one at a time, every
allocation that a context's set-up and a truncated evaluation make, and
checks that exactly that call returns SDOT_ENOMEM with a message, that the
context then reports the measure as not set (SDOT_ESTATE) instead of running
on missing buffers, and that a fresh context afterwards evaluates correctly.
"""
import numpy as np
import pytest

from semidiscreteot_b200 import SolverParameters, SotSolver, _lib, structured_source


def test_injection_control_without_gpu():
    L = _lib.load()
    assert L.sdot_debug_fail_allocation(-1) == -1          # off by default
    assert L.sdot_debug_fail_allocation(5) == -1
    assert L.sdot_debug_fail_allocation(-7) == 5           # any negative value turns it off
    assert L.sdot_debug_fail_allocation(-1) == -1
    assert L.sdot_debug_allocation_count() >= 0


def _problem():
    rng = np.random.default_rng(3)
    src = structured_source(3, 6, 2, nodal_density=lambda p: 1.0 + p[:, 0])
    N = 300
    y = np.clip(0.5 + 0.2 * rng.standard_normal((N, 3)), 0, 1)
    nu = rng.dirichlet(np.ones(N) * 4)
    prm = SolverParameters(epsilon=5e-3, tau=1e-10, use_log_sum_exp_trick=True)
    psi = 1e-3 * rng.standard_normal(N)
    return src, y, nu, prm, psi


def _run(src, y, nu, prm, psi):
    s = SotSolver(dim=3, device=0, precision="hybrid")
    try:
        s.setup_source_measure(src)
        s.setup_target(y, nu)
        s.configure(prm)
        g = np.zeros(len(nu))
        J = s.evaluate_functional(psi, g)
        return J, g, None, s
    except _lib.SdotError as e:
        return None, None, e, s


@pytest.mark.gpu
def test_every_allocation_failure_is_reported(oracle_mod):
    L = _lib.load()
    src, y, nu, prm, psi = _problem()
    n0 = L.sdot_debug_allocation_count()
    J, g, err, s = _run(src, y, nu, prm, psi)
    s.close()
    assert err is None
    n_alloc = L.sdot_debug_allocation_count() - n0
    assert n_alloc >= 10
    try:
        for k in range(n_alloc):
            L.sdot_debug_fail_allocation(k)
            Jk, gk, err, s = _run(src, y, nu, prm, psi)
            L.sdot_debug_fail_allocation(-1)
            assert err is not None and err.status == _lib.SDOT_ENOMEM, (k, err)
            assert "out of memory" in str(err) or "memory" in str(err)
            # the context never runs on missing buffers: either the failed call
            # left a measure unset (SDOT_ESTATE), or, after a failure inside the
            # evaluation, a new evaluation allocates again and succeeds
            import ctypes as C
            g2 = np.zeros(len(nu))
            val = C.c_double(0.0)
            st = L.sdot_evaluate(s._h, psi.ctypes.data, g2.ctypes.data, C.byref(val), None)
            assert st in (_lib.SDOT_OK, _lib.SDOT_ESTATE), (k, st)
            if st == _lib.SDOT_OK:
                assert abs(val.value - J) <= 1e-12 * abs(J)
                assert np.max(np.abs(g2 - g)) <= 1e-15
            s.close()
    finally:
        L.sdot_debug_fail_allocation(-1)
    # the device is healthy afterwards: a fresh context matches the oracle
    J3, g3, err, s = _run(src, y, nu, prm, psi)
    s.close()
    assert err is None
    P = oracle_mod.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"], y, nu)
    Jo, go, _ = P.evaluate(psi, oracle_mod.Params(epsilon=prm.epsilon, tau=prm.tau, use_log_sum_exp=True))
    assert abs(J3 - Jo) <= 1e-10 * abs(Jo)
    assert np.max(np.abs(g3 - go)) <= 1e-8
