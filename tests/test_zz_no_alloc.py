"""sdot_evaluate_device_noalloc against sdot_evaluate_device.

The no-allocation entry point keeps its scratch in a static device array (one
per device, SDOT_NOALLOC_SCRATCH_BYTES) and must give the results of the
allocating entry point bit for bit (same kernels, same launch shapes), on two
calls in a row, without changing the device's free memory after its first
(set-up) call.  Oversize and truncated requests are rejected with SDOT_EINVAL.
The file name sorts last so that the test also runs after every other test of
the session; it passes alone as well.
"""
import numpy as np
import pytest

from semidiscreteot_b200 import SolverParameters, SotSolver, structured_source
from semidiscreteot_b200._lib import NOALLOC_SCRATCH_BYTES, SdotError

pytestmark = pytest.mark.gpu


def problem(dim, seed):
    rng = np.random.default_rng(seed)
    if dim == 2:
        src = structured_source(2, 16, 3, nodal_density=lambda p: 1.0 + np.cos(2 * p[:, 0]) ** 2)
        N, eps = 600, 2e-2
    else:
        src = structured_source(3, 8, 2)
        N, eps = 500, 1e-2
    y = rng.random((N, dim))
    nu = rng.dirichlet(np.ones(N) * 5)
    return src, y, nu, eps


def make(src, y, nu, eps, precision, tau=0.0):
    s = SotSolver(dim=y.shape[1], device=0, precision=precision)
    s.setup_source(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"])
    s.setup_target(y, nu)
    s.configure(SolverParameters(epsilon=eps, tau=tau, use_log_sum_exp_trick=True))
    return s


@pytest.mark.parametrize("precision", ["fp64", "hybrid"])
@pytest.mark.parametrize("dim", [2, 3])
def test_noalloc_matches_allocating_entry_point(dim, precision):
    import torch
    src, y, nu, eps = problem(dim, seed=11 + dim)
    N = len(nu)
    rng = np.random.default_rng(3)
    psis = [torch.tensor(0.3 * eps * rng.standard_normal(N), dtype=torch.float64, device="cuda") for _ in range(2)]
    ref = make(src, y, nu, eps, precision)
    want = []
    for psi in psis:
        g = torch.empty(N, dtype=torch.float64, device="cuda")
        J = ref.evaluate_functional_device(psi.data_ptr(), g.data_ptr())
        torch.cuda.synchronize()
        want.append((J, g.cpu().numpy(), ref.get_C_global()))
    ref.close()

    s = make(src, y, nu, eps, precision)
    got = []
    for psi in psis:  # two calls in a row on the no-allocation path
        g = torch.full((N,), np.nan, dtype=torch.float64, device="cuda")
        J = s.evaluate_functional_device_noalloc(psi.data_ptr(), g.data_ptr())
        torch.cuda.synchronize()
        got.append((J, g.cpu().numpy(), s.get_C_global()))
    for (Jw, gw, Cw), (Jg, gg, Cg) in zip(want, got):
        assert Jg == Jw
        assert np.array_equal(gg, gw)
        assert Cg == Cw
    assert s.get_last_distance_threshold() == np.finfo(np.float64).max
    s.close()


def test_noalloc_allocates_nothing_after_setup():
    import torch
    src, y, nu, eps = problem(2, seed=5)
    N = len(nu)
    s = make(src, y, nu, eps, "hybrid")
    psi = torch.zeros(N, dtype=torch.float64, device="cuda")
    g = torch.empty(N, dtype=torch.float64, device="cuda")
    J0 = s.evaluate_functional_device_noalloc(psi.data_ptr(), g.data_ptr())  # first call: one-time set-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        J = s.evaluate_functional_device_noalloc(psi.data_ptr(), g.data_ptr())
        assert J == J0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    s.close()


def test_noalloc_rejects_oversize_and_truncated():
    import torch
    # 256^2 cells x 16 points: the L_q segment alone (8 MiB) exceeds the limit
    src = structured_source(2, 256, 4)
    nq = src["jxw"].size
    assert nq * 8 >= NOALLOC_SCRATCH_BYTES
    rng = np.random.default_rng(1)
    N = 64
    y, nu = rng.random((N, 2)), np.full(N, 1.0 / N)
    psi = torch.zeros(N, dtype=torch.float64, device="cuda")
    g = torch.empty(N, dtype=torch.float64, device="cuda")
    s = make(src, y, nu, 1e-2, "hybrid")
    with pytest.raises(SdotError) as ei:
        s.evaluate_functional_device_noalloc(psi.data_ptr(), g.data_ptr())
    assert ei.value.status == 1 and "static limit" in str(ei.value)
    s.close()
    src2, y2, nu2, eps2 = problem(2, seed=2)
    s = make(src2, y2, nu2, eps2, "hybrid", tau=1e-8)
    psi2 = torch.zeros(len(nu2), dtype=torch.float64, device="cuda")
    g2 = torch.empty(len(nu2), dtype=torch.float64, device="cuda")
    with pytest.raises(SdotError) as ei:
        s.evaluate_functional_device_noalloc(psi2.data_ptr(), g2.data_ptr())
    assert ei.value.status == 1 and "untruncated" in str(ei.value)
    s.close()
