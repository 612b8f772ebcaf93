"""Tensor-core Hessian (tcgen05, BF16 hi+lo, FP64 drains) against FP64.

The tensor method computes the same matrix as the FP64 Hessian (the
declared-only SotSolver::compute_hessian, SotSolver.h:343-344) with BF16
hi+lo operands (three products, lo*lo dropped) and FP32 exponentials, so it is
compared with a relative bound: Frobenius error <= 1e-5 of ||H||_F and every
entry within 2e-5 of max|H| (measured 2e-7 to 1.6e-6 on B200).  It must be
exactly symmetric and bitwise repeatable.
Sizes are chosen so that n_targets is not a multiple of the 128 x 256 tile and
the point count is not a multiple of the 64-point stage.
"""
import numpy as np
import pytest

from semidiscreteot_b200 import SolverParameters, SotSolver, structured_source

pytestmark = pytest.mark.gpu

FRO_TOL = 1e-5
MAX_TOL = 2e-5


def problem(kind, seed=0):
    rng = np.random.default_rng(seed)
    if kind == "dense2d":
        src = structured_source(2, 15, 3, nodal_density=lambda p: 1.0 + np.cos(2 * p[:, 0]) ** 2)  # 2025 points
        N, eps = 300, 2e-2
        y = rng.random((N, 2))
        nu = rng.dirichlet(np.ones(N) * 5)
    elif kind == "dense3d":
        src = structured_source(3, 7, 2)                      # 2744 points
        N, eps = 777, 1e-2
        y = rng.random((N, 3))
        nu = np.full(N, 1.0 / N)
    elif kind == "dense3d_small_eps":
        def dens(p):
            return np.exp(-np.sum((p - 0.4) ** 2, axis=1) / (2 * 0.2 ** 2)) + 0.2
        src = structured_source(3, 9, 2, nodal_density=dens)  # 5832 points
        N, eps = 640, 5e-3
        y = np.clip(0.5 + 0.25 * rng.standard_normal((N, 3)), 0, 1)
        nu = rng.dirichlet(np.ones(N) * 3)
    else:
        raise KeyError(kind)
    return src, y, nu, eps


def make(src, y, nu, eps, tau=0.0):
    s = SotSolver(dim=y.shape[1], device=0, precision="fp64")
    s.setup_source(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"])
    s.setup_target(y, nu)
    s.configure(SolverParameters(epsilon=eps, tau=tau, use_log_sum_exp_trick=True))
    return s


def rel_errors(H, Href):
    d = H - Href
    return float(np.linalg.norm(d) / np.linalg.norm(Href)), float(np.max(np.abs(d)) / np.max(np.abs(Href)))


def hessian(s, psi, method, out_f32=False):
    import torch
    n = psi.size
    p = torch.tensor(psi, dtype=torch.float64, device="cuda")
    H = torch.full((n, n), float("nan"), dtype=torch.float32 if out_f32 else torch.float64, device="cuda")
    info = s.compute_hessian_device(p.data_ptr(), H.data_ptr(), method=method, out_f32=out_f32)
    torch.cuda.synchronize()
    return H.cpu().numpy().astype(np.float64), info


@pytest.mark.parametrize("kind", ["dense2d", "dense3d", "dense3d_small_eps"])
def test_tensor_hessian_matches_oracle(oracle_mod, kind):
    src, y, nu, eps = problem(kind)
    N = len(nu)
    s = make(src, y, nu, eps)
    psi = 0.3 * eps * np.random.default_rng(1).standard_normal(N)
    Ht, info = hessian(s, psi, "tensor")
    assert info["method"] == "tensor"
    assert np.all(np.isfinite(Ht))
    assert np.array_equal(Ht, Ht.T)
    P = oracle_mod.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"], y, nu)
    op = oracle_mod.Params(epsilon=eps, tau=0.0, use_log_sum_exp=True)
    Ho = P.hessian(psi, op, 1e300)
    fro, mx = rel_errors(Ht, Ho)
    print(f"{kind}: tensor Hessian vs FP64 oracle: Frobenius {fro:.2e}, max {mx:.2e}")
    assert fro <= FRO_TOL and mx <= MAX_TOL
    # the FP64 method on the device agrees with the oracle to 1e-9
    Hf, info64 = hessian(s, psi, "fp64")
    assert info64["method"] == "fp64"
    assert np.max(np.abs(Hf - Ho)) <= 1e-9 * np.max(np.abs(Ho))
    # FP32 output: the same matrix rounded once
    H32, _ = hessian(s, psi, "tensor", out_f32=True)
    assert np.max(np.abs(H32 - Ht)) <= 1e-6 * np.max(np.abs(Ht))
    s.close()


def test_tensor_hessian_chunking_and_repeatability():
    src, y, nu, eps = problem("dense3d", seed=3)
    s = make(src, y, nu, eps)
    N = len(nu)
    psi = 0.2 * eps * np.random.default_rng(2).standard_normal(N)
    Hf, _ = hessian(s, psi, "fp64")
    errs = {}
    for ch in (1, 4, 16, 1000):
        s.set_hessian_chunk(ch)
        Ha, _ = hessian(s, psi, "tensor")
        Hb, _ = hessian(s, psi, "tensor")
        assert np.array_equal(Ha, Hb)   # deterministic: no atomics, fixed order
        errs[ch] = rel_errors(Ha, Hf)
        assert errs[ch][0] <= FRO_TOL and errs[ch][1] <= MAX_TOL, (ch, errs[ch])
    print("chunk -> (Frobenius, max) relative error:", errs)
    s.close()


def test_tensor_hessian_larger_against_fp64_kernel():
    # 16^3 x 8 = 32768 points, 2000 targets: several tiles in both directions
    rng = np.random.default_rng(7)
    src = structured_source(3, 16, 2)
    N, eps = 2000, 5e-3
    y = rng.random((N, 3))
    nu = np.full(N, 1.0 / N)
    s = make(src, y, nu, eps)
    psi = 0.2 * eps * rng.standard_normal(N)
    Hf, _ = hessian(s, psi, "fp64")
    Ht, info = hessian(s, psi, "tensor")
    fro, mx = rel_errors(Ht, Hf)
    print(f"2000 targets: Frobenius {fro:.2e}, max {mx:.2e}, tiles {info['tiles']}")
    assert fro <= FRO_TOL and mx <= MAX_TOL
    # SM pairs (the default): 256 x 256 tiles of the upper triangle, 8 x 9 / 2
    assert s.set_hessian_pairs(None) == 2 and info["tiles"] == 36
    s.set_hessian_pairs(0)
    Hs, info = hessian(s, psi, "tensor")
    assert info["tiles"] == sum(max(0, 8 - (ta * 128) // 256) for ta in range(16))   # single SMs: 128 x 256
    assert rel_errors(Hs, Hf)[0] <= FRO_TOL
    s.set_hessian_pairs(2)
    # rows sum to ~0: H 1 = 0 for the exact Hessian (mass conservation)
    assert np.max(np.abs(Ht.sum(axis=1))) <= 1e-3 * np.max(np.abs(Ht))
    s.close()


def test_tensor_hessian_rejects_truncated():
    src, y, nu, eps = problem("dense2d")
    s = make(src, y, nu, 5e-3, tau=1e-8)
    psi = np.zeros(len(nu))
    with pytest.raises(RuntimeError, match="untruncated"):
        hessian(s, psi, "tensor")
    _, info = hessian(s, psi, "auto")
    assert info["method"] == "fp64"
    s.close()


def test_wait_timeout_reports_and_recovers():
    """The tensor Hessian's device-side waits are bounded.  With a bound far
    below the latency of one stage's tensor-core products (12 MMAs of
    128 x 256 x 16, some 1,600 SM cycles), the wait for the last chunk's
    accumulator expires: the kernel stops, waits (with the default bound) for
    the products in flight, releases its tensor memory and reports
    SDOT_ETIMEOUT.  The context stays usable: with the default bound restored,
    the next Hessian equals one computed before the timeout, bit for bit."""
    from semidiscreteot_b200 import _lib
    src, y, nu, eps = problem("dense3d", seed=5)
    s = make(src, y, nu, eps)
    N = len(nu)
    psi = 0.2 * eps * np.random.default_rng(4).standard_normal(N)
    H0, _ = hessian(s, psi, "tensor")
    s.set_hessian_wait_limit(100)
    with pytest.raises(_lib.SdotError) as ei:
        hessian(s, psi, "tensor")
    assert ei.value.status == _lib.SDOT_ETIMEOUT
    s.set_hessian_wait_limit(0)
    H1, _ = hessian(s, psi, "tensor")
    assert np.array_equal(H0, H1)
    # evaluations on the same context are unaffected
    g = np.zeros(N)
    s.evaluate_functional(psi, g)
    assert np.all(np.isfinite(g))
    s.close()



def test_factored_generation_matches_per_point(oracle_mod):
    """On 2 x 2 x 2 Gauss cells the tensor Hessian's operands are generated
    per cell (one ex2 for the cell and one per dimension, the 8 values by
    products); the result agrees with the per-point generation and with the
    FP64 oracle within the tensor method's bounds.  11^3 cells (10,648 points,
    not a multiple of the 64-point stage), 501 targets, eps = 1.5e-2: the
    per-dimension factors stay within 2^9."""
    rng = np.random.default_rng(2)

    def dens(p):
        return np.exp(-np.sum((p - 0.3) ** 2, axis=1) / (2 * 0.15 ** 2)) + 0.05

    src = structured_source(3, 11, 2, nodal_density=dens)
    N, eps = 501, 1.5e-2
    y = rng.random((N, 3))
    nu = rng.dirichlet(np.ones(N) * 4)
    s = make(src, y, nu, eps)
    psi = 0.2 * eps * rng.standard_normal(N)
    Hf, _ = hessian(s, psi, "tensor")
    assert s.set_hessian_generation(None) is True
    s.set_hessian_generation(False)
    Hp, _ = hessian(s, psi, "tensor")
    assert s.set_hessian_generation(None) is False
    s.set_hessian_generation(True)
    P = oracle_mod.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"], y, nu)
    Ho = P.hessian(psi, oracle_mod.Params(epsilon=eps, tau=0.0, use_log_sum_exp=True), 1e300)
    for H in (Hf, Hp):
        fro, mx = rel_errors(H, Ho)
        print(f"tensor Hessian vs FP64: Frobenius {fro:.2e}, max {mx:.2e}")
        assert fro <= FRO_TOL and mx <= MAX_TOL, (fro, mx)
        assert np.array_equal(H, H.T)
    Hf2, _ = hessian(s, psi, "tensor")
    assert np.array_equal(Hf, Hf2)
    s.close()


def test_factored_generation_not_used_outside_its_bound():
    """9^3 cells at eps = 5e-3: a per-dimension factor could reach 2^32, so
    the per-point generation runs even though the cells are Gauss grids."""
    src, y, nu, eps = problem("dense3d_small_eps", seed=2)
    s = make(src, y, nu, eps)
    psi = np.zeros(len(nu))
    hessian(s, psi, "tensor")
    assert s.set_hessian_generation(None) is False
    s.close()


@pytest.mark.parametrize("kind", ["dense2d", "dense3d", "dense3d_small_eps"])
def test_sm_pairs_match_single_sm(oracle_mod, kind):
    """Whole Hessians on SM pairs (tcgen05 cta_group::2 over 256 x 256 tiles),
    with two generation groups (the default) or one, agree with the FP64
    oracle within the tensor method's bounds, are exactly symmetric and
    repeatable, and agree with the single-SM kernel."""
    src, y, nu, eps = problem(kind, seed=4)
    N = len(nu)
    s = make(src, y, nu, eps)
    psi = 0.3 * eps * np.random.default_rng(8).standard_normal(N)
    H2, _ = hessian(s, psi, "tensor")          # SM pairs, two generation groups: the default
    assert s.set_hessian_pairs(None) == 2
    H3, _ = hessian(s, psi, "tensor")
    s.set_hessian_pairs(1)
    H1p, _ = hessian(s, psi, "tensor")         # SM pairs, one generation group
    assert s.set_hessian_pairs(None) == 1
    s.set_hessian_pairs(0)
    H1, _ = hessian(s, psi, "tensor")          # single SMs
    assert s.set_hessian_pairs(None) == 0
    s.set_hessian_pairs(2)
    P = oracle_mod.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"], y, nu)
    Ho = P.hessian(psi, oracle_mod.Params(epsilon=eps, tau=0.0, use_log_sum_exp=True), 1e300)
    assert np.all(np.isfinite(H2))
    assert np.array_equal(H2, H2.T)
    assert np.array_equal(H2, H3)
    fro, mx = rel_errors(H2, Ho)
    print(f"SM pairs vs FP64: Frobenius {fro:.2e}, max {mx:.2e}; single SM: {rel_errors(H1, Ho)}")
    assert fro <= FRO_TOL and mx <= MAX_TOL, (fro, mx)
    for Hx in (H1, H1p):
        assert rel_errors(Hx, Ho)[0] <= FRO_TOL
        assert rel_errors(H2, Hx)[0] <= FRO_TOL
    assert np.array_equal(H1p, H1p.T)
    s.close()
