"""Generate the golden fixtures of tests/golden/ from the FP64 CPU oracle.

The reference (SemiDiscreteOT) ships no golden vectors and cannot be built
here, so these fixtures freeze the oracle's outputs on small seeded inputs.
They pin the oracle against later changes (tests/test_golden.py, CPU) and give
the CUDA path fixed targets that need no oracle at run time (GPU).

Each case stores its inputs (flattened source in the save_discrete_measures
layout, targets, weights, potential) and the outputs: J, gradient, C_global,
pair count and radius of each of three evaluations in a row; the potential,
iteration count and status of a solve; a dense Hessian; the covering radius.

Run:  python tests/golden/make_golden.py     (rewrites tests/golden/*.npz)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as orc  # noqa: E402


def source(dim, n, order, seed, bumpy):
    rng = np.random.default_rng(seed)
    nodal = None
    if bumpy:
        nv = (n + 1) ** dim
        nodal = 0.5 + rng.random(nv)
    x, jxw, rho, off, ctr = orc.structured_source(dim, n, 0.0, 1.0, order, nodal, True)
    return x, jxw, rho, off, ctr


CASES = {
    # name: (dim, cells per axis, Gauss order, N, eps, tau, lse, threshold type, seed)
    "dense2d_o3": (2, 8, 3, 40, 2e-2, 0.0, True, "pointwise", 1),
    "dense2d_nolse": (2, 8, 2, 50, 5e-2, 0.0, False, "pointwise", 2),
    "trunc2d_o2": (2, 12, 2, 60, 5e-3, 1e-8, True, "pointwise", 3),
    "trunc3d_o2": (3, 6, 2, 80, 4e-3, 1e-10, True, "pointwise", 4),
    "trunc3d_o3": (3, 4, 3, 50, 1e-2, 1e-9, False, "pointwise", 5),
    "integral2d": (2, 10, 2, 40, 1e-2, 1e-8, True, "integral", 6),
    "geometric3d": (3, 5, 2, 40, 1e-2, 1e-8, True, "geometric", 7),
}


def make(name, spec):
    dim, n, order, N, eps, tau, lse, ttype, seed = spec
    x, jxw, rho, off, ctr = source(dim, n, order, seed, bumpy=(seed % 2 == 1))
    rng = np.random.default_rng(100 + seed)
    y = rng.random((N, dim))
    nu = rng.dirichlet(np.ones(N) * 4)
    psi1 = eps * rng.standard_normal(N)
    psi2 = psi1 + 0.5 * eps * rng.standard_normal(N)
    P = orc.Problem(x, jxw, rho, off, ctr, y, nu)
    prm = orc.Params(epsilon=eps, tau=tau, use_log_sum_exp=lse, distance_threshold_type=ttype)
    out = {}
    # three evaluations in a row: a pointwise one at psi1 (it sets the state
    # J, C_global that the integral / geometric radii read), then the case's
    # threshold type at psi1 and psi2
    pw = orc.Params(epsilon=eps, tau=tau, use_log_sum_exp=lse)
    for k, (psi, pk) in enumerate(((psi1, pw), (psi1, prm), (psi2, prm))):
        J, g, st = P.evaluate(psi, pk)
        out[f"J{k}"] = np.float64(J)
        out[f"g{k}"] = g
        out[f"C{k}"] = np.float64(st["C_global"])
        out[f"pairs{k}"] = np.int64(st["n_pairs"])
        out[f"r{k}"] = np.float64(st["threshold"])
    out["covering_radius"] = np.float64(P.covering_radius())
    # Hessian at psi1 with the pointwise radius of psi1
    P.reset_state()
    pp = orc.Params(epsilon=eps, tau=tau, use_log_sum_exp=lse)
    r1 = P.distance_threshold(psi1, pp)
    out["H"] = P.hessian(psi1, pp, r1)
    out["H_r"] = np.float64(r1)
    # solve from zero to |g|_inf <= 1e-8; truncated cases solve with tau = 1e-14
    # (a coarser truncation makes the functional too rough for the line search
    # at this tolerance, in the reference's arithmetic as well)
    P.reset_state()
    sp = orc.Params(epsilon=eps, tau=min(tau, 1e-14) if tau > 0 else 0.0, use_log_sum_exp=lse,
                    solver_control_type="linf", tolerance=1e-8, max_iterations=2000)
    psi_s, info = P.solve(np.zeros(N), sp)
    out["solve_psi"] = psi_s
    out["solve_iterations"] = np.int64(info["iterations"])
    out["solve_converged"] = np.int64(info["converged"])
    out["solve_status"] = np.int64(info["status"])
    meta = np.array([dim, n, order, N, eps, tau, float(lse), seed], dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), x=x, jxw=jxw, rho=rho, cell_offsets=off,
                        cell_centers=ctr, y=y, nu=nu, psi1=psi1, psi2=psi2, meta=meta,
                        threshold_type=np.array(ttype), **out)
    return out


def main():
    orc.build()
    for name, spec in CASES.items():
        o = make(name, spec)
        print(f"{name}: J0={o['J0']:.15g} pairs0={int(o['pairs0'])} r0={o['r0']:.6g} "
              f"solve_it={int(o['solve_iterations'])} converged={int(o['solve_converged'])}")


if __name__ == "__main__":
    main()
