"""Multi-GPU evaluation: source cells sharded across ranks, targets replicated.

Replaces the MPI layer of ``SotSolver::evaluate_functional``: the reference's
ranks own cells of a distributed triangulation and sum value, gradient and
C_global with ``Utilities::MPI::sum`` (src/solvers/SotSolver.cc:316-319), then
rank 0 subtracts the linear term (:322-327) and broadcasts (:330-331).  Here
each rank (one process per GPU) evaluates its contiguous range of cells
(``sdot_evaluate_partial_device``), the (n_targets + 3)-double partial vector
is all-reduced once (NCCL over NVLink on GPUs, gloo on CPU), and every rank
finishes identically (no broadcast needed: the all-reduce already
replicates).  The truncation radius depends only on the replicated psi, so no
further collective is needed; the covering radius is a max-reduction.

The Newton solve shards differently: every rank holds all points and
targets, the (cheap) evaluation is replicated, and the tensor-core Hessian is
split by its 128 x 256 output tiles (``tile_range``, ``hessian_tile_mask``).
Each rank keeps its tiles (and their mirrors) in a zeroed n x n matrix, so its
matrix-vector product is its share of H x: one all-reduce per CG step gives
the product, one more the Jacobi diagonal (``sharded_newton``,
``ShardedHessianNewton``).  The reference declares the Hessian without
implementing it (SotSolver.h:343-344).
"""
from __future__ import annotations

from typing import Callable, Optional

import numpy as np


def shard_range(n: int, rank: int, world: int):
    """Contiguous [begin, end) of n items for rank of world."""
    return (n * rank) // world, (n * (rank + 1)) // world


def shard_source(src: dict, rank: int, world: int) -> dict:
    """Cells [c0, c1) of a flattened source and their quadrature points."""
    off = np.asarray(src["cell_offsets"])
    ncell = off.size - 1
    c0, c1 = shard_range(ncell, rank, world)
    q0, q1 = int(off[c0]), int(off[c1])
    dim = np.asarray(src["cell_centers"]).reshape(ncell, -1).shape[1]
    return {
        "x": np.asarray(src["x"]).reshape(-1, dim)[q0:q1],
        "jxw": np.asarray(src["jxw"])[q0:q1],
        "density": np.asarray(src["density"])[q0:q1],
        "cell_offsets": off[c0:c1 + 1] - off[c0],
        "cell_centers": np.asarray(src["cell_centers"]).reshape(ncell, dim)[c0:c1],
    }


def finish(reduced, psi, nu):
    """From the all-reduced partial vector [grad_src(N), J_src, C, pairs] to
    (J, grad, C, pairs): g_j = grad_src_j - nu_j, J = J_src - sum psi_j nu_j."""
    n = nu.shape[0]
    g = reduced[:n] - nu
    J = reduced[n] - (psi * nu).sum()
    return J, g, reduced[n + 1], reduced[n + 2]


class DistributedSotSolver:
    """One rank of a source-sharded evaluation.

    ``partial_fn(psi) -> out`` computes this rank's (N+3) partial vector; by
    default the GPU library (``SotSolver.evaluate_partial_device``) on this
    rank's shard.  ``all_reduce(t)`` sums a tensor over the ranks in place
    (default ``torch.distributed.all_reduce``)."""

    def __init__(self, dim: int, rank: int, world: int, device: Optional[int] = None, precision: str = "hybrid",
                 partial_fn: Optional[Callable] = None, all_reduce: Optional[Callable] = None):
        self.dim, self.rank, self.world = dim, rank, world
        self.device = device
        self.precision = precision
        self._partial_fn = partial_fn
        self._all_reduce = all_reduce
        self.local = None
        if partial_fn is None:
            from .solver import SotSolver
            self.local = SotSolver(dim=dim, device=device if device is not None else 0, precision=precision)

    def setup_source(self, src: dict):
        self.shard = shard_source(src, self.rank, self.world)
        if self.local is not None:
            self.local.setup_source_measure(self.shard)

    def setup_target(self, y, nu):
        self.nu_np = np.ascontiguousarray(nu, dtype=np.float64)
        if self.local is not None:
            self.local.setup_target(y, nu)

    def configure(self, params):
        self.params = params
        if self.local is not None:
            self.local.configure(params)

    def _reduce(self, t):
        if self._all_reduce is not None:
            self._all_reduce(t)
        else:
            import torch.distributed as dist
            dist.all_reduce(t)

    def evaluate(self, psi):
        """psi: torch tensor (float64) on this rank's device (or CPU with a
        custom partial_fn).  Returns (J, grad tensor, C_global, pairs)."""
        import torch
        n = psi.numel()
        if self._partial_fn is not None:
            out = self._partial_fn(psi)
        else:
            out = torch.empty(n + 3, dtype=torch.float64, device=psi.device)
            self.local.evaluate_partial_device(psi.data_ptr(), out.data_ptr())
        self._reduce(out)
        nu = torch.as_tensor(self.nu_np, device=out.device)
        J, g, C, pairs = finish(out, psi, nu)
        J, C, pairs = float(J), float(C), float(pairs)
        if self.local is not None:
            self.local.set_state(J, C)
        return J, g, C, pairs

    def close(self):
        if self.local is not None:
            self.local.close()
            self.local = None


# ---------------------------------------------------------------------------
# Newton with the Hessian sharded by output tiles
# ---------------------------------------------------------------------------

HT_M, HT_N = 128, 256  # tile rows x columns of the tensor-core Hessian


def hessian_tiles(n: int):
    """The upper-triangle tiles (row tile, column tile) in the library's order:
    row tiles of 128, column tiles of 256 from the one holding the row tile's
    first row (sdot_hessian_tile_count gives their number)."""
    na, nb = -(-n // HT_M), -(-n // HT_N)
    return [(ta, tb) for ta in range(na) for tb in range((ta * HT_M) // HT_N, nb)]


def tile_range(n_tiles: int, rank: int, world: int):
    """Contiguous, balanced share [begin, end) of the tiles (all cost the same)."""
    return shard_range(n_tiles, rank, world)


def hessian_tile_mask(n: int, t0: int, t1: int) -> np.ndarray:
    """Entries of an n x n Hessian written for tiles [t0, t1): (a, b) with
    a <= b in those tiles, and their mirrors (b, a)."""
    m = np.zeros((n, n), dtype=bool)
    for ta, tb in hessian_tiles(n)[t0:t1]:
        r0, r1 = ta * HT_M, min(n, ta * HT_M + HT_M)
        c0, c1 = tb * HT_N, min(n, tb * HT_N + HT_N)
        a = np.arange(r0, r1)[:, None]
        b = np.arange(c0, c1)[None, :]
        up = b >= a
        blk = m[r0:r1, c0:c1]
        blk |= up
        m[c0:c1, r0:r1] |= up.T
    return m


def control_value(g: np.ndarray, control: str) -> float:
    if control == "linf":
        return float(np.max(np.abs(g)))
    if control == "l1norm":
        return float(np.sum(np.abs(g)))
    raise ValueError(f"sharded Newton supports l1norm and linf controls, not {control}")


def sharded_newton(psi0: np.ndarray, evaluate: Callable, hessian_part: Callable, matvec_part: Callable,
                   diag_part: Callable, all_reduce: Callable, tol: float, control: str = "linf",
                   max_iterations: int = 1000, reuse: float = 0.1, max_halvings: int = 40):
    """Newton on the dual with this rank's share of the Hessian.

    evaluate(psi) -> (J, g) is replicated (every rank gets the same numbers);
    hessian_part(psi) computes this rank's tiles at psi (after the evaluation at
    psi) and returns a handle; matvec_part(h, x) and diag_part(h) return this
    rank's shares of H x and of diag(H); all_reduce(v) returns the sum over
    the ranks.  Steps as sdot_solve_newton: Jacobi-preconditioned CG on
    H d = -g with the constant null vector projected out and the forcing term
    min(0.5, sqrt(|g|_2)), Armijo backtracking on J, the Hessian kept after a
    full step that reduced |g|_2 by `reuse`.  Returns (psi, info)."""
    psi = np.array(psi0, dtype=np.float64)
    n = psi.size
    J, g = evaluate(psi)
    k, n_hess, cg_total, evals = 0, 0, 0, 1
    h, D = None, None
    g2_prev, alpha_prev = 0.0, 0.0
    check = control_value(g, control)
    while check > tol and k < max_iterations:
        g2 = float(np.sqrt(g @ g))
        if not (h is not None and reuse > 0.0 and alpha_prev == 1.0 and g2 <= reuse * g2_prev):
            h = hessian_part(psi)
            D = all_reduce(np.asarray(diag_part(h), dtype=np.float64))
            D = np.where(D > 0.0, D, 1.0)
            n_hess += 1
        g2_prev = g2
        eta = max(1e-10, min(0.5, np.sqrt(g2)))
        b = -(g - g.mean())
        x = np.zeros(n)
        r = b.copy()
        z = r / D
        z -= z.mean()
        p = z.copy()
        rz = r @ z
        bn = np.sqrt(b @ b)
        for it in range(4 * min(n, 2500)):
            if np.sqrt(r @ r) <= eta * bn:
                break
            Ap = all_reduce(np.asarray(matvec_part(h, p), dtype=np.float64))
            pAp = p @ Ap
            if not pAp > 0.0:
                break
            a = rz / pAp
            x += a * p
            r -= a * Ap
            r -= r.mean()
            z = r / D
            z -= z.mean()
            rz_new = r @ z
            p = z + (rz_new / rz) * p
            rz = rz_new
            cg_total += 1
        d = x if g @ x < 0.0 else -g
        gp = float(g @ d)
        alpha, accepted = 1.0, False
        for _ in range(max_halvings):
            Jn, gn = evaluate(psi + alpha * d)
            evals += 1
            if np.isfinite(Jn) and Jn <= J + 1e-4 * alpha * gp:
                accepted = True
                break
            alpha *= 0.5
        if not accepted:
            raise RuntimeError("sharded Newton: no sufficient decrease after step halvings")
        psi = psi + alpha * d
        J, g = Jn, gn
        alpha_prev = alpha
        k += 1
        check = control_value(g, control)
    return psi, {"iterations": k, "converged": check <= tol, "n_hessians": n_hess, "cg_iterations": cg_total,
                 "n_evaluations": evals, "last_value": J, "last_check_value": check}


class ShardedHessianNewton:
    """One rank of a Newton solve whose tensor-core Hessian is sharded by tiles.

    ``solver``: a ``SotSolver`` holding all points and targets (set up and
    configured alike on every rank).  ``all_reduce(tensor)`` sums in place
    (default ``torch.distributed.all_reduce``; world 1 needs none)."""

    def __init__(self, solver, rank: int = 0, world: int = 1, all_reduce: Optional[Callable] = None):
        import torch
        self.s, self.rank, self.world = solver, rank, world
        self._all_reduce = all_reduce
        n = solver._n_targets
        self.n = n
        self.t0, self.t1 = tile_range(solver.hessian_tile_count(), rank, world)
        self.dev = torch.device("cuda", solver.device)
        self.H = torch.zeros(n * n, dtype=torch.float32, device=self.dev)  # entries of other tiles stay 0
        self._x = torch.empty(n, dtype=torch.float64, device=self.dev)
        self._y = torch.empty(n, dtype=torch.float64, device=self.dev)
        self._psi = torch.empty(n, dtype=torch.float64, device=self.dev)

    def _reduce(self, v: np.ndarray) -> np.ndarray:
        if self.world == 1:
            return v
        import torch
        t = torch.as_tensor(v, device=self.dev) if self._all_reduce is None else torch.as_tensor(v)
        if self._all_reduce is not None:
            self._all_reduce(t)
        else:
            import torch.distributed as dist
            dist.all_reduce(t)
        return t.cpu().numpy()

    def _evaluate(self, psi):
        g = np.zeros(self.n)
        J = self.s.evaluate_functional(psi, g)
        return J, g

    def _hessian(self, psi):
        import torch
        self._psi.copy_(torch.as_tensor(psi))
        self.info = self.s.compute_hessian_tiles_device(self._psi.data_ptr(), self.H.data_ptr(), self.t0, self.t1)
        return self.H

    def _matvec(self, H, x):
        import torch
        self._x.copy_(torch.as_tensor(x))
        self.s.hessian_matvec_device(H.data_ptr(), self._x.data_ptr(), self._y.data_ptr(), f32=True)
        return self._y.cpu().numpy()

    def _diag(self, H):
        return H.view(self.n, self.n).diagonal().double().cpu().numpy()

    def solve(self, psi0, params):
        self.s.configure(params)
        return sharded_newton(psi0, self._evaluate, self._hessian, self._matvec, self._diag, self._reduce,
                              params.tolerance, params.solver_control_type, params.max_iterations)
