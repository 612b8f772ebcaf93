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
