"""The multi-GPU data path (source shards + one sum of N + 3 doubles) on one GPU.

A truncated 3D problem of the clustered-mixture kind, at a quarter of the
benchmark's cells per axis (16^3 hex cells x 8 Gauss points = 32,768 points,
1,562 targets, eps = 1e-3, tau = 1e-12), is split into 2 and 4 contiguous
ranges of cells (distributed.shard_source).  Each shard is evaluated by
sdot_evaluate_partial_device in its own context (own stream) on the one GPU;
the (N + 3)-vectors are summed on the host in rank order and finished
(distributed.finish).  That must equal the unsharded sdot_evaluate: pair
count exactly, the gradient to 1e-15 absolute and the value to 1e-13
relative (FP64 sweeps; the shards sum in a different order), and the oracle
to the parity tolerances (value 1e-10 relative, gradient 1e-12 absolute).

DistributedSotSolver, the product class bench.py drives under torchrun, is
run the same way: one instance per rank, each in its own host thread with its
own context, and an all_reduce that sums the ranks' vectors on the host in
rank order (a barrier stands in for the collective).  The ranks' kernels do
not wait on one another: the exchange happens on the host.
"""
import threading

import numpy as np
import pytest
import torch

from semidiscreteot_b200 import SotSolver, workloads
from semidiscreteot_b200.distributed import DistributedSotSolver, finish, shard_source

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problem():
    return workloads.trunc_3d(seed=3, n_cells=16, n_targets=1562)


def _full(wl, precision):
    s = SotSolver(dim=3, device=0, precision=precision)
    s.setup_source_measure(wl["source"])
    s.setup_target(wl["y"], wl["nu"])
    s.configure(wl["params"])
    return s


def _psi(wl):
    N = wl["y"].shape[0]
    return 2e-3 * np.random.default_rng(8).standard_normal(N)


@pytest.mark.parametrize("world", [2, 4])
def test_partial_shards_sum_to_full(problem, oracle_mod, world):
    wl = problem
    N = wl["y"].shape[0]
    psi = _psi(wl)
    full = _full(wl, "fp64")
    g_full = np.zeros(N)
    J_full = full.evaluate_functional(psi, g_full)
    pairs_full = full.last_eval_info["n_pairs"]
    r_full = full.get_last_distance_threshold()
    full.close()

    psi_d = torch.tensor(psi, dtype=torch.float64, device="cuda")
    total = np.zeros(N + 3)
    for rank in range(world):
        sh = shard_source(wl["source"], rank, world)
        s = SotSolver(dim=3, device=0, precision="fp64")
        s.setup_source_measure(sh)
        s.setup_target(wl["y"], wl["nu"])
        s.configure(wl["params"])
        out = torch.empty(N + 3, dtype=torch.float64, device="cuda")
        s.evaluate_partial_device(psi_d.data_ptr(), out.data_ptr())
        assert s.get_last_distance_threshold() == r_full
        total += out.cpu().numpy()
        s.close()
    J, g, C, pairs = finish(total, psi, wl["nu"])
    assert int(pairs) == pairs_full
    assert np.max(np.abs(g - g_full)) <= 1e-15
    assert abs(J - J_full) <= 1e-13 * abs(J_full)

    src = wl["source"]
    P = oracle_mod.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"],
                           wl["y"], wl["nu"])
    prm = wl["params"]
    op = oracle_mod.Params(epsilon=prm.epsilon, tau=prm.tau, use_log_sum_exp=True)
    Jo, go, st = P.evaluate(psi, op)
    assert int(pairs) == st["n_pairs"]
    assert abs(J - Jo) <= 1e-10 * abs(Jo)
    assert np.max(np.abs(g - go)) <= 1e-12
    assert abs(C - st["C_global"]) <= 1e-10 * abs(st["C_global"])


class _HostAllReduce:
    """Sum of the ranks' vectors in rank order, exchanged through host memory."""

    def __init__(self, world):
        self.world = world
        self.slots = [None] * world
        self.bar = threading.Barrier(world, timeout=120)

    def for_rank(self, rank):
        def all_reduce(t):
            self.slots[rank] = t.cpu().numpy().copy()
            self.bar.wait()
            s = np.zeros_like(self.slots[0])
            for v in self.slots:
                s += v
            self.bar.wait()
            t.copy_(torch.from_numpy(s).to(t.device))
        return all_reduce


@pytest.mark.parametrize("precision", ["fp64", "hybrid"])
def test_distributed_solver_ranks_on_one_gpu(problem, oracle_mod, precision):
    wl = problem
    world = 2
    N = wl["y"].shape[0]
    psi = _psi(wl)
    red = _HostAllReduce(world)
    results = [None] * world
    errors = []

    def rank_main(rank):
        try:
            ds = DistributedSotSolver(3, rank, world, device=0, precision=precision,
                                      all_reduce=red.for_rank(rank))
            ds.setup_source(wl["source"])
            ds.setup_target(wl["y"], wl["nu"])
            ds.configure(wl["params"])
            psi_d = torch.tensor(psi, dtype=torch.float64, device="cuda")
            outs = []
            for _ in range(2):   # the second evaluation reads the state the first one set
                J, g, C, pairs = ds.evaluate(psi_d)
                outs.append((J, g.cpu().numpy(), C, pairs))
            ds.close()
            results[rank] = outs
        except Exception as e:  # noqa: BLE001 - reported below
            errors.append(repr(e))
            red.bar.abort()

    th = [threading.Thread(target=rank_main, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=300)
    assert not errors, errors
    # every rank finishes identically
    for k in range(2):
        J0, g0, C0, p0 = results[0][k]
        for r in range(1, world):
            J1, g1, C1, p1 = results[r][k]
            assert J0 == J1 and C0 == C1 and p0 == p1 and np.array_equal(g0, g1)
    J, g, C, pairs = results[0][1]
    src = wl["source"]
    P = oracle_mod.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"],
                           wl["y"], wl["nu"])
    prm = wl["params"]
    op = oracle_mod.Params(epsilon=prm.epsilon, tau=prm.tau, use_log_sum_exp=True)
    Jo, go, st = P.evaluate(psi, op)
    assert int(pairs) == st["n_pairs"]
    assert abs(J - Jo) <= 1e-10 * abs(Jo)
    assert np.max(np.abs(g - go)) <= (1e-12 if precision == "fp64" else max(1e-8, 5e-6 * np.max(wl["nu"])))
    assert abs(C - st["C_global"]) <= 1e-10 * abs(st["C_global"])
