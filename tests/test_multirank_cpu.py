"""Multi-rank (source-sharded) evaluation on CPU: world_size 2, gloo.

Each rank evaluates its contiguous range of cells, the (N + 3)-double
partial vector is all-reduced, and every rank finishes identically
(semidiscreteot_b200.distributed).  The per-rank partial here comes from the
CPU oracle (no GPU on this machine); on GPUs it comes from
sdot_evaluate_partial_device and the all-reduce runs on NCCL.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _problem():
    from semidiscreteot_b200.source import structured_source
    rng = np.random.default_rng(11)
    src = structured_source(2, 12, 3, nodal_density=lambda p: 1.0 + p[:, 0])
    N = 80
    y = rng.random((N, 2))
    nu = rng.dirichlet(np.ones(N) * 4)
    psi = 0.01 * rng.standard_normal(N)
    return src, y, nu, psi


def _worker(rank, world, port, tau, out_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from oracle import oracle as orc
        from semidiscreteot_b200.distributed import DistributedSotSolver, shard_source
        src, y, nu, psi = _problem()
        prm = orc.Params(epsilon=0.02, tau=tau, use_log_sum_exp=True)
        full = orc.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"], y, nu)
        sh = shard_source(src, rank, world)
        P = orc.Problem(sh["x"], sh["jxw"], sh["density"], sh["cell_offsets"], sh["cell_centers"], y, nu)

        def partial(psi_t):
            p = psi_t.numpy()
            r = full.distance_threshold(p, prm)    # depends only on the replicated psi
            J, g, C, pairs = P.evaluate_cells(p, prm, r, 0, P.ctr.shape[0])
            return torch.from_numpy(np.concatenate([g, [J, C, float(pairs)]]))

        ds = DistributedSotSolver(2, rank, world, partial_fn=partial)
        ds.setup_source(src)
        ds.setup_target(y, nu)
        J, g, C, pairs = ds.evaluate(torch.from_numpy(psi))
        out_q.put((rank, J, g.numpy(), C, pairs))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("tau", [0.0, 1e-6])
def test_sharded_evaluation_matches_full(oracle_mod, tau):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, tau, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    src, y, nu, psi = _problem()
    full = oracle_mod.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"], y, nu)
    Jf, gf, st = full.evaluate(psi, oracle_mod.Params(epsilon=0.02, tau=tau, use_log_sum_exp=True))
    for rank, J, g, C, pairs in res:
        assert abs(J - Jf) <= 1e-13
        np.testing.assert_allclose(g, gf, atol=1e-15)
        assert abs(C - st["C_global"]) <= 1e-12 * st["C_global"]
        assert pairs == st["n_pairs"]
    # both ranks finish with bitwise identical results (all-reduce replicates)
    assert res[0][1] == res[1][1] and np.array_equal(res[0][2], res[1][2])


def test_shard_ranges_cover_cells():
    from semidiscreteot_b200.distributed import shard_range
    for n in (1, 7, 64, 1000):
        for w in (1, 2, 3, 8):
            ranges = [shard_range(n, r, w) for r in range(w)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            assert all(ranges[i][1] == ranges[i + 1][0] for i in range(w - 1))
