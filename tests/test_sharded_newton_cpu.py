"""Newton with the Hessian sharded by output tiles, on CPU: world_size 2, gloo.

Every rank holds the whole problem and evaluates it (replicated); rank r
keeps the Hessian entries of its contiguous range of 128 x 256 upper-triangle
tiles (and their mirrors) in an otherwise zero matrix, so its matrix-vector
product is its share of H x and one all-reduce per CG step completes it
(semidiscreteot_b200.distributed.sharded_newton).  Here the evaluation and the
Hessian come from the FP64 CPU oracle; on GPUs they come from
sdot_evaluate / sdot_hessian_tiles_device and the all-reduce runs on NCCL.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

TOL = 1e-10


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _problem():
    from semidiscreteot_b200.source import structured_source
    rng = np.random.default_rng(5)
    src = structured_source(2, 12, 3, nodal_density=lambda p: 1.0 + p[:, 0])
    N = 300                                  # 5 tiles: split 2 / 3 over two ranks
    y = rng.random((N, 2))
    nu = rng.dirichlet(np.ones(N) * 4)
    return src, y, nu


def _backend(orc, rank, world, reduce):
    from semidiscreteot_b200.distributed import hessian_tile_mask, hessian_tiles, tile_range
    src, y, nu = _problem()
    prm = orc.Params(epsilon=0.05, tau=0.0, use_log_sum_exp=True)
    P = orc.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"], y, nu)
    n = len(nu)
    t0, t1 = tile_range(len(hessian_tiles(n)), rank, world)
    mask = hessian_tile_mask(n, t0, t1)

    def evaluate(psi):
        J, g, _ = P.evaluate(psi, prm)
        return J, g

    def hessian_part(psi):
        return np.where(mask, P.hessian(psi, prm, 1e300), 0.0)

    return n, evaluate, hessian_part, (lambda h, x: h @ x), (lambda h: np.diag(h).copy()), reduce


def _worker(rank, world, port, out_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from oracle import oracle as orc
        from semidiscreteot_b200.distributed import sharded_newton

        def reduce(v):
            t = torch.from_numpy(np.ascontiguousarray(v))
            dist.all_reduce(t)
            return t.numpy()

        n, ev, hp, mv, dg, red = _backend(orc, rank, world, reduce)
        psi, info = sharded_newton(np.zeros(n), ev, hp, mv, dg, red, TOL, "linf", 200)
        out_q.put((rank, psi, info))
    finally:
        dist.destroy_process_group()


def test_tile_masks_partition_the_matrix():
    from semidiscreteot_b200.distributed import hessian_tile_mask, hessian_tiles, tile_range
    for n in (1, 129, 300, 777):
        T = len(hessian_tiles(n))
        for world in (1, 2, 3, 4):
            count = sum(hessian_tile_mask(n, *tile_range(T, r, world)).astype(int) for r in range(world))
            assert np.all(count == 1), (n, world)


def test_sharded_newton_matches_one_rank(oracle_mod):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in procs], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from semidiscreteot_b200.distributed import sharded_newton
    n, ev, hp, mv, dg, red = _backend(oracle_mod, 0, 1, lambda v: v)
    psi1, info1 = sharded_newton(np.zeros(n), ev, hp, mv, dg, red, TOL, "linf", 200)
    (_, psi_a, info_a), (_, psi_b, info_b) = res
    # the ranks move in lockstep: same numbers everywhere
    assert np.array_equal(psi_a, psi_b) and info_a == info_b
    assert info_a["converged"] and info1["converged"]
    assert info_a["n_hessians"] <= info_a["iterations"]
    _, g = ev(psi_a)
    assert np.max(np.abs(g)) <= TOL
    # one rank and two ranks reach the same potential (the sums differ only in rounding)
    assert np.max(np.abs(psi_a - psi1)) <= 1e-8
