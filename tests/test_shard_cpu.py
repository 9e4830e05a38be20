"""Batch sharding across ranks (pfcuda_b200/shard.py), on CPU process groups.

The per-rank compute is replaced by the oracle (these tests need no GPU); what
is tested is the host logic: which rank owns which matrices, the ragged
balance, and the gather of per-matrix results, with world size 2 over gloo.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from pfcuda_b200.shard import shard_range, shard_ragged, slog_pfaffian_sharded


def test_shard_range_partitions():
    for count in (0, 1, 7, 8, 4096):
        for world in (1, 2, 3, 8):
            spans = [shard_range(count, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == count
            assert all(spans[r][1] == spans[r + 1][0] for r in range(world - 1))
            sizes = [hi - lo for lo, hi in spans]
            assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)
    with pytest.raises(ValueError):
        shard_range(4, 2, 2)


def test_shard_ragged_balance():
    rng = np.random.default_rng(2)
    orders = rng.integers(4, 257, size=4000) * 2
    for world in (2, 4, 8):
        plan = shard_ragged(orders, world)
        assert sorted(i for lst in plan for i in lst) == list(range(len(orders)))
        loads = [sum(int(orders[i]) ** 3 for i in lst) for lst in plan]
        # LPT: no rank exceeds the mean by more than the largest single item
        assert max(loads) - sum(loads) / world <= int(orders.max()) ** 3
        assert plan == shard_ragged(orders, world)        # deterministic


def _oracle_compute(A):
    from oracle import oracle as O
    la, sg = O.slog_pf(A.numpy())
    return torch.from_numpy(np.asarray(la)), torch.from_numpy(np.asarray(sg))


def _worker(rank, world, port, cplx, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle as O
        rng = np.random.default_rng(5)
        A = torch.from_numpy(O.skew_normal(rng, 7, 40, scale=0.2, complex_=cplx))
        la, sg = slog_pfaffian_sharded(A, compute=_oracle_compute)
        own_l, _ = slog_pfaffian_sharded(A, compute=_oracle_compute, gather=False)
        q.put((rank, la.numpy(), sg.numpy(), own_l.numpy()))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("cplx", [False, True])
def test_sharded_gather_world2(cplx):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, cplx, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from oracle import oracle as O
    rng = np.random.default_rng(5)
    A = O.skew_normal(rng, 7, 40, scale=0.2, complex_=cplx)
    wl, ws = O.slog_pf(A)
    for rank, la, sg, own in got:
        assert np.array_equal(la, wl) and np.array_equal(sg, ws)
        lo, hi = shard_range(7, 2, rank)
        assert np.array_equal(own, wl[lo:hi])


# ------------------------------------------- ragged, small path, gradients

def _worker_more(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle as O
        from pfcuda_b200.shard import (slog_pfaffian_ragged_sharded, pfaffian_sharded,
                                       slog_pfaffian_grad_sharded)
        rng = np.random.default_rng(9)
        orders = [8, 40, 100, 34, 200, 12, 66, 150, 90]
        mats = [torch.from_numpy(O.skew_normal(rng, 1, m, scale=1 / np.sqrt(m))[0]) for m in orders]
        # other ranks' matrices are placeholders: only their shapes are read
        plan = shard_ragged(orders, world)
        given = [M if i in plan[rank] else torch.empty(M.shape, device="meta") for i, M in enumerate(mats)]

        def ragged_compute(lst):
            la, sg = O.slog_pf_list([M.numpy() for M in lst])
            return torch.from_numpy(la), torch.from_numpy(sg)

        rl, rs = slog_pfaffian_ragged_sharded(given, compute=ragged_compute)
        ol, osg, oidx = slog_pfaffian_ragged_sharded(given, compute=ragged_compute, gather=False)
        S = torch.from_numpy(O.skew_normal(rng, 5, 12))
        pf_all = pfaffian_sharded(S, compute=lambda X: torch.from_numpy(np.asarray(O.pf_product(X.numpy()))))
        G = torch.from_numpy(O.skew_normal(rng, 5, 20, scale=0.3))
        ct = torch.linspace(-1.0, 2.0, 5, dtype=torch.float64)
        g_all = slog_pfaffian_grad_sharded(
            G, ct, compute=lambda X, c: torch.from_numpy(O.slog_pf_vjp(X.numpy(), None if c is None else c.numpy())))
        q.put((rank, rl.numpy(), rs.numpy(), ol.numpy(), oidx.numpy(), pf_all.numpy(), g_all.numpy()))
    finally:
        dist.destroy_process_group()


def test_sharded_ragged_small_and_grad_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_more, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from oracle import oracle as O
    rng = np.random.default_rng(9)
    orders = [8, 40, 100, 34, 200, 12, 66, 150, 90]
    mats = [O.skew_normal(rng, 1, m, scale=1 / np.sqrt(m))[0] for m in orders]
    wl, ws = O.slog_pf_list(mats)
    S = O.skew_normal(rng, 5, 12)
    G = O.skew_normal(rng, 5, 20, scale=0.3)
    plan = shard_ragged(orders, 2)
    for rank, rl, rs, ol, oidx, pf_all, g_all in got:
        assert np.array_equal(rl, wl) and np.array_equal(rs, ws)
        assert list(oidx) == plan[rank] and np.array_equal(ol, wl[plan[rank]])
        assert np.array_equal(pf_all, O.pf_product(S))
        assert np.array_equal(g_all, O.slog_pf_vjp(G, np.linspace(-1.0, 2.0, 5)))
