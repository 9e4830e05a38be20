"""The sharded calls (pfcuda_b200/shard.py) with the engine's own compute, on
one GPU: a process group of world size 1 over NCCL, so every collective runs
and the results must equal the unsharded calls bit for bit.  (Runs on more
GPUs follow the same code; their host logic is tested at world size 2 over
gloo in tests/test_shard_cpu.py.)"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist

import pfcuda_b200 as pf
from pfcuda_b200 import shard
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def group():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    import datetime
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60), device_id=torch.device("cuda", 0))
    yield dist.group.WORLD
    dist.destroy_process_group()


def test_uniform_slog(group):
    rng = np.random.default_rng(3)
    A = torch.from_numpy(O.skew_normal(rng, 5, 300, scale=1 / np.sqrt(300))).cuda()
    la, sg = shard.slog_pfaffian_sharded(A, group=group)
    l1, s1 = pf.slog_pfaffian_raw(A)
    assert torch.equal(la, l1) and torch.equal(sg, s1)


def test_uniform_complex(group):
    rng = np.random.default_rng(4)
    A = torch.from_numpy(O.skew_normal(rng, 3, 130, scale=1 / np.sqrt(130), complex_=True)).cuda()
    la, sg = shard.slog_pfaffian_sharded(A, group=group)
    l1, s1 = pf.slog_pfaffian_raw(A)
    assert torch.equal(la, l1) and torch.equal(sg, s1)


def test_small_path(group):
    A = torch.from_numpy(O.config_small()[:64]).cuda()
    assert torch.equal(shard.pfaffian_sharded(A, group=group), pf.pfaffian_raw(A))


def test_ragged_with_large_bin(group):
    rng = np.random.default_rng(5)
    mats = [torch.from_numpy(O.skew_normal(rng, 1, m, scale=1 / np.sqrt(m))[0]).cuda()
            for m in (10, 600, 80, 1030, 40, 600)]
    la, sg = shard.slog_pfaffian_ragged_sharded(mats, group=group)
    l1, s1 = pf.slog_pfaffian_ragged(mats)
    assert torch.equal(la, l1) and torch.equal(sg, s1)


def test_grad(group):
    rng = np.random.default_rng(6)
    A = torch.from_numpy(O.skew_normal(rng, 3, 96, scale=0.1)).cuda()
    ct = torch.tensor([1.0, -0.5, 2.0], dtype=torch.float64, device="cuda")
    G = shard.slog_pfaffian_grad_sharded(A, ct, group=group)
    assert torch.equal(G, pf.slog_pfaffian_grad(A, ct=ct))
