"""Ragged batches (pfb_slog_pfaffian_ragged) against the FP64 oracle.

Every matrix is factored in FP64 whatever its dtype, so float32 inputs are
compared with the oracle run on the same float32 values; the bar is the large
path's: |log|Pf| - oracle| <= 1e-10 |log|Pf|| (+1e-12), sign identical.
"""
import numpy as np
import pytest
import torch

import pfcuda_b200 as pf
from pfcuda_b200 import _lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def mixed(seed, count, lo=8, hi=512):
    rng = np.random.default_rng(seed)
    sizes = rng.choice(np.arange(lo, hi + 1, 2), size=count)
    mats = []
    for i, n in enumerate(sizes):
        G = rng.normal(scale=1 / np.sqrt(n), size=(n, n))
        A = (G - G.T) / 2
        mats.append(A.astype(np.float32 if i % 2 else np.float64))
    return mats


def check(mats, la, sg):
    la, sg = la.cpu().numpy(), sg.cpu().numpy()
    for i, A in enumerate(mats):
        wl, ws = O.slog_pf(A)
        assert abs(la[i] - wl) <= 1e-10 * abs(wl) + 1e-12, (i, A.shape, la[i], wl)
        assert sg[i] == ws, (i, A.shape)


def test_mixed_sizes_and_dtypes():
    mats = mixed(2, 150)
    la, sg = pf.slog_pfaffian_ragged([torch.from_numpy(A).cuda() for A in mats])
    check(mats, la, sg)


def test_edge_orders():
    rng = np.random.default_rng(5)
    mats = []
    for n in (2, 4, 6, 8, 30, 32, 34, 62, 64, 66, 96, 98, 510, 512, 544):
        G = rng.normal(size=(n, n)) / np.sqrt(n)
        mats.append((G - G.T) / 2)
    la, sg = pf.slog_pfaffian_ragged([torch.from_numpy(A).cuda() for A in mats])
    check(mats, la, sg)


def test_edge_orders_narrow_panels():
    """Batches whose largest order is at most 528 run two CTAs per SM with
    16-row panels; 528 fills every trailing column of the first panel."""
    rng = np.random.default_rng(15)
    mats = []
    for n in (2, 4, 14, 16, 18, 30, 32, 34, 48, 50, 510, 512, 526, 528):
        G = rng.normal(size=(n, n)) / np.sqrt(n)
        mats.append((G - G.T) / 2)
    la, sg = pf.slog_pfaffian_ragged([torch.from_numpy(A).cuda() for A in mats])
    check(mats, la, sg)
    # one order above 528 moves the whole batch to the 32-row configuration
    G = rng.normal(size=(530, 530)) / np.sqrt(530)
    mats.append((G - G.T) / 2)
    la, sg = pf.slog_pfaffian_ragged([torch.from_numpy(A).cuda() for A in mats])
    check(mats, la, sg)


def test_unaligned_inputs():
    """Matrices that start off a 16-byte boundary take the element-wise copy."""
    rng = np.random.default_rng(16)
    mats, views = [], []
    for n, dt, off in ((64, np.float64, 1), (66, np.float32, 1), (130, np.float32, 2), (96, np.float64, 0)):
        G = rng.normal(size=(n, n)) / np.sqrt(n)
        A = ((G - G.T) / 2).astype(dt)
        buf = torch.zeros(n * n + 4, dtype=torch.from_numpy(A).dtype, device="cuda")
        buf[off:off + n * n] = torch.from_numpy(A.reshape(-1)).cuda()
        mats.append(A)
        views.append(buf[off:off + n * n].view(n, n))
    la, sg = pf.slog_pfaffian_ragged(views)
    check(mats, la, sg)


def test_odd_zero_singular():
    rng = np.random.default_rng(6)
    G = rng.normal(size=(40, 40)) / 6
    sing = (G - G.T) / 2
    sing[7, :] = 0
    sing[:, 7] = 0
    mats = [np.ones((35, 35)), np.zeros((64, 64)), sing, (G - G.T) / 2]
    la, sg = pf.slog_pfaffian_ragged([torch.from_numpy(A).cuda() for A in mats])
    la, sg = la.cpu().numpy(), sg.cpu().numpy()
    assert np.isneginf(la[0]) and sg[0] == 0
    assert np.isneginf(la[1]) and sg[1] == 0
    assert np.isneginf(la[2]) and sg[2] == 0
    wl, ws = O.slog_pf(mats[3])
    assert abs(la[3] - wl) <= 1e-10 * abs(wl) and sg[3] == ws


def test_column_major():
    mats = mixed(7, 20, lo=34, hi=200)
    mats = [A.astype(np.float64) for A in mats]
    t = [torch.from_numpy(np.ascontiguousarray(A.T)).cuda() for A in mats]
    la, sg = pf.slog_pfaffian_ragged(t, layout=_lib.COL_MAJOR)
    check(mats, la, sg)


def test_graph_capture_replays():
    mats = mixed(8, 60, lo=8, hi=300)
    plan = pf.RaggedPlan([torch.from_numpy(A).cuda() for A in mats])
    la0, sg0 = [x.clone() for x in plan.run()]
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        plan.run()                      # warm-up on the capture stream
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        plan.run()
    plan.log.zero_()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(plan.log, la0) and torch.equal(plan.sign, sg0)
    check(mats, plan.log, plan.sign)
