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


# ------------------------------------------------------------- the large bin

def large_mix(seed):
    """Orders on both sides of the ragged bin's limit (544), odd ones included,
    float32 and float64, several matrices of one large order."""
    rng = np.random.default_rng(seed)
    orders = [10, 544, 546, 200, 600, 1030, 600, 777, 33, 1200, 600, 2048]
    mats = []
    for i, n in enumerate(orders):
        G = rng.normal(scale=1 / np.sqrt(n), size=(n, n))
        mats.append(((G - G.T) / 2).astype(np.float32 if i % 3 == 1 else np.float64))
    return mats


def check_any(mats, la, sg):
    la, sg = la.cpu().numpy(), sg.cpu().numpy()
    for i, A in enumerate(mats):
        if A.shape[0] & 1:
            assert np.isneginf(la[i]) and sg[i] == 0
            continue
        wl, ws = O.slog_pf(A)
        assert abs(la[i] - wl) <= 1e-10 * abs(wl) + 1e-12, (i, A.shape, la[i], wl)
        assert sg[i] == ws, (i, A.shape)


@pytest.mark.parametrize("mode", ["split", "fp64"])
def test_large_bin_in_the_same_call(mode):
    """Orders above 544 share the call: each (order, dtype) group runs on the
    blocked cluster-panel path from the matrices where they lie."""
    mats = large_mix(21)
    plan = pf.RaggedPlan([torch.from_numpy(A).cuda() for A in mats], mode=mode)
    # (546, f64) (600, f32) (600, f64) (1030, f64) (1200, f64) (2048, f64)
    assert len(plan._groups) == 6
    la, sg = plan.run()
    check_any(mats, la, sg)


def test_large_bin_graph_capture_replays():
    mats = large_mix(22)
    plan = pf.RaggedPlan([torch.from_numpy(A).cuda() for A in mats])
    la0, sg0 = [x.clone() for x in plan.run()]
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        plan.run()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        plan.run()
    plan.log.zero_()
    plan.sign.zero_()
    g.replay()
    torch.cuda.synchronize()
    la1, sg1 = plan.log.clone(), plan.sign.clone()
    # the odd large order keeps the (-inf, 0) written when the plan was built
    odd = [i for i, A in enumerate(mats) if A.shape[0] & 1 and A.shape[0] > 544]
    for i in odd:
        la1[i], sg1[i] = la0[i], sg0[i]
    assert torch.equal(la1, la0) and torch.equal(sg1, sg0)


def test_large_bin_matches_uniform_calls():
    """Each large group equals a uniform pfb_slog_pfaffian call on the same
    matrices stacked, bit for bit."""
    mats = large_mix(23)
    t = [torch.from_numpy(A).cuda() for A in mats]
    la, sg = pf.slog_pfaffian_ragged(t)
    idx = [i for i, A in enumerate(mats) if A.shape[0] == 600 and A.dtype == np.float64]
    gm = pf.resolve_mode("auto", torch.float64, 600, len(idx))
    l2, s2 = pf.slog_pfaffian_raw(torch.stack([t[i] for i in idx]), mode=gm)
    assert torch.equal(la[idx], l2) and torch.equal(sg[idx], s2.to(torch.float64))
