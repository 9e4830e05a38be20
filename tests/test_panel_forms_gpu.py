"""The two panel forms of the large path (pfb_slog_config.panel).

PFB_PANEL_REGISTERS keeps each trailing column's panel rows in one thread's
registers (one CTA per SM); PFB_PANEL_HALF_SHARED keeps half of them in shared
memory (two CTAs per SM).  Both run the same pivot steps with the same partial
sums in the same order, so the results and the pivot columns must be equal bit
for bit -- and equal to the oracle's to the large path's bar (1e-10 relative,
signs identical, pivots identical).
"""
import numpy as np
import pytest
import torch

import pfcuda_b200 as pf
from pfcuda_b200 import _lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FORMS = ["registers", "half_shared"]


def cuda(a):
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def run(X, mode, panel):
    return pf.slog_pfaffian_raw(X, mode=mode, return_pivots=True, config={"panel": panel, "ranges": 1})


@pytest.mark.parametrize("mode", ["fp64", "split"])
@pytest.mark.parametrize("n", [34, 66, 96, 128, 130, 194, 256, 290, 514, 1030])
def test_forms_equal_f64(mode, n):
    rng = np.random.default_rng(500 + n)
    A = O.skew_normal(rng, 3, n, scale=1 / np.sqrt(n))
    X = cuda(A)
    r1 = run(X, mode, "registers")
    r2 = run(X, mode, "half_shared")
    for a, b in zip(r1, r2):
        assert torch.equal(a, b)
    if n <= 514:
        wl, ws, wp = O.slog_pf(A, with_pivots=True)
        la, sg, piv = (x.cpu().numpy() for x in r2)
        assert np.all(np.abs(la - wl) <= 1e-10 * np.abs(wl) + 1e-12)
        assert np.array_equal(sg, ws) and np.array_equal(piv, wp)


@pytest.mark.parametrize("mode", ["fp64", "split"])
@pytest.mark.parametrize("n", [34, 66, 100, 258])
def test_forms_equal_c128(mode, n):
    rng = np.random.default_rng(600 + n)
    A = O.skew_normal(rng, 2, n, scale=1 / np.sqrt(n), complex_=True)
    X = cuda(A)
    r1 = run(X, mode, "registers")
    r2 = run(X, mode, "half_shared")
    for a, b in zip(r1, r2):
        assert torch.equal(a, b)
    wl, ws, wp = O.slog_pf(A, with_pivots=True)
    la, sg, piv = (x.cpu().numpy() for x in r2)
    assert np.all(np.abs(la - wl) <= 1e-10 * np.abs(wl) + 1e-12)
    assert np.all(np.abs(sg - ws) <= 1e-10) and np.array_equal(piv, wp)


def test_forms_equal_at_the_headline_order():
    """2n = 4096, the widest clusters (16 CTAs): a few matrices, split mode."""
    rng = np.random.default_rng(7)
    X = cuda(O.skew_normal(rng, 2, 4096, scale=1 / 64))
    r1 = run(X, "split", "registers")
    r2 = run(X, "split", "half_shared")
    for a, b in zip(r1, r2):
        assert torch.equal(a, b)


def test_zero_and_singular_matrices():
    """A zero pivot stops either form the same way: (-inf, 0)."""
    n = 130
    A = np.zeros((2, n, n))
    rng = np.random.default_rng(8)
    B = O.skew_normal(rng, 1, n // 2, scale=1.0)[0]
    A[1, : n // 2, : n // 2] = B                      # rank-deficient: Pf = 0
    for form in FORMS:
        la, sg, _ = run(cuda(A), "fp64", form)
        assert np.all(np.isneginf(la.cpu().numpy())) and np.all(sg.cpu().numpy() == 0)


def test_half_shared_fits_more_clusters():
    L = _lib.lib()
    m1 = L.pfb_slog_max_concurrent_form(_lib.F64, 4096, _lib.PANEL_REGISTERS)
    m2 = L.pfb_slog_max_concurrent_form(_lib.F64, 4096, _lib.PANEL_HALF_SHARED)
    assert m1 == L.pfb_slog_max_concurrent(_lib.F64, 4096) and m1 > 0
    assert m2 > m1
    # orders whose panel holds two trailing columns per thread have no such form
    assert L.pfb_slog_max_concurrent_form(_lib.F64, 6000, _lib.PANEL_HALF_SHARED) == 0


def test_config_overrides_are_checked():
    X = cuda(np.zeros((1, 66, 66)))
    with pytest.raises(_lib.PfbError):
        pf.slog_pfaffian_raw(X, mode="fp64", config={"panel": 3})
    with pytest.raises(_lib.PfbError):
        pf.slog_pfaffian_raw(X, mode="split", config={"slices": 8})
    cfg = pf.slog_config(torch.float64, 28, 4096, "split")
    assert cfg["panel"] in ("registers", "half_shared") and 1 <= cfg["slices"] <= 7 and cfg["ranges"] in (1, 2)


# ------------------------------------------------------ split epilogues

@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("n", [34, 66, 130, 256, 514, 1030])
def test_split_epilogues_equal(cplx, n):
    """The split update's epilogues -- the C tile through shared memory (round
    trip), the L2 reduce-add of the increment, and the transposed tile with C
    read and written from global memory (direct; real input, complex falls
    back to the round trip) -- round identically: the increment value * 2^e is
    exact and C + increment is rounded once in each, so results and pivots
    are equal bit for bit."""
    rng = np.random.default_rng(700 + n + cplx)
    A = O.skew_normal(rng, 3, n, scale=1 / np.sqrt(n), complex_=cplx)
    X = cuda(A)
    r1 = pf.slog_pfaffian_raw(X, mode="split", return_pivots=True, config={"epilogue": "roundtrip"})
    r2 = pf.slog_pfaffian_raw(X, mode="split", return_pivots=True, config={"epilogue": "reduce"})
    r3 = pf.slog_pfaffian_raw(X, mode="split", return_pivots=True, config={"epilogue": "direct"})
    for a, b, c in zip(r1, r2, r3):
        assert torch.equal(a, b) and torch.equal(a, c)
    if n <= 256:
        wl, ws, wp = O.slog_pf(A, with_pivots=True)
        la, sg, piv = (x.cpu().numpy() for x in r2)
        assert np.all(np.abs(la - wl) <= 1e-10 * np.abs(wl) + 1e-12)
        assert np.array_equal(piv, wp)


def test_split_epilogues_equal_at_the_headline_order():
    rng = np.random.default_rng(9)
    X = cuda(O.skew_normal(rng, 2, 4096, scale=1 / 64))
    r1 = pf.slog_pfaffian_raw(X, mode="split", return_pivots=True, config={"epilogue": "roundtrip"})
    r2 = pf.slog_pfaffian_raw(X, mode="split", return_pivots=True,
                              config={"epilogue": "reduce", "panel": "half_shared"})
    r3 = pf.slog_pfaffian_raw(X, mode="split", return_pivots=True,
                              config={"epilogue": "direct", "panel": "half_shared"})
    for a, b, c in zip(r1, r2, r3):
        assert torch.equal(a, b) and torch.equal(a, c)
