"""Large path (pfb_slog_pfaffian, blocked skew-LTL^T) against the oracle.

Bar (the engine's accuracy target): |log|Pf| - oracle| <= 1e-10 * |log|Pf||
(plus 1e-12 absolute for logs near 0), the sign identical (real) or the phase
within 1e-10 (complex), and the pivot columns identical to the oracle's.
"""
import numpy as np
import pytest
import torch

import pfcuda_b200 as pf
from pfcuda_b200 import _lib
from oracle import oracle as O
from golden_io import load, split

pytestmark = pytest.mark.gpu

MODES = ["fp64", "split"]
# the register panel form with two ranges: a three-wave batch runs on two streams
TWO = {"panel": "registers", "ranges": 2}


def cuda(a):
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def check(A, mode, pivots=True, tol=1e-10):
    la, sg, piv = pf.slog_pfaffian_raw(cuda(A), mode=mode, return_pivots=True)
    la, sg, piv = la.cpu().numpy(), sg.cpu().numpy(), piv.cpu().numpy()
    wl, ws, wp = O.slog_pf(A, with_pivots=True)
    err = np.abs(la - wl)
    assert np.all(err <= tol * np.abs(wl) + 1e-12), (A.shape, err.max())
    if np.iscomplexobj(A):
        assert np.all(np.abs(sg - ws) <= 1e-10)
    else:
        assert np.array_equal(sg, ws)
    if pivots:
        assert np.array_equal(piv, wp)
    return la, sg


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("n", [34, 36, 40, 62, 64, 66, 100, 126, 128, 130, 192, 200, 256, 290])
def test_orders_f64(mode, n):
    rng = np.random.default_rng(n)
    check(O.skew_normal(rng, 3, n, scale=1 / np.sqrt(n)), mode)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("n", [34, 64, 66, 100, 256])
def test_orders_c128(mode, n):
    rng = np.random.default_rng(n + 1)
    check(O.skew_normal(rng, 2, n, scale=1 / np.sqrt(n), complex_=True), mode)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("npdt", [np.float32, np.complex64])
def test_single_precision_inputs_run_in_fp64(mode, npdt):
    rng = np.random.default_rng(4)
    A = O.skew_normal(rng, 2, 96, scale=0.1, complex_=np.dtype(npdt).kind == "c").astype(npdt)
    la, sg, piv = pf.slog_pfaffian_raw(cuda(A), mode=mode, return_pivots=True)
    wl, ws = O.slog_pf(A)           # the oracle upcasts the same values
    assert np.all(np.abs(la.cpu().numpy() - wl) <= 1e-10 * np.abs(wl))
    assert np.all(np.abs(sg.cpu().numpy() - ws) <= 1e-6)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("n", [64, 130, 258])
def test_column_major_layout(mode, n):
    rng = np.random.default_rng(n)
    for cplx in (False, True):
        A = O.skew_normal(rng, 2, n, scale=1 / np.sqrt(n), complex_=cplx)
        At = np.ascontiguousarray(np.swapaxes(A, -1, -2))
        l1, s1 = pf.slog_pfaffian_raw(cuda(A), mode=mode)
        l2, s2 = pf.slog_pfaffian_raw(cuda(At), mode=mode, layout=_lib.COL_MAJOR)
        assert torch.equal(l1, l2) and torch.equal(s1, s2)


@pytest.mark.parametrize("mode", MODES)
def test_zero_and_singular(mode):
    for n in range(34, 68, 8):
        la, sg = pf.slog_pfaffian(cuda(np.zeros((n, n))), mode=mode)
        assert np.isneginf(la.item()) and sg.item() == 0
    rng = np.random.default_rng(2)
    A = O.skew_normal(rng, 3, 80, scale=0.1)
    A[1, 17, :] = 0
    A[1, :, 17] = 0
    la, sg = pf.slog_pfaffian_raw(cuda(A), mode=mode)
    la = la.cpu().numpy()
    assert np.isneginf(la[1]) and sg[1].item() == 0 and np.isfinite(la[0]) and np.isfinite(la[2])


@pytest.mark.parametrize("mode", MODES)
def test_reference_det_relation(mode):
    rng = np.random.default_rng(1)                 # test/slog_pfaffian_test.py:47-59
    for n in range(34, 66, 2):
        G = rng.normal(size=(n, n))
        A = G - G.T
        la, sg = pf.slog_pfaffian(cuda(A), mode=mode)
        assert np.isclose(np.exp(2 * la.item()), np.linalg.det(A), rtol=1e-8, atol=1e-10)


@pytest.mark.parametrize("mode", MODES)
def test_reference_random_and_identity(mode):
    rng = np.random.default_rng(123)               # test/slog_pfaffian_test.py:61-74
    for n in range(40, 300, 10):
        G = rng.normal(size=(3, n, n))
        A = G - np.swapaxes(G, -1, -2)
        la, sg = pf.slog_pfaffian_raw(cuda(A), mode=mode)
        wl, ws = O.slog_pf(A)
        np.testing.assert_allclose(sg.cpu().numpy() * np.exp(la.cpu().numpy() - wl), ws, rtol=1e-8)
    g = load("known.npz")                          # test/slog_pfaffian_test.py:76-107
    for A, want in zip(split(g["A"], g["n"]), g["pf"]):
        if A.shape[0] <= 32:
            continue
        la, sg = pf.slog_pfaffian(cuda(A), mode=mode)
        assert np.isclose(sg.item() * np.exp(la.item()), want, rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("mode", MODES)
def test_reference_cpu_large_values(mode):
    g = load("cpu_large.npz")
    for seed, n, want in zip(g["seeds"], g["n"], g["pf"]):
        A = O.config_large(int(n), seed=int(seed))
        la, sg = pf.slog_pfaffian(cuda(A), mode=mode)
        assert abs(la.item() - np.log(abs(want))) <= 1e-10 * abs(la.item())
        assert sg.item() == np.sign(want)


@pytest.mark.parametrize("mode", MODES)
def test_batch_and_input_untouched(mode):
    rng = np.random.default_rng(6)
    A = O.skew_normal(rng, 5, 300, scale=0.05)
    X = cuda(A)
    X0 = X.clone()
    la, sg = pf.slog_pfaffian_raw(X, mode=mode)
    assert torch.equal(X, X0)
    for b in range(5):
        l1, s1 = pf.slog_pfaffian_raw(X[b], mode=mode)
        assert l1.item() == la[b].item() and s1.item() == sg[b].item()


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("n", [1024, 2048])
@pytest.mark.parametrize("cplx", [False, True])
def test_benchmark_orders(mode, n, cplx):
    A = O.config_large(n, dtype=np.complex128 if cplx else np.float64, seed=1)
    check(A, mode, pivots=not cplx)


@pytest.mark.parametrize("mode", MODES)
def test_order_4096_f64(mode):
    A = O.config_large(4096, seed=1)
    la, sg = pf.slog_pfaffian(cuda(A), mode=mode)
    s, ld = np.linalg.slogdet(A[0])
    assert abs(2 * la.item() - ld) <= 1e-10 * abs(ld)
    assert s > 0


@pytest.mark.parametrize("mode", MODES)
def test_ill_conditioned(mode):
    A, logs, signs = O.config_illcond(seed=4, B=2, n=256)
    la, sg = pf.slog_pfaffian(cuda(A), mode=mode)
    la, sg = la.cpu().numpy(), sg.cpu().numpy()
    assert np.all(np.abs(la - logs) <= 1e-10 * np.abs(logs))
    assert np.array_equal(sg, signs)


@pytest.mark.parametrize("n,cplx", [(4200, False), (6144, False), (3000, True), (4128, True)])
def test_widest_configurations(n, cplx):
    """The 32-row panels with two columns per thread (real 2n > 4160) and the
    complex panels up to their limit: log|Pf| = (1/2) log|det A| (NumPy's LU on
    the host) in both modes, split within 1e-10 of FP64, a unit sign."""
    A = O.config_large(n, dtype=np.complex128 if cplx else np.float64, seed=11)
    got = {}
    for mode in MODES:
        la, sg, piv = pf.slog_pfaffian_raw(cuda(A), mode=mode, return_pivots=True)
        got[mode] = (la.cpu().numpy(), sg.cpu().numpy(), piv.cpu().numpy())
    s, ld = np.linalg.slogdet(A[0])
    for mode in MODES:
        la = got[mode][0][0]
        assert abs(2 * la - ld) <= 1e-10 * abs(ld), (mode, 2 * la, ld)
    assert abs(got["split"][0][0] - got["fp64"][0][0]) <= 1e-10 * abs(got["fp64"][0][0])
    assert np.all(np.abs(np.abs(got["split"][1]) - 1) < 1e-10)


def test_max_concurrent_query():
    L = _lib.lib()
    for n in (64, 1024, 4096, 8000):
        m = L.pfb_slog_max_concurrent(_lib.F64, n)
        assert m >= 1
    assert L.pfb_slog_max_concurrent(_lib.F64, 16) == 0          # small path
    assert L.pfb_slog_max_concurrent(_lib.F64, 1 << 20) == 0     # beyond the large path


def test_auto_mode_picks_per_dtype():
    """slog_pfaffian's default mode is the one resolve_mode picks from the
    tuned table for the dtype, order and batch."""
    rng = np.random.default_rng(31)
    for cplx in (False, True):
        A = cuda(O.skew_normal(rng, 2, 130, scale=1 / np.sqrt(130), complex_=cplx))
        want = pf.resolve_mode("auto", A.dtype, 130, 2)
        la, sg = pf.slog_pfaffian(A)
        lw, sw = pf.slog_pfaffian(A, mode=want)
        assert torch.equal(la, lw) and torch.equal(sg, sw)


@pytest.mark.parametrize("mode", ["fp64", "split"])
def test_two_stream_batches_match_single_ranges(mode):
    """A batch of three or more waves of wide panel clusters runs as two ranges
    on two streams; every matrix's arithmetic is independent of the rest of
    the batch, so the results equal those of calls on one wave at a time, bit
    for bit, and the oracle's on a sample."""
    n = 2176                                   # widest panel cluster: 9 CTAs
    mc = _lib.lib().pfb_slog_max_concurrent(_lib.F64, n)
    assert mc > 0
    B = 3 * mc
    # the call under test does run as two ranges, and a one-wave call as one
    m = _lib.MODE_SPLIT if mode == "split" else _lib.MODE_FP64
    cfg = pf.slog_config(torch.float64, B, n, mode)
    if cfg["ranges"] == 2 and cfg["panel"] == "registers":
        assert _lib.lib().pfb_slog_stream_ranges(_lib.F64, B, n, m) == 2
        assert _lib.lib().pfb_slog_stream_ranges(_lib.F64, 2 * mc, n, m) == 2     # halves
    assert _lib.lib().pfb_slog_stream_ranges(_lib.F64, mc, n, m) == 1
    rng = np.random.default_rng(77)
    A = O.skew_normal(rng, B, n, scale=1 / np.sqrt(n))
    At = cuda(A)
    la, sg = pf.slog_pfaffian_raw(At, mode=mode, config=TWO)
    parts = [pf.slog_pfaffian_raw(At[i:i + mc].contiguous(), mode=mode, config=TWO) for i in range(0, B, mc)]
    la1 = torch.cat([p[0] for p in parts])
    sg1 = torch.cat([p[1] for p in parts])
    assert torch.equal(la, la1) and torch.equal(sg, sg1)
    wl, ws = O.slog_pf(A[-2:])
    got = la[-2:].cpu().numpy()
    assert np.all(np.abs(got - wl) <= 1e-10 * np.abs(wl)) and np.array_equal(sg[-2:].cpu().numpy(), ws)


def _two_range_batch(seed):
    n = 2176
    mc = _lib.lib().pfb_slog_max_concurrent(_lib.F64, n)
    B = 3 * mc                                 # three waves of the register form's clusters
    rng = np.random.default_rng(seed)
    return cuda(O.skew_normal(rng, B, n, scale=1 / np.sqrt(n)))


def test_two_threads_call_at_once():
    """Two host threads, each on its own stream, run two-range calls at the same
    time; each thread's second stream is its own, so every result equals the
    one of the same call made alone, bit for bit."""
    import threading
    ins = [_two_range_batch(90 + i) for i in range(2)]
    alone = [pf.slog_pfaffian_raw(X, mode="split", config=TWO) for X in ins]
    torch.cuda.synchronize()
    out = [None, None]
    errs = []

    def work(i):
        try:
            s = torch.cuda.Stream()
            with torch.cuda.stream(s):
                res = [pf.slog_pfaffian_raw(ins[i], mode="split", config=TWO) for _ in range(3)]
            s.synchronize()
            out[i] = res
        except Exception as e:          # surfaced on the main thread below
            errs.append(e)

    ts = [threading.Thread(target=work, args=(i,)) for i in range(2)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errs, errs
    for i in range(2):
        for la, sg in out[i]:
            assert torch.equal(la, alone[i][0]) and torch.equal(sg, alone[i][1])


def test_graph_capture_of_two_ranges():
    """A two-range call captured in a CUDA graph (the second stream forks from
    and joins the capturing stream) replays to the uncaptured results."""
    X = _two_range_batch(95)
    n, B = X.shape[-1], X.shape[0]
    wsb = pf.slog_workspace_bytes(X.dtype, B, n, "split")
    ws = torch.empty(wsb, dtype=torch.uint8, device=X.device)
    want = pf.slog_pfaffian_raw(X, mode="split", workspace=ws, config=TWO)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        la, sg = pf.slog_pfaffian_raw(X, mode="split", workspace=ws, config=TWO)
    for _ in range(2):
        la.zero_()
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(la, want[0]) and torch.equal(sg, want[1])


def test_split_timeout_path_marks_only_its_matrix():
    """PFB_SPLIT_TEST_TIMEOUT makes every bounded wait of the split update give
    up at once for the call's first matrix: that matrix comes back as
    (NaN, 0), the others are exact, and the device stays usable (a normal call
    right after is exact for all)."""
    rng = np.random.default_rng(41)
    n, B = 256, 3
    A = O.skew_normal(rng, B, n, scale=1 / np.sqrt(n))
    X = cuda(A)
    L = _lib.lib()
    wsb = pf.slog_workspace_bytes(X.dtype, B, n, "split")
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    la = torch.empty(B, dtype=torch.float64, device="cuda")
    sg = torch.empty(B, dtype=torch.float64, device="cuda")
    mode = _lib.MODE_SPLIT | (1 << 12)           # PFB_SPLIT_TEST_TIMEOUT
    st = L.pfb_slog_pfaffian(_lib.F64, X.data_ptr(), B, n, _lib.ROW_MAJOR, mode, la.data_ptr(), sg.data_ptr(),
                             ws.data_ptr(), wsb, torch.cuda.current_stream().cuda_stream)
    assert st == 0
    torch.cuda.synchronize()
    got_l, got_s = la.cpu().numpy(), sg.cpu().numpy()
    wl, wsg = O.slog_pf(A)
    assert np.isnan(got_l[0]) and got_s[0] == 0
    assert np.all(np.abs(got_l[1:] - wl[1:]) <= 1e-10 * np.abs(wl[1:]))
    assert np.array_equal(got_s[1:], wsg[1:])
    la2, sg2 = pf.slog_pfaffian_raw(X, mode="split")
    assert np.all(np.abs(la2.cpu().numpy() - wl) <= 1e-10 * np.abs(wl))
    assert np.array_equal(sg2.cpu().numpy(), wsg)


@pytest.mark.parametrize("mode,epilogue", [("fp64", None), ("split", "roundtrip"), ("split", "reduce"),
                                           ("split", "direct")])
@pytest.mark.parametrize("n", [130, 514])
def test_extreme_scales_match_the_exact_relation(mode, epilogue, n):
    """Pf(D A D) = det(D) Pf(A) for a diagonal D, so with D of powers of two
    log|Pf(DAD)| = sum log d_i + log|Pf(A)| and the sign is Pf(A)'s.  Every
    other index scaled by 2^-490: the split update's increments between two
    scaled indices need the scale 2^(e_a + e_b - 56) ~ 2^-1036, below the
    normal range, which the epilogue forms by the general path instead of
    from exponent bits; all matrix entries stay normal (~2^-980 and up)."""
    rng = np.random.default_rng(1200 + n)
    A = O.skew_normal(rng, 2, n, scale=1 / np.sqrt(n))
    d = np.where(np.arange(n) % 2 == 0, 2.0 ** -490, 1.0)
    As = A * d[None, :, None] * d[None, None, :]
    cfg = None if epilogue is None else {"epilogue": epilogue}
    la, sg = pf.slog_pfaffian_raw(cuda(As), mode=mode, config=cfg)
    la, sg = la.cpu().numpy(), sg.cpu().numpy()
    wl, ws = O.slog_pf(A)
    shift = float(np.sum(np.log(d)))
    # 1e-8 absolute: la sums ~n/2 logs of about -340 each (their rounding); a
    # lost or wrong scale would move log|Pf| by O(1)
    assert np.all(np.abs((la - shift) - wl) <= 1e-10 * np.abs(wl) + 1e-8), np.abs((la - shift) - wl).max()
    assert np.array_equal(sg, ws)
