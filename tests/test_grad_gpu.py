"""Adjoint of log|Pf| (pfb_slog_pfaffian_grad) against the reference's rule.

The reference's slog_pfaffian_jvp (pfcuda/cuda_api.py:92-107) gives
d log Pf = (1/2) tr(A^-1 dA); the oracle restates it with a general inverse
(oracle.slog_pf_vjp = ct * (1/2) A^-T) and pins it against central differences
of the C restatement of log|Pf| (h = 1e-6).

Bars: relative Frobenius error <= max(1e-9, 1e-13 cond(A)) against the
oracle's inverse for FP64 / complex128 work (both sides carry forward errors of
order n * eps * cond(A)); <= 2e-6 for float32 / complex64 outputs (the engine
computes in FP64 and rounds once);
directional derivatives within 1e-6 (relative) of the central difference.
"""
import numpy as np
import pytest
import torch

import pfcuda_b200 as pf
from pfcuda_b200 import _lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def cuda(a):
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def rel(a, b):
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    return np.linalg.norm((a - b).reshape(len(a), -1), axis=1) / np.linalg.norm(b.reshape(len(b), -1), axis=1)


def bound(A):
    """Per-matrix bar for FP64 work: max(1e-9, 1e-13 * cond_2(A))."""
    A = np.asarray(A, dtype=np.complex128)
    return np.maximum(1e-9, 1e-13 * np.linalg.cond(A))


def run(A, mode="fp64", ct=None, layout=_lib.ROW_MAJOR):
    G, la, sg = pf.slog_pfaffian_grad(cuda(A), ct=None if ct is None else cuda(ct), mode=mode,
                                      layout=layout, return_forward=True)
    return G.cpu().numpy(), la.cpu().numpy(), sg.cpu().numpy()


@pytest.mark.parametrize("mode", ["fp64", "split"])
@pytest.mark.parametrize("n", [2, 4, 8, 20, 34, 64, 66, 100, 130, 200, 290])
def test_grad_f64(mode, n):
    rng = np.random.default_rng(100 + n)
    A = O.skew_normal(rng, 3, n, scale=1 / np.sqrt(n))
    G, la, sg = run(A, mode)
    assert G.dtype == np.float64 and G.shape == A.shape
    assert np.all(rel(G, O.slog_pf_vjp(A)) <= bound(A))
    assert np.allclose(G, -np.swapaxes(G, -1, -2), rtol=0, atol=0)     # exactly skew
    wl, ws = O.slog_pf(A)
    assert np.all(np.abs(la - wl) <= 1e-10 * np.abs(wl) + 1e-12)
    assert np.array_equal(sg, ws)


@pytest.mark.parametrize("mode", ["fp64", "split"])
@pytest.mark.parametrize("n", [4, 34, 100, 256])
def test_grad_c128(mode, n):
    rng = np.random.default_rng(200 + n)
    A = O.skew_normal(rng, 2, n, scale=1 / np.sqrt(n), complex_=True)
    G, la, sg = run(A, mode)
    assert G.dtype == np.complex128
    assert np.all(rel(G, O.slog_pf_vjp(A)) <= bound(A))
    wl, ws = O.slog_pf(A)
    assert np.all(np.abs(la - wl) <= 1e-10 * np.abs(wl) + 1e-12)
    assert np.all(np.abs(sg - ws) <= 1e-10)


def test_grad_workload_slice():
    """Eight matrices of the 256 x complex128 x 512 gradient workload."""
    A = O.config_grad()[:8]
    ct = np.linspace(-2.0, 3.0, 8)
    G, _, _ = run(A, "fp64", ct=ct)
    assert np.all(rel(G, O.slog_pf_vjp(A, ct)) <= bound(A))


@pytest.mark.parametrize("npdt", [np.float32, np.complex64])
def test_grad_single_precision(npdt):
    rng = np.random.default_rng(7)
    A = O.skew_normal(rng, 2, 96, scale=0.1, complex_=np.dtype(npdt).kind == "c").astype(npdt)
    G, _, _ = run(A)
    assert G.dtype == npdt
    # the engine widens the input exactly, so the oracle sees the same matrix
    assert np.all(rel(G, O.slog_pf_vjp(A)) <= 2e-6)


def test_grad_column_major():
    """Memory M read column-major is A = M^T; the gradient comes back column-major."""
    rng = np.random.default_rng(8)
    M = O.skew_normal(rng, 2, 130, scale=1 / np.sqrt(130))
    G, la, _ = run(M, layout=_lib.COL_MAJOR)
    A = np.swapaxes(M, -1, -2)
    want = np.swapaxes(O.slog_pf_vjp(A), -1, -2)     # column-major memory of the gradient
    assert np.all(rel(G, want) <= bound(M))
    wl, _ = O.slog_pf(A)
    assert np.all(np.abs(la - wl) <= 1e-10 * np.abs(wl))


def test_grad_cotangents():
    rng = np.random.default_rng(9)
    A = O.skew_normal(rng, 4, 66, scale=1 / np.sqrt(66))
    G1, _, _ = run(A)
    ct = np.array([0.5, -1.0, 0.0, 7.0])
    Gc, _, _ = run(A, ct=ct)
    assert np.array_equal(Gc, G1 * ct[:, None, None])      # the scale is applied in FP64 once


@pytest.mark.parametrize("cplx", [False, True])
def test_grad_matches_central_difference(cplx):
    rng = np.random.default_rng(10 + cplx)
    A = O.skew_normal(rng, 3, 80, scale=1 / np.sqrt(80), complex_=cplx)
    E = O.skew_normal(rng, 3, 80, complex_=cplx)
    G, _, _ = run(A)
    d = np.sum(G * E, axis=(-1, -2)).real
    fd = O.fd_slog(A, E, h=1e-6)
    assert np.all(np.abs(d - fd) <= 1e-6 * np.abs(fd) + 1e-7), (d, fd)
    # and against the reference's JVP rule itself
    scale = np.sum(np.abs(O.slog_pf_vjp(A) * E), axis=(-1, -2))
    assert np.all(np.abs(d - O.slog_pf_jvp(A, E).real) <= bound(A) * scale)


def test_grad_zero_pfaffian_is_nan():
    rng = np.random.default_rng(11)
    A = O.skew_normal(rng, 2, 64, scale=0.1)
    A[1, 5, :] = 0.0
    A[1, :, 5] = 0.0
    G, la, sg = run(A)
    assert np.all(np.isfinite(G[0])) and np.all(np.isnan(G[1]))
    assert la[1] == -np.inf and sg[1] == 0


def test_grad_odd_order():
    A = torch.zeros(2, 35, 35, dtype=torch.float64, device="cuda")
    G, la, sg = pf.slog_pfaffian_grad(A, return_forward=True)
    assert torch.isnan(G).all() and torch.isinf(la).all()
    assert _lib.lib().pfb_slog_pfaffian_grad(_lib.F64, A.data_ptr(), 2, 35, 0, 0, None, G.data_ptr(),
                                             la.data_ptr(), sg.data_ptr(), None, 0, None) != 0


def test_autograd_slog_pfaffian():
    rng = np.random.default_rng(12)
    for cplx in (False, True):
        A = O.skew_normal(rng, 3, 72, scale=1 / np.sqrt(72), complex_=cplx)
        At = cuda(A).requires_grad_(True)
        la, sg = pf.slog_pfaffian(At, mode="split")
        w = torch.tensor([1.0, -0.5, 2.0], dtype=torch.float64, device="cuda")
        (la * w).sum().backward()
        want = O.slog_pf_vjp(A, w.cpu().numpy())
        if cplx:
            want = want.conj()
        assert np.all(rel(At.grad.cpu().numpy(), want) <= bound(A))


def test_autograd_pfaffian_small():
    rng = np.random.default_rng(13)
    for cplx in (False, True):
        A = O.skew_normal(rng, 5, 16, complex_=cplx)
        At = cuda(A).requires_grad_(True)
        p = pf.pfaffian(At)
        g = torch.ones_like(p)
        p.backward(g)
        pfv = O.pf_product(A)
        want = pfv[:, None, None] * O.slog_pf_vjp(A)
        if cplx:
            want = want.conj()
        assert np.all(rel(At.grad.cpu().numpy(), want) <= bound(A))


def test_grad_ignores_lower_triangle():
    """The adjoint, like the forward pass, reads only the upper triangle of
    the input's row-major view: NaN below the diagonal changes nothing."""
    rng = np.random.default_rng(14)
    for cplx in (False, True):
        A = O.skew_normal(rng, 2, 130, scale=1 / np.sqrt(130), complex_=cplx)
        D = A.copy()
        il = np.tril_indices(130, -1)
        D[:, il[0], il[1]] = np.nan
        G1, l1, s1 = run(A)
        G2, l2, s2 = run(D)
        assert np.array_equal(G1, G2) and np.array_equal(l1, l2) and np.array_equal(s1, s2)


# ------------------------------------------------------------ forward mode

@pytest.mark.parametrize("cplx", [False, True])
def test_forward_mode_slog(cplx):
    """torch.func.jvp of slog_pfaffian through the engine: the tangent of
    log|Pf| is Re (1/2) tr(A^-1 dA) (the reference's rule, pfcuda/cuda_api.py:
    92-107, restated with NumPy's inverse), and matches central differences
    along skew directions; the phase of complex A turns by i Im of the trace."""
    rng = np.random.default_rng(300 + cplx)
    n = 130
    A = O.skew_normal(rng, 2, n, scale=1 / np.sqrt(n), complex_=cplx)
    E = O.skew_normal(rng, 2, n, scale=1 / np.sqrt(n), complex_=cplx)
    (la, sg), (dla, dsg) = torch.func.jvp(lambda X: pf.slog_pfaffian(X, mode="fp64"), (cuda(A),), (cuda(E),))
    t = O.slog_pf_jvp(A, E)
    assert np.all(np.abs(dla.cpu().numpy() - np.real(t)) <= 1e-9 * np.abs(t) + 1e-10)
    assert np.all(np.abs(dla.cpu().numpy() - O.fd_slog(A, E)) <= 1e-6 * np.abs(t) + 1e-8)
    if cplx:
        want = sg.cpu().numpy() * 1j * np.imag(t)
        assert np.all(np.abs(dsg.cpu().numpy() - want) <= 1e-9 * np.abs(t) + 1e-10)


@pytest.mark.parametrize("cplx", [False, True])
def test_forward_mode_pfaffian(cplx):
    """torch.func.jvp of pfaffian: d Pf = Pf (1/2) tr(A^-1 dA) (pfcuda/cuda_api.py:78-90)."""
    rng = np.random.default_rng(310 + cplx)
    A = O.skew_normal(rng, 16, 24, complex_=cplx)
    E = O.skew_normal(rng, 16, 24, complex_=cplx)
    p, dp = torch.func.jvp(pf.pfaffian, (cuda(A),), (cuda(E),))
    want = O.pf_product(A) * O.slog_pf_jvp(A, E)
    assert np.all(np.abs(dp.cpu().numpy() - want) <= 1e-9 * np.abs(want) + 1e-9)


# ------------------------------------------------------------ memory budget

@pytest.mark.parametrize("mode", ["fp64", "split"])
def test_budget_chunks_are_bit_identical(mode):
    """A workspace below the whole batch's need runs the batch in chunks of as
    many matrices as fit; the gradients and forward values equal those of one
    unbounded call bit for bit, down to one matrix at a time."""
    from pfcuda_b200.grad import grad_min_workspace_bytes, grad_workspace_bytes
    rng = np.random.default_rng(320)
    n, B = 160, 7
    A = cuda(O.skew_normal(rng, B, n, scale=1 / np.sqrt(n)))
    ct = cuda(np.linspace(-1.0, 2.0, B))
    full = pf.slog_pfaffian_grad(A, ct=ct, mode=mode, return_forward=True)
    w1 = grad_min_workspace_bytes(A.dtype, n, mode)
    assert w1 < grad_workspace_bytes(A.dtype, B, n, mode)
    for budget in (w1, 3 * w1 - 1, grad_workspace_bytes(A.dtype, 3, n, mode)):
        got = pf.slog_pfaffian_grad(A, ct=ct, mode=mode, return_forward=True, budget_bytes=budget)
        for x, y in zip(got, full):
            assert torch.equal(x, y)
    with pytest.raises(ValueError):
        pf.slog_pfaffian_grad(A, mode=mode, budget_bytes=w1 - 1)


def test_budget_below_one_matrix_is_refused_by_the_c_abi():
    from pfcuda_b200.grad import grad_min_workspace_bytes
    n = 66
    A = cuda(np.zeros((2, n, n)))
    w1 = grad_min_workspace_bytes(A.dtype, n, "fp64")
    ws = torch.empty(w1, dtype=torch.uint8, device="cuda")
    G = torch.empty_like(A)
    la = torch.empty(2, dtype=torch.float64, device="cuda")
    sg = torch.empty(2, dtype=torch.float64, device="cuda")
    L = _lib.lib()
    s = torch.cuda.current_stream().cuda_stream
    st = L.pfb_slog_pfaffian_grad(_lib.F64, A.data_ptr(), 2, n, 0, 0, None, G.data_ptr(), la.data_ptr(),
                                  sg.data_ptr(), ws.data_ptr(), w1 - 256, s)
    assert st == 3                                  # PFB_ERR_WORKSPACE
    st = L.pfb_slog_pfaffian_grad(_lib.F64, A.data_ptr(), 2, n, 0, 0, None, G.data_ptr(), la.data_ptr(),
                                  sg.data_ptr(), ws.data_ptr(), w1, s)
    assert st == 0


# ------------------------------------------------- ill-conditioned, exact

@pytest.mark.parametrize("mode", ["fp64", "split"])
def test_grad_ill_conditioned_vs_exact_inverse(mode):
    """The ill-conditioned construction A = Q blockdiag(s_k J) Q^T (s_k in
    [1e-6, 1], cond_2 = 1e6) has the exact adjoint (1/2) Q blockdiag(J/s_k) Q^T,
    formed from the stored Q (oracle.illcond_half_inv_t).  The adjoint's error
    is the factors' element error amplified by cond_2: bar = 4 cond_2 sqrt(n) u
    with u the unit of the trailing updates -- eps for the FP64 path (about
    4e-8 at 2n = 2048, well below the worst-case cond n eps = 2.3e-7 that a
    general inverse may reach), sqrt(K) 2^(-7S) for the split path (its 64-term
    int8 products keep S = 7 digits of 7 bits: about 2.5e-6 here; measured
    2.2e-7)."""
    A, logs, signs, Q = O.config_illcond(B=2, n=2048, return_q=True)
    G = pf.slog_pfaffian_grad(cuda(A), mode=mode).cpu().numpy()
    Gx = O.illcond_half_inv_t(Q)
    err = rel(G, Gx)
    u = np.finfo(np.float64).eps if mode == "fp64" else np.sqrt(64) * 2.0 ** (-49)
    bar = 4 * 1e6 * np.sqrt(2048) * u
    assert np.all(err <= bar), (err, bar)
