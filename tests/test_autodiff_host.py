"""Host logic of the differentiation rules (pfcuda_b200/api.py), on CPU.

The engine's kernels are replaced by the oracle (forward values) and by the
reference's rule restated with NumPy's inverse (the adjoint (1/2) A^-T), so
this checks only the torch glue: forward mode (torch.func.jvp and dual numbers)
against the reference's JVP rule (pfcuda/cuda_api.py:78-107) and finite
differences, and reverse mode with both cotangents of complex slog_pfaffian.
The same rules through the real kernels are in tests/test_grad_gpu.py.
"""
import numpy as np
import pytest
import torch
import torch.autograd.forward_ad as fwAD

import pfcuda_b200.api as api
import pfcuda_b200.grad as gradmod
from oracle import oracle as O


@pytest.fixture
def fake_engine(monkeypatch):
    def slog_raw(A, mode="split", **kw):
        la, sg = O.slog_pf(A.detach().cpu().numpy())
        return (torch.as_tensor(np.asarray(la), dtype=torch.float64),
                torch.as_tensor(np.asarray(sg)).to(A.dtype))

    def pf_raw(A, layout=0):
        return torch.as_tensor(np.asarray(O.pf_product(A.detach().cpu().numpy()))).to(A.dtype)

    def grad(A, ct=None, mode="fp64", **kw):
        c = None if ct is None else ct.detach().cpu().numpy()
        return torch.as_tensor(O.slog_pf_vjp(A.detach().cpu().numpy(), c)).to(A.dtype)

    monkeypatch.setattr(api, "slog_pfaffian_raw", slog_raw)
    monkeypatch.setattr(api, "pfaffian_raw", pf_raw)
    monkeypatch.setattr(gradmod, "slog_pfaffian_grad", grad)


def skew(rng, B, n, cplx=False, scale=None):
    return torch.from_numpy(O.skew_normal(rng, B, n, scale=scale or 1 / np.sqrt(n), complex_=cplx))


@pytest.mark.parametrize("cplx", [False, True])
def test_slog_jvp_matches_reference_rule(fake_engine, cplx):
    rng = np.random.default_rng(1)
    A, E = skew(rng, 3, 40, cplx), skew(rng, 3, 40, cplx)
    (la, sg), (dla, dsg) = torch.func.jvp(lambda X: api._SlogFn.apply(X, "fp64"), (A,), (E,))
    t = O.slog_pf_jvp(A.numpy(), E.numpy())
    assert dla.dtype == torch.float64
    np.testing.assert_allclose(dla.numpy(), np.real(t), rtol=1e-12, atol=1e-12)
    if cplx:
        np.testing.assert_allclose(dsg.numpy(), sg.numpy() * 1j * np.imag(t), rtol=1e-12, atol=1e-12)
    else:
        assert torch.count_nonzero(dsg) == 0


@pytest.mark.parametrize("cplx", [False, True])
def test_slog_jvp_matches_central_differences(fake_engine, cplx):
    rng = np.random.default_rng(2)
    A, E = skew(rng, 2, 36, cplx), skew(rng, 2, 36, cplx)
    with fwAD.dual_level():
        la, sg = api._SlogFn.apply(fwAD.make_dual(A, E), "fp64")
        dla = fwAD.unpack_dual(la).tangent
        dsg = fwAD.unpack_dual(sg).tangent
    h = 1e-6
    np.testing.assert_allclose(dla.numpy(), O.fd_slog(A.numpy(), E.numpy(), h), rtol=1e-6)
    if cplx:
        sp = O.slog_pf(A.numpy() + h * E.numpy())[1]
        sm = O.slog_pf(A.numpy() - h * E.numpy())[1]
        np.testing.assert_allclose(dsg.numpy(), (sp - sm) / (2 * h), rtol=1e-5, atol=1e-8)


@pytest.mark.parametrize("cplx", [False, True])
def test_pfaffian_jvp(fake_engine, cplx):
    rng = np.random.default_rng(3)
    A, E = skew(rng, 4, 12, cplx), skew(rng, 4, 12, cplx)
    pf, dpf = torch.func.jvp(api._PfaffianFn.apply, (A,), (E,))
    want = pf.numpy() * O.slog_pf_jvp(A.numpy(), E.numpy())
    np.testing.assert_allclose(dpf.numpy(), want, rtol=1e-11, atol=1e-12)
    h = 1e-6
    fd = (O.pf_product(A.numpy() + h * E.numpy()) - O.pf_product(A.numpy() - h * E.numpy())) / (2 * h)
    np.testing.assert_allclose(dpf.numpy(), fd, rtol=1e-6, atol=1e-9)


def test_complex_backward_with_both_cotangents(fake_engine):
    """A real loss of log|Pf| and of the phase: torch's gradient g satisfies
    dL = Re(sum conj(g) dA) along any direction dA (checked by central
    differences along skew directions)."""
    rng = np.random.default_rng(4)
    A = skew(rng, 2, 20, True).requires_grad_(True)
    wl = torch.tensor([0.7, -1.3], dtype=torch.float64)
    hs = torch.tensor([0.4 - 0.9j, 1.1 + 0.2j], dtype=torch.complex128)

    def loss_np(X):
        la, sg = O.slog_pf(X)
        return float(np.sum(wl.numpy() * la) + np.sum(np.real(np.conj(hs.numpy()) * sg)))

    la, sg = api._SlogFn.apply(A, "fp64")
    L = (wl * la).sum() + (hs.conj() * sg).real.sum()
    L.backward()
    g = A.grad.numpy()
    h = 1e-6
    for _ in range(3):
        E = skew(rng, 2, 20, True).numpy()
        fd = (loss_np(A.detach().numpy() + h * E) - loss_np(A.detach().numpy() - h * E)) / (2 * h)
        got = float(np.real(np.sum(np.conj(g) * E)))
        assert abs(got - fd) <= 1e-6 * max(1.0, abs(fd)), (got, fd)


def test_real_backward_is_unchanged(fake_engine):
    rng = np.random.default_rng(5)
    A = skew(rng, 3, 34).requires_grad_(True)
    la, sg = api._SlogFn.apply(A, "fp64")
    assert not sg.requires_grad
    (la * torch.tensor([1.0, 2.0, -0.5], dtype=torch.float64)).sum().backward()
    want = O.slog_pf_vjp(A.detach().numpy(), [1.0, 2.0, -0.5])
    np.testing.assert_allclose(A.grad.numpy(), want, rtol=1e-12, atol=1e-14)


def test_torch_func_grad(fake_engine):
    """torch.func.grad reaches the adjoint through the same rule."""
    rng = np.random.default_rng(6)
    A = skew(rng, 2, 38)
    g = torch.func.grad(lambda X: api._SlogFn.apply(X, "fp64")[0].sum())(A)
    np.testing.assert_allclose(g.numpy(), O.slog_pf_vjp(A.numpy()), rtol=1e-12, atol=1e-14)
