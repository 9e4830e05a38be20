"""Small path (pfb_pfaffian, n <= 32) against the oracle and the reference's own values.

Tolerances: float64 / complex128 results agree with the FP64 oracle to a
relative 1e-10 (the reference's own tests use rtol 1e-8 for Pf^2 = det and 1e-10
for the exact-answer construction, test/pfaffian_test.py:65,105-110); float32 /
complex64 are computed in single precision like the reference and are held to
a relative 2e-3 per matrix.
"""
import numpy as np
import pytest
import torch

import pfcuda_b200 as pf
from pfcuda_b200 import _lib
from oracle import oracle as O
from golden_io import load, split

pytestmark = pytest.mark.gpu

DTYPES = {np.float32: torch.float32, np.float64: torch.float64,
          np.complex64: torch.complex64, np.complex128: torch.complex128}


def cuda(a):
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def rel_err(got, want):
    return np.abs(got - want) / np.maximum(np.abs(want), 1e-300)


def test_benchmark_batch_matches_oracle():
    A = O.config_small(seed=0)                       # 4096 x 32 x 32 float64
    got = pf.pfaffian(cuda(A)).cpu().numpy()
    want = O.pf_product(A)
    assert np.max(rel_err(got, want)) < 1e-10
    g = load("cpu_f64.npz")                          # reference pfaffian_cpu, as shipped
    assert np.array_equal(g["bench_A"], A[:64])
    assert np.max(rel_err(got[:64], g["bench_pf"])) < 1e-10


@pytest.mark.parametrize("npdt", list(DTYPES))
@pytest.mark.parametrize("n", [2, 4, 6, 8, 10, 14, 16, 18, 24, 30, 32])
def test_all_orders_and_dtypes(npdt, n):
    rng = np.random.default_rng(1000 + n)
    cplx = np.dtype(npdt).kind == "c"
    A = O.skew_normal(rng, 37, n, complex_=cplx).astype(npdt)   # 37: partial warps
    got = pfaffian_raw_np(A)
    want = O.pf_product(A.astype(np.complex128 if cplx else np.float64))
    if np.dtype(npdt).itemsize * (1 if not cplx else 0.5) >= 8:
        assert np.max(rel_err(got, want)) < 1e-10, (n, npdt)
    else:
        # single precision: a per-matrix bar from the conditioning of each
        # matrix, 0.5 n eps32 cond_2(A) -- a float32 emulation of the same
        # elimination on 1600 random matrices per dtype stays below
        # 0.09 n eps32 cond_2(A); the FP64 oracle runs on the same rounded input
        eps = np.finfo(np.float32).eps
        bar = 0.5 * n * eps * np.linalg.cond(A.astype(np.complex128))
        assert np.all(rel_err(got, want) <= bar), (n, npdt, np.max(rel_err(got, want) / bar))


def pfaffian_raw_np(A, layout=_lib.ROW_MAJOR):
    return pf.pfaffian_raw(cuda(A), layout).cpu().numpy()


@pytest.mark.parametrize("n", [6, 16, 22, 32])
def test_column_major_layout(n):
    rng = np.random.default_rng(n)
    A = O.skew_normal(rng, 9, n)
    At = np.ascontiguousarray(np.swapaxes(A, -1, -2))   # each matrix stored column-major
    np.testing.assert_array_equal(pfaffian_raw_np(At, _lib.COL_MAJOR), pfaffian_raw_np(A))


def test_reference_golden_values():
    g = load("cpu_f64.npz")
    mats = split(g["sizes_A"], g["sizes_n"])
    for A, want in zip(mats, g["sizes_pf"]):
        got = pf.pfaffian(cuda(A)).item()
        assert abs(got - want) <= 1e-10 * abs(want) + 1e-300


def test_reference_numpy_path_complex():
    g = load("py_c128.npz")
    for A, want in zip(split(g["A"], g["n"]), g["pf"]):
        if A.shape[0] > 32:
            continue
        got = pf.pfaffian(cuda(A)).item()
        assert abs(got - want) <= 1e-10 * abs(want)


# --- the reference's own test cases (test/pfaffian_test.py), restated

def test_zero_matrix():
    for n in range(2, 20, 2):
        assert pf.pfaffian(cuda(np.zeros((n, n)))).item() == 0.0


def test_odd_dimension():
    rng = np.random.default_rng(0)
    for n in [1, 3, 5, 11, 15]:
        G = rng.normal(size=(n, n))
        assert pf.pfaffian(cuda(G - G.T)).item() == 0.0


def test_det_relation():
    rng = np.random.default_rng(1)
    for n in range(2, 33, 2):
        G = rng.normal(size=(n, n))
        A = G - G.T
        p = pf.pfaffian(cuda(A)).item()
        assert np.isclose(p * p, np.linalg.det(A), rtol=1e-8, atol=1e-10)


def test_random_against_oracle():
    rng = np.random.default_rng(123)
    for n in range(2, 33, 2):
        G = rng.normal(size=(20, n, n))
        A = G - np.swapaxes(G, -1, -2)
        np.testing.assert_allclose(pf.pfaffian(cuda(A)).cpu().numpy(), O.pf_product(A), rtol=1e-8, atol=1e-10)


def test_by_identity():
    g = load("known.npz")
    for A, want in zip(split(g["A"], g["n"]), g["pf"]):
        if A.shape[0] > 32:
            continue
        assert np.isclose(pf.pfaffian(cuda(A)).item(), want, rtol=1e-10, atol=1e-12)


def test_singular_and_nan():
    rng = np.random.default_rng(5)
    A = O.skew_normal(rng, 4, 12)
    A[1, 3, :] = 0
    A[1, :, 3] = 0
    A[2, 5, 7] = np.nan
    A[2, 7, 5] = np.nan
    got = pfaffian_raw_np(A)
    assert got[1] == 0.0 and np.isnan(got[2]) and np.isfinite(got[0]) and np.isfinite(got[3])


def test_slog_entry_for_small_orders():
    rng = np.random.default_rng(8)
    for npdt in (np.float64, np.complex128):
        A = O.skew_normal(rng, 50, 20, complex_=np.dtype(npdt).kind == "c").astype(npdt)
        la, sg = pf.slog_pfaffian_raw(cuda(A), mode="fp64")
        wl, ws = O.slog_pf(A)
        assert np.max(np.abs(la.cpu().numpy() - wl)) < 1e-11
        assert np.max(np.abs(sg.cpu().numpy() - ws)) < 1e-11


def test_gradient_of_pfaffian():
    rng = np.random.default_rng(9)
    A = O.skew_normal(rng, 1, 12)[0]
    X = cuda(A).requires_grad_(True)
    y = pf.pfaffian(X)
    y.backward()
    # d Pf / dA along a skew direction E equals <grad, E>
    G = rng.normal(size=(12, 12))
    E = G - G.T
    h = 1e-6
    fd = (O.pf_product(A + h * E) - O.pf_product(A - h * E)) / (2 * h)
    assert np.isclose(np.sum(X.grad.cpu().numpy() * E), fd, rtol=1e-6)
