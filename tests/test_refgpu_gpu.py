"""The engine against the reference's own CUDA kernels, run on the same GPU.

oracle/_ref/libref_gpu.so is the reference's src/*.cu compiled unchanged for
sm_100a (oracle/Makefile) with a C shim that replays its XLA handlers.  The
reference takes each matrix column-major (pfcuda/cuda_api.py:50); the engine is
called on the same buffers with PFB_COL_MAJOR.

The reference differs from the engine in pivoting details -- a zero threshold of
10 eps (include/pfaffian_utils.cuh:22-29) and, in the large path, an argmax whose
second pass re-reads the matrix row instead of the block results
(src/slog_pfaffian_lg.cu:175-176), which restricts the pivot search when more
than 256 columns remain -- so values agree to rounding, not bit for bit.
"""
import ctypes
import os

import numpy as np
import pytest
import torch

import pfcuda_b200 as pf
from pfcuda_b200 import _lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def refgpu():
    if not os.path.exists(O.REF_GPU_SO):
        pytest.skip("oracle/_ref/libref_gpu.so not built")
    L = ctypes.CDLL(O.REF_GPU_SO)
    for name in ("refgpu_pfaffian_f32", "refgpu_pfaffian_f64", "refgpu_pfaffian_c64", "refgpu_pfaffian_c128"):
        getattr(L, name).argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    for name in ("refgpu_slog_f32", "refgpu_slog_f64", "refgpu_slog_c64", "refgpu_slog_c128"):
        getattr(L, name).argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return L


def colmajor(A):
    return torch.from_numpy(np.ascontiguousarray(np.swapaxes(A, -1, -2))).cuda()


@pytest.mark.parametrize("npdt,fn", [(np.float64, "refgpu_pfaffian_f64"), (np.complex128, "refgpu_pfaffian_c128")])
def test_small_path_vs_reference_kernel(npdt, fn):
    L = refgpu()
    A = O.config_small(seed=0)[:512].astype(npdt)
    if np.dtype(npdt).kind == "c":
        A = A + 1j * O.config_small(seed=10)[:512]
    X = colmajor(A)
    ref = torch.empty(A.shape[0], dtype=X.dtype, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    assert getattr(L, fn)(X.data_ptr(), A.shape[0], 32, ref.data_ptr(), s) == 0
    ours = pf.pfaffian_raw(X, _lib.COL_MAJOR)
    torch.cuda.synchronize()
    r, o = ref.cpu().numpy(), ours.cpu().numpy()
    assert np.max(np.abs(r - o) / np.abs(r)) < 1e-10


@pytest.mark.parametrize("n", [64, 128, 250, 290])
def test_large_path_vs_reference_kernel(n):
    L = refgpu()
    A = O.config_large(n, seed=3, B=2)
    X = colmajor(A)
    log = torch.empty(2, dtype=torch.float64, device="cuda")
    ph = torch.empty(2, dtype=torch.float64, device="cuda")
    tmp = torch.empty(n * n, dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    assert L.refgpu_slog_f64(X.data_ptr(), 2, n, log.data_ptr(), ph.data_ptr(), tmp.data_ptr(), s) == 0
    la, sg = pf.slog_pfaffian_raw(X, mode="fp64", layout=_lib.COL_MAJOR)
    torch.cuda.synchronize()
    # The reference's slog kernels see the matrix column-major and return the
    # log and the sign of that matrix; its argmax restriction above 256 columns
    # costs accuracy, hence the looser bound there.
    tol = 1e-10 if n <= 257 else 1e-8
    assert np.all(np.abs(log.cpu().numpy() - la.cpu().numpy()) <= tol * np.abs(la.cpu().numpy()))
    assert np.array_equal(np.sign(ph.cpu().numpy()), sg.cpu().numpy())


@pytest.mark.parametrize("npdt,fn", [(np.float32, "refgpu_pfaffian_f32"), (np.complex64, "refgpu_pfaffian_c64")])
def test_small_path_single_precision_vs_reference_kernel(npdt, fn):
    """Both single-precision kernels against the FP64 oracle on the same
    rounded inputs: the engine within 0.5 n eps32 cond_2(A) per matrix (the
    bar of test_small_gpu.py), the reference (built with --use_fast_math,
    CMakeLists.txt:47-50) within four times that."""
    L = refgpu()
    cplx = np.dtype(npdt).kind == "c"
    A = O.config_small(seed=1)[:512]
    if cplx:
        A = A + 1j * O.config_small(seed=11)[:512]
    A = A.astype(npdt)
    X = colmajor(A)
    ref = torch.empty(A.shape[0], dtype=X.dtype, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    assert getattr(L, fn)(X.data_ptr(), A.shape[0], 32, ref.data_ptr(), s) == 0
    ours = pf.pfaffian_raw(X, _lib.COL_MAJOR)
    torch.cuda.synchronize()
    want = O.pf_product(A.astype(np.complex128 if cplx else np.float64))
    bar = 0.5 * 32 * np.finfo(np.float32).eps * np.linalg.cond(A.astype(np.complex128))
    rel = lambda x: np.abs(x - want) / np.abs(want)
    assert np.all(rel(ours.cpu().numpy()) <= bar)
    assert np.all(rel(ref.cpu().numpy()) <= 4 * bar)


@pytest.mark.parametrize("npdt,fn", [(np.float32, "refgpu_slog_f32"), (np.complex64, "refgpu_slog_c64"),
                                     (np.complex128, "refgpu_slog_c128")])
def test_large_path_other_dtypes_vs_reference_kernel(npdt, fn):
    """slog_pfaffian on float32, complex64 and complex128 against the
    reference's kernels (orders below the 256-column argmax restriction).  The
    reference works in the input precision and returns a float32 log for
    float32 / complex64 (ProjectionType, include/pfaffian_utils.cuh:13-15);
    the engine works in FP64 / complex128 from the same values."""
    L = refgpu()
    cplx = np.dtype(npdt).kind == "c"
    n = 128
    A = O.config_large(n, dtype=npdt, seed=3, B=2)
    X = colmajor(A)
    single = np.dtype(npdt) in (np.dtype(np.float32), np.dtype(np.complex64))
    log = torch.empty(2, dtype=torch.float32 if single else torch.float64, device="cuda")
    ph = torch.empty(2, dtype=X.dtype, device="cuda")
    tmp = torch.empty(n * n, dtype=X.dtype, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    assert getattr(L, fn)(X.data_ptr(), 2, n, log.data_ptr(), ph.data_ptr(), tmp.data_ptr(), s) == 0
    la, sg = pf.slog_pfaffian_raw(X, mode="fp64", layout=_lib.COL_MAJOR)
    torch.cuda.synchronize()
    rl, rp = log.cpu().numpy().astype(np.float64), ph.cpu().numpy()
    la, sg = la.cpu().numpy(), sg.cpu().numpy()
    wl, ws = O.slog_pf(A.astype(np.complex128 if cplx else np.float64))   # the matrix both see
    assert np.all(np.abs(la - wl) <= 1e-10 * np.abs(wl))            # the engine: the FP64 bar
    if single:
        assert np.all(np.abs(rl - la) <= 1e-4 * np.abs(la) + 1e-3)
        assert np.all(np.abs(rp.astype(np.complex128) - sg) <= 1e-3)
    else:
        assert np.all(np.abs(rl - la) <= 1e-10 * np.abs(la))
        assert np.all(np.abs(rp - sg) <= 1e-9)
