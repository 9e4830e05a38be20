"""CPU oracle for the Pfaffian hot path.

TEST INFRASTRUCTURE ONLY.  This module is the checker: tests/, the smoke test in
__graft_entry__.py and the cpu_baseline leg of bench.py import it to produce the
values the CUDA engine is compared against.  The engine (pfcuda_b200) never
imports it and has no CPU fallback.

Contents
--------
* ctypes bindings to ``_build/libpforacle.so`` (pf_oracle.c): the log-space C
  restatement of the reference's lazy Parlett-Reid recurrence
  (src/pfaffian_cpu.cpp:22-103; pfcuda/pfaffian_py.py:17-50 for complex).
* ctypes bindings to ``_ref/libref_cpu.so``: the reference's own
  src/pfaffian_cpu.cpp, compiled unchanged, with a threaded batch driver.
* ``slog_pf_numpy``: a small pure-NumPy restatement of the same recurrence, for
  cross-checking the C restatement on tiny cases.
* Seeded input generators for the benchmark workloads and the reference's own
  known-answer constructions (test/pfaffian_test.py:12-26, 80-109).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libpforacle.so")
REF_CPU_SO = os.path.join(HERE, "_ref", "libref_cpu.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libref_gpu.so")

_i32p = ctypes.POINTER(ctypes.c_int32)
_f64p = ctypes.POINTER(ctypes.c_double)


def build():
    """Compile the checker libraries (and the reference ones when its tree is present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        L.pfo_slog_d.argtypes = [_f64p, ctypes.c_int, _f64p, _f64p, _i32p]
        L.pfo_slog_d.restype = ctypes.c_int
        L.pfo_pf_d.argtypes = [_f64p, ctypes.c_int, _i32p]
        L.pfo_pf_d.restype = ctypes.c_double
        L.pfo_slog_z.argtypes = [_f64p, ctypes.c_int, _f64p, _f64p, _i32p]
        L.pfo_slog_z.restype = ctypes.c_int
        L.pfo_pf_z.argtypes = [_f64p, ctypes.c_int, _f64p, _i32p]
        L.pfo_pf_z.restype = None
        L.pfo_slog_batch_d.argtypes = [_f64p, ctypes.c_int64, ctypes.c_int, _f64p, _f64p, _i32p]
        L.pfo_slog_batch_d.restype = ctypes.c_int
        L.pfo_slog_batch_z.argtypes = [_f64p, ctypes.c_int64, ctypes.c_int, _f64p, _f64p, _i32p]
        L.pfo_slog_batch_z.restype = ctypes.c_int
        L.pfo_pf_batch_d.argtypes = [_f64p, ctypes.c_int64, ctypes.c_int, _f64p, ctypes.c_int]
        L.pfo_pf_batch_d.restype = ctypes.c_int
        L.pfo_num_threads.argtypes = []
        L.pfo_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def ref_cpu():
    """The reference's own src/pfaffian_cpu.cpp (built by oracle/Makefile), or None."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_CPU_SO):
            return None
        L = ctypes.CDLL(REF_CPU_SO)
        L.refcpu_pfaffian.argtypes = [_f64p, ctypes.c_int]
        L.refcpu_pfaffian.restype = ctypes.c_double
        L.refcpu_pfaffian_batch.argtypes = [_f64p, ctypes.c_int64, ctypes.c_int, _f64p, ctypes.c_int]
        L.refcpu_pfaffian_batch.restype = ctypes.c_int
        _ref = L
    return _ref


def _p(a, t=_f64p):
    return a.ctypes.data_as(t)


# ----------------------------------------------------------------- oracle calls

def _as_batch(A):
    A = np.asarray(A)
    if A.ndim < 2 or A.shape[-1] != A.shape[-2]:
        raise ValueError("expected (..., n, n) matrices")
    n = A.shape[-1]
    lead = A.shape[:-2]
    return A.reshape((int(np.prod(lead, dtype=np.int64)), n, n)), n, lead


def slog_pf(A, with_pivots=False):
    """(log|Pf|, sign) per matrix of a (..., n, n) array, computed in FP64 / C128.

    Real inputs (f32 or f64) are evaluated in float64, complex inputs (c64 or
    c128) in complex128.  ``sign`` is +-1 (real) or a unit complex phase; a
    singular or odd-sized matrix gives (-inf, 0).  With ``with_pivots`` the
    column index chosen at each pivot step is returned as well (n//2 per matrix).
    """
    Ab, n, lead = _as_batch(A)
    B = Ab.shape[0]
    L = lib()
    la = np.empty(B, np.float64)
    piv = np.zeros((B, max(n // 2, 1)), np.int32)
    if np.iscomplexobj(Ab):
        X = np.ascontiguousarray(Ab, dtype=np.complex128)
        ph = np.empty(2 * B, np.float64)
        L.pfo_slog_batch_z(_p(X.view(np.float64)), B, n, _p(la), _p(ph), _p(piv, _i32p))
        sign = ph[0::2] + 1j * ph[1::2]
    else:
        X = np.ascontiguousarray(Ab, dtype=np.float64)
        sign = np.empty(B, np.float64)
        L.pfo_slog_batch_d(_p(X), B, n, _p(la), _p(sign), _p(piv, _i32p))
    la = la.reshape(lead)
    sign = sign.reshape(lead)
    if with_pivots:
        return la, sign, piv[:, : n // 2].reshape(lead + (n // 2,))
    return la, sign


def slog_pf_list(mats):
    """slog_pf of each matrix of a list of square matrices of any orders:
    (log|Pf|, sign) as two float64 arrays (real input)."""
    la = np.empty(len(mats))
    sg = np.empty(len(mats))
    for i, M in enumerate(mats):
        l_, s_ = slog_pf(np.asarray(M)[None])
        la[i], sg[i] = l_[0], s_[0]
    return la, sg


def pf_product(A, as_shipped=False):
    """Plain product Pf per matrix (the value the reference returns), in FP64 / C128.

    Pivots are chosen on the updated row, as pfcuda/pfaffian_py.py:29-32 and
    src/pfaffian_sm.cu:29-46 do.  ``as_shipped`` (real only) reproduces
    src/pfaffian_cpu.cpp bit for bit instead, including its closed forms for
    n = 2, 4 and its argmax that starts from the value of A[k][k+1] read before
    the lazy update (pfaffian_cpu.cpp:29-30)."""
    Ab, n, lead = _as_batch(A)
    B = Ab.shape[0]
    L = lib()
    if np.iscomplexobj(Ab):
        out = np.empty(B, np.complex128)
        o2 = np.empty(2, np.float64)
        for b in range(B):
            S = np.ascontiguousarray(Ab[b], dtype=np.complex128).copy()
            L.pfo_pf_z(_p(S.view(np.float64)), n, _p(o2), None)
            out[b] = o2[0] + 1j * o2[1]
    else:
        X = np.ascontiguousarray(Ab, dtype=np.float64)
        out = np.empty(B, np.float64)
        L.pfo_pf_batch_d(_p(X), B, n, _p(out), 1 if as_shipped else 0)
    return out.reshape(lead)


def ref_cpu_pfaffian(A, threads=0):
    """Run the reference's own pfaffian_cpu on each (row-major float64) matrix."""
    R = ref_cpu()
    if R is None:
        raise RuntimeError("oracle/_ref/libref_cpu.so is not built")
    Ab, n, lead = _as_batch(A)
    X = np.ascontiguousarray(Ab, dtype=np.float64)
    out = np.empty(X.shape[0], np.float64)
    R.refcpu_pfaffian_batch(_p(X), X.shape[0], n, _p(out), threads)
    return out.reshape(lead)


# ----------------------------------------------------------- NumPy restatement

def slog_pf_numpy(A):
    """Pure-NumPy restatement of the lazy recurrence (pfcuda/pfaffian_py.py:17-50),
    in log space; one matrix, any dtype.  Slow; for cross-checks on small n."""
    A = np.array(A, dtype=np.complex128 if np.iscomplexobj(A) else np.float64)
    n = A.shape[0]
    if n == 0 or n % 2:
        return -np.inf, 0.0 * A.dtype.type(1)
    la = 0.0
    sg = A.dtype.type(1)
    V = A[0::2, :]            # rows holding the scaled Gauss vectors
    W = A[1::2, :]            # rows holding the negated updated rows

    def dR(i, k):
        return V[:i, k] @ W[:i, k + 1:] - W[:i, k] @ V[:i, k + 1:]

    for i, k in enumerate(range(0, n - 1, 2)):
        Ak = A[k, k + 1:]
        Ak += dR(i, k)
        km = int(np.abs(Ak).argmax())
        if Ak[km] == 0:
            return -np.inf, 0.0 * sg
        if km != 0:
            kp = k + 1 + km
            A[[k + 1, kp], :] = A[[kp, k + 1], :]
            A[:, [k + 1, kp]] = A[:, [kp, k + 1]]
            sg = -sg
        A[k + 1, k + 2:] = -(A[k + 1, k + 2:] + dR(i, k + 1))
        p = Ak[0]
        la += np.log(np.abs(p))
        sg = sg * (p / np.abs(p))
        Ak[1:] /= p
    return la, sg


# ------------------------------------------------------------------ generators

def skew_normal(rng, B, n, scale=1.0, complex_=False, halve=True):
    """A = (G - G^T)/2 (or G - G^T when ``halve`` is False) with G ~ N(0, scale^2);
    complex inputs draw real and imaginary parts independently."""
    shape = (B, n, n)
    G = rng.normal(scale=scale, size=shape)
    if complex_:
        G = G + 1j * rng.normal(scale=scale, size=shape)
    A = G - np.swapaxes(G, -1, -2)
    return A / 2 if halve else A


def config_small(seed=0, B=4096, n=32):
    """4096 independent 32x32 float64 matrices A=(G-G^T)/2, G_ij ~ N(0,1), seed 0."""
    rng = np.random.default_rng(seed)
    return skew_normal(rng, B, n)


def config_large(n, dtype=np.float64, seed=1, B=1):
    """Single large matrices, entries (real and imaginary parts) N(0, 1/n) in G,
    A=(G-G^T)/2; n is the matrix order 2n."""
    rng = np.random.default_rng(seed)
    cplx = np.dtype(dtype).kind == "c"
    A = skew_normal(rng, B, n, scale=1.0 / np.sqrt(n), complex_=cplx)
    return A.astype(dtype)


def config_ragged(seed=2, count=2000, lo=8, hi=512):
    """Even sizes drawn uniformly from [lo, hi], entries N(0, 1/n): one list per dtype."""
    rng = np.random.default_rng(seed)
    evens = np.arange(lo, hi + 1, 2)
    out = {}
    for dt in (np.float32, np.float64):
        sizes = rng.choice(evens, size=count)
        mats = []
        for n in sizes:
            G = rng.normal(scale=1.0 / np.sqrt(n), size=(n, n))
            mats.append(((G - G.T) / 2).astype(dt))
        out[np.dtype(dt).name] = mats
    return out


def config_grad(seed=3, B=256, n=512):
    """256 complex128 matrices of order 512, real and imaginary parts N(0, 1/n)."""
    rng = np.random.default_rng(seed)
    return skew_normal(rng, B, n, scale=1.0 / np.sqrt(n), complex_=True)


def haar_orthogonal(rng, n):
    """Haar orthogonal Q, sign-fixed as in test/pfaffian_test.py:18-26."""
    Q, R = np.linalg.qr(rng.normal(size=(n, n)))
    return Q * np.sign(np.diag(R))


def config_illcond(seed=4, B=64, n=2048, dtype=np.float64, return_q=False):
    """A = Q blockdiag(s_k J) Q^T, s_k log-spaced in [1e-6, 1]; returns (A, exact
    log|Pf| = sum log s_k, exact sign = det Q) per matrix, and with ``return_q``
    the Haar factors Q as well (for the exact inverse, illcond_half_inv_t)."""
    rng = np.random.default_rng(seed)
    s = np.logspace(-6, 0, n // 2)
    D = np.zeros((n, n))
    idx = np.arange(0, n, 2)
    D[idx, idx + 1] = s
    D[idx + 1, idx] = -s
    As, logs, signs, Qs = [], [], [], []
    for _ in range(B):
        Q = haar_orthogonal(rng, n)
        A = Q @ D @ Q.T
        A = (A - A.T) / 2
        As.append(A.astype(dtype))
        logs.append(np.sum(np.log(s)))
        signs.append(np.sign(np.linalg.det(Q)))
        if return_q:
            Qs.append(Q)
    out = (np.stack(As), np.array(logs), np.array(signs))
    return out + (np.stack(Qs),) if return_q else out


def illcond_half_inv_t(Q):
    """The exact d log Pf / dA = (1/2) A^-T of config_illcond's construction:
    A^-1 = Q blockdiag(-J / s_k) Q^T (J^-1 = -J), so (1/2) A^-T = -(1/2) A^-1 =
    (1/2) Q blockdiag(J / s_k) Q^T, formed in float64 from the stored Q."""
    Q = np.asarray(Q, dtype=np.float64)
    n = Q.shape[-1]
    s = np.logspace(-6, 0, n // 2)
    idx = np.arange(0, n, 2)
    # Q blockdiag(J / s) Q^T = sum_k (q_2k q_2k+1^T - q_2k+1 q_2k^T) / s_k
    Qe = Q[..., :, idx] / s
    Qo = Q[..., :, idx + 1]
    M = Qe @ np.swapaxes(Qo, -1, -2)
    return 0.5 * (M - np.swapaxes(M, -1, -2))


def tridiag_known(rng, n):
    """Known-answer construction of test/pfaffian_test.py:80-103: a tridiagonal
    skew matrix with superdiagonal 1+N(0,1) on even positions, conjugated by a
    Haar orthogonal B.  Returns (B A B^T, exact Pf = det(B) * prod(even diag))."""
    alt = 1.0 + rng.normal(size=(n - 1,))
    alt = alt * (1 - (np.arange(n - 1) % 2))
    A = np.diag(alt, k=1) - np.diag(alt, k=-1)
    Bq = haar_orthogonal(rng, n)
    pf = np.linalg.det(Bq) * np.prod(alt[0::2])
    return Bq @ A @ Bq.T, pf


# ------------------------------------------------------------- derivatives

def slog_pf_jvp(A, Adot):
    """Tangent of log|Pf| by the reference's rule slog_pfaffian_jvp
    (pfcuda/cuda_api.py:92-107): (1/2) tr(A^-1 Adot), with a general inverse
    (NumPy's LU, standing in for jnp.linalg.inv).  Complex for complex input;
    its real part is the derivative of log|Pf|."""
    A = np.asarray(A)
    Ainv = np.linalg.inv(A.astype(np.complex128 if np.iscomplexobj(A) else np.float64))
    return 0.5 * np.einsum("...ij,...ji->...", Ainv, np.asarray(Adot))


def slog_pf_vjp(A, ct=None):
    """The adjoint of the same rule: ct * (1/2) A^-T per matrix (holomorphic,
    unconjugated), so that sum(G * Adot) equals slog_pf_jvp(A, Adot) * ct."""
    A = np.asarray(A)
    Ainv = np.linalg.inv(A.astype(np.complex128 if np.iscomplexobj(A) else np.float64))
    G = 0.5 * np.swapaxes(Ainv, -1, -2)
    if ct is not None:
        G = G * np.asarray(ct, dtype=np.float64)[..., None, None]
    return G


def fd_slog(A, E, h=1e-6):
    """Central difference of log|Pf| along the direction E, (f(A+hE) - f(A-hE)) / 2h,
    with log|Pf| from the C restatement in FP64 / C128."""
    lp, _ = slog_pf(np.asarray(A) + h * np.asarray(E))
    lm, _ = slog_pf(np.asarray(A) - h * np.asarray(E))
    return (lp - lm) / (2 * h)
