"""Python API of the engine, mirroring pfcuda/cuda_api.py.

``pfaffian(A)`` and ``slog_pfaffian(A)`` keep the reference's names, argument
meaning, shape rules and error behaviour (pfcuda/cuda_api.py:27-76); the host
framework here is PyTorch (JAX is not part of this engine's runtime), so inputs
are torch tensors on a CUDA device, with any leading batch dimensions standing
in for jax.vmap (the reference registers vmap_method='broadcast_all',
cuda_api.py:51,73).  NumPy arrays are accepted too: they are copied to the
current CUDA device and the result comes back as NumPy.

Differentiation mirrors the reference's JVP rules (cuda_api.py:78-107): the
tangent of log|Pf| is (1/2) tr(A^-1 dA) and the tangent of Pf is that times Pf.
``slog_pfaffian`` is a torch.autograd.Function whose backward is the engine's
adjoint kernel (pfcuda_b200.grad).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

_DT = {
    torch.float32: _lib.F32,
    torch.float64: _lib.F64,
    torch.complex64: _lib.C64,
    torch.complex128: _lib.C128,
}
_MODES = {"fp64": _lib.MODE_FP64, "split": _lib.MODE_SPLIT}


def _stream(t: torch.Tensor) -> int:
    return torch.cuda.current_stream(t.device).cuda_stream


def _prep(A):
    """torch CUDA tensor (contiguous) and a flag telling to return NumPy."""
    as_np = isinstance(A, np.ndarray)
    if as_np:
        A = torch.from_numpy(np.ascontiguousarray(A))
    if not isinstance(A, torch.Tensor):
        raise TypeError("expected a torch.Tensor or numpy.ndarray")
    if A.ndim < 2 or A.shape[-1] != A.shape[-2]:
        raise ValueError(f"expected (..., n, n) matrices, got shape {tuple(A.shape)}")
    if A.dtype not in _DT:
        raise TypeError(f"unsupported dtype {A.dtype}; use float32, float64, complex64 or complex128")
    return A, as_np


def _out(x, as_np):
    return x.cpu().numpy() if as_np else x


def _to_device(A, as_np):
    """NumPy input goes to the current CUDA device; a CPU torch tensor is refused
    (the engine has no CPU fallback)."""
    if as_np:
        return A.cuda()
    if not A.is_cuda:
        raise ValueError("the engine runs on CUDA tensors only (no CPU fallback)")
    return A


def pfaffian(A):
    """Pf(A) for 2n <= 32 (pfcuda/cuda_api.py:27-54).

    Odd or empty order gives 0; 2x2 and 4x4 use the closed forms (cuda_api.py:
    34-42); orders above 32 raise ValueError (cuda_api.py:44-45).
    """
    A, as_np = _prep(A)
    n = A.shape[-1]
    if n == 0 or n & 1:
        return _out(torch.zeros(A.shape[:-2], dtype=A.dtype, device=A.device), as_np)
    if n == 2:
        return _out(A[..., 0, 1].clone(), as_np)
    if n == 4:
        return _out(A[..., 0, 1] * A[..., 2, 3] - A[..., 0, 2] * A[..., 1, 3]
                    + A[..., 0, 3] * A[..., 1, 2], as_np)
    if n > 32:
        raise ValueError("Matrix size exceeds the maximum supported size of 32x32.")
    A = _to_device(A, as_np)
    return _out(_PfaffianFn.apply(A.contiguous()), as_np)


_TUNED = None


def _tuned_entries():
    """The measured entries of pfcuda_b200/tune_table.json (loaded once)."""
    global _TUNED
    if _TUNED is None:
        import json
        import os
        try:
            with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "tune_table.json")) as f:
                _TUNED = json.load(f).get("entries", [])
        except (OSError, ValueError):
            _TUNED = []
    return _TUNED


def resolve_mode(mode: str, dtype: torch.dtype, n: int | None = None, batch: int | None = None) -> str:
    """"auto" -> the faster trailing update for this dtype class, order and
    batch by the tuned table's measurements (both modes meet the 1e-10 bar on
    log|Pf|), else the defaults: "split" for real inputs, "fp64" for complex
    ones (the complex split update's int8 products are twice as deep)."""
    if mode == "auto":
        cplx = dtype in (torch.complex64, torch.complex128)
        if n is not None and batch is not None:
            cls = "complex" if cplx else "real"
            ms = {}
            for e in _tuned_entries():
                if (e.get("dtype") == cls and e["n_min"] <= n <= e["n_max"]
                        and e["batch_min"] <= batch <= e["batch_max"] and "ms" in e):
                    ms.setdefault(e["mode"], e["ms"])
            if "split" in ms and "fp64" in ms:
                return "split" if ms["split"] <= ms["fp64"] else "fp64"
        return "fp64" if cplx else "split"
    if mode not in _MODES:
        raise ValueError(f"mode must be 'auto' or one of {sorted(_MODES)}")
    return mode


def slog_pfaffian(A, mode: str = "auto"):
    """(log|Pf(A)|, sign) for 2n > 32 (pfcuda/cuda_api.py:56-76).

    Orders up to 32 raise ValueError (cuda_api.py:60-61); odd order returns
    (-inf, 0) (cuda_api.py:63-67).  The log is float64 (cuda_api.py:71); the sign
    has A's dtype (a unit-modulus phase for complex A, 0 when Pf = 0).
    ``mode`` picks the arithmetic of the trailing update: "split" (int8 slices on
    the tensor cores, recombined in FP64), "fp64" (the FP64 tensor cores), or
    "auto" (resolve_mode: the faster of the two by the tuned table's
    measurements for this dtype, order and batch).
    """
    A, as_np = _prep(A)
    n = A.shape[-1]
    if n <= 32:
        raise ValueError("Matrix size is less than the minimum supported size of (33x33). "
                         "Use pfaffian() for smaller matrices.")
    if n & 1:
        lead = A.shape[:-2]
        la = torch.full(lead, -float("inf"), dtype=torch.float64, device=A.device)
        sg = torch.zeros(lead, dtype=A.dtype, device=A.device)
        return _out(la, as_np), _out(sg, as_np)
    mode = resolve_mode(mode, A.dtype, n, int(np.prod(A.shape[:-2])) if A.ndim > 2 else 1)
    A = _to_device(A, as_np)
    la, sg = _SlogFn.apply(A.contiguous(), mode)
    return _out(la, as_np), _out(sg, as_np)


# ------------------------------------------------------------------ raw calls

def pfaffian_raw(A: torch.Tensor, layout: int = _lib.ROW_MAJOR) -> torch.Tensor:
    """One pfb_pfaffian call on a contiguous (..., n, n) CUDA tensor (n <= 32)."""
    n = A.shape[-1]
    B = A.numel() // max(n * n, 1) if n else int(np.prod(A.shape[:-2]))
    out = torch.empty(A.shape[:-2], dtype=A.dtype, device=A.device)
    st = _lib.lib().pfb_pfaffian(_DT[A.dtype], A.data_ptr(), B, n, layout, out.data_ptr(), _stream(A))
    _lib.check(st, "pfb_pfaffian")
    return out


def slog_workspace_bytes(dtype: torch.dtype, batch: int, n: int, mode: str = "split") -> int:
    return int(_lib.lib().pfb_slog_workspace_bytes(_DT[dtype], batch, n, _MODES[mode]))


def _config(config):
    """A pfb_slog_config from a dict (panel: "registers" | "half_shared" | 1 | 2,
    slices: 1..7, ranges: 1 | 2, epilogue: "roundtrip" | "reduce" | "direct" | 1..3;
    missing keys take the tuned table's choice)."""
    if config is None:
        return None
    panel = config.get("panel", 0)
    panel = {"registers": _lib.PANEL_REGISTERS, "half_shared": _lib.PANEL_HALF_SHARED}.get(panel, panel)
    epi = config.get("epilogue", 0)
    epi = {"roundtrip": _lib.EPILOGUE_ROUNDTRIP, "reduce": _lib.EPILOGUE_REDUCE,
           "direct": _lib.EPILOGUE_DIRECT}.get(epi, epi)
    return _lib.SlogConfig(int(panel), int(config.get("slices", 0)), int(config.get("ranges", 0)), int(epi))


def slog_config(dtype: torch.dtype, batch: int, n: int, mode: str = "split") -> dict:
    """The configuration (panel form, split digits, stream ranges) that the
    tuned table picks for a pfb_slog_pfaffian call on these arguments."""
    c = _lib.SlogConfig()
    _lib.check(_lib.lib().pfb_slog_config_for(_DT[dtype], batch, n, _MODES[mode], ctypes.byref(c)),
               "pfb_slog_config_for")
    return c.as_dict()


def slog_pfaffian_raw(A: torch.Tensor, mode: str = "split", layout: int = _lib.ROW_MAJOR,
                      workspace: torch.Tensor | None = None, return_pivots: bool = False,
                      config: dict | None = None):
    """One pfb_slog_pfaffian call on a contiguous (..., n, n) CUDA tensor, any even n.

    ``config`` overrides the tuned table's settings (see ``slog_config``)."""
    n = A.shape[-1]
    lead = A.shape[:-2]
    B = int(np.prod(lead)) if len(lead) else 1
    la = torch.empty(lead, dtype=torch.float64, device=A.device)
    sg = torch.empty(lead, dtype=A.dtype, device=A.device)
    wsb = slog_workspace_bytes(A.dtype, B, n, mode)
    if workspace is None or workspace.numel() < wsb:
        workspace = torch.empty(max(wsb, 1), dtype=torch.uint8, device=A.device)
    cfg = _config(config)
    st = _lib.lib().pfb_slog_pfaffian_ex(_DT[A.dtype], A.data_ptr(), B, n, layout, _MODES[mode],
                                         la.data_ptr(), sg.data_ptr(), workspace.data_ptr(), wsb,
                                         _stream(A), None, ctypes.byref(cfg) if cfg is not None else None)
    _lib.check(st, "pfb_slog_pfaffian")
    if return_pivots:
        piv = torch.empty(lead + (n // 2,), dtype=torch.int32, device=A.device)
        st = _lib.lib().pfb_slog_pivots(B, n, workspace.data_ptr(), wsb, piv.data_ptr(), _stream(A))
        _lib.check(st, "pfb_slog_pivots")
        return la, sg, piv
    return la, sg


def upload_upper(A_host: torch.Tensor, out: torch.Tensor | None = None,
                 device: torch.device | None = None) -> torch.Tensor:
    """Copy a contiguous (..., n, n) host batch to the device moving only what
    ``slog_pfaffian`` reads: the upper triangle (diagonal included) of each
    matrix's row-major view, in 256-row rectangles (pfb_upload_upper), about
    half the bytes of a full copy.  Entries below the diagonal of the result
    are left as they were in ``out`` (uninitialised for a new tensor) and are
    never read by the large path; orders n <= 32 are copied whole.  The copies
    are enqueued on the current stream and are asynchronous when ``A_host`` is
    page-locked (``tensor.pin_memory()``)."""
    if A_host.is_cuda:
        raise ValueError("upload_upper copies from host memory")
    if A_host.ndim < 2 or A_host.shape[-1] != A_host.shape[-2]:
        raise ValueError(f"expected (..., n, n) matrices, got shape {tuple(A_host.shape)}")
    if A_host.dtype not in _DT:
        raise TypeError(f"unsupported dtype {A_host.dtype}")
    if not A_host.is_contiguous():
        raise ValueError("the host batch must be contiguous")
    if out is None:
        out = torch.empty(A_host.shape, dtype=A_host.dtype,
                          device=device if device is not None else torch.device("cuda"))
    elif out.shape != A_host.shape or out.dtype != A_host.dtype or not out.is_cuda or not out.is_contiguous():
        raise ValueError("out must be a contiguous CUDA tensor of the host batch's shape and dtype")
    n = A_host.shape[-1]
    B = int(np.prod(A_host.shape[:-2])) if A_host.ndim > 2 else 1
    st = _lib.lib().pfb_upload_upper(_DT[A_host.dtype], A_host.data_ptr(), out.data_ptr(), B, n, _stream(out))
    _lib.check(st, "pfb_upload_upper")
    return out


def upload_upper_bytes(dtype: torch.dtype, batch: int, n: int) -> int:
    """Bytes ``upload_upper`` moves for a batch of `batch` n x n matrices."""
    return int(_lib.lib().pfb_upload_upper_bytes(_DT[dtype], batch, n))


# ------------------------------------------------------------- ragged batches

class RaggedPlan:
    """A ragged batch prepared once and run many times.

    ``mats`` is a list of square CUDA tensors (float32 or float64, row-major
    unless ``layout`` says otherwise) of any orders.  Orders up to
    PFB_RAGGED_MAX_N (544) share one persistent launch (pfb_slog_pfaffian_ragged:
    a device-side sort, largest first, and an atomic work queue, every matrix
    factored in FP64); larger orders -- the large bin -- go to the blocked
    cluster-panel path, one pfb_slog_pfaffian_ptrs call per (order, dtype) on
    the matrices where they lie, in ``mode`` ("auto": per group, the faster
    update by the tuned table).
    The device arrays of pointers, orders and dtypes, the workspaces and the
    index maps are built here; ``run()`` enqueues everything on the current
    stream and returns (log|Pf|, sign) as float64 tensors in the input order.
    ``run()`` allocates nothing, so it may be captured in a torch.cuda.CUDAGraph.
    """

    RAGGED_MAX_N = 544

    def __init__(self, mats, layout: int = _lib.ROW_MAJOR, mode: str = "auto"):
        if not mats:
            raise ValueError("empty batch")
        dev = mats[0].device
        for M in mats:
            if M.ndim != 2 or M.shape[0] != M.shape[1]:
                raise ValueError("every matrix must be square")
            if M.dtype not in (torch.float32, torch.float64):
                raise TypeError("ragged batches take float32 or float64 matrices")
            if not M.is_cuda or M.device != dev:
                raise ValueError("all matrices must be CUDA tensors on one device")
        self.mats = [M.contiguous() for M in mats]
        self.count = len(self.mats)
        self.layout = layout
        self.mode = mode
        orders = [M.shape[0] for M in self.mats]
        self.max_n = max(orders)
        small = [i for i, m in enumerate(orders) if m <= self.RAGGED_MAX_N]
        odd_large = [i for i, m in enumerate(orders) if m > self.RAGGED_MAX_N and m & 1]
        groups = {}
        for i, m in enumerate(orders):
            if m > self.RAGGED_MAX_N and not m & 1:
                groups.setdefault((m, self.mats[i].dtype), []).append(i)
        L = _lib.lib()
        self.log = torch.empty(self.count, dtype=torch.float64, device=dev)
        self.sign = torch.empty(self.count, dtype=torch.float64, device=dev)
        # odd orders above the ragged bin: Pf = 0, set once here, never rewritten
        if odd_large:
            oi = torch.tensor(odd_large, dtype=torch.int64, device=dev)
            self.log.index_fill_(0, oi, -float("inf"))
            self.sign.index_fill_(0, oi, 0.0)
        self._direct = len(small) == self.count
        self._small = None
        if small:
            sm_mats = [self.mats[i] for i in small]
            ns = max(orders[i] for i in small)
            self._small_n = ns
            self._ptrs = torch.tensor([M.data_ptr() for M in sm_mats], dtype=torch.int64, device=dev)
            self._ns = torch.tensor([M.shape[0] for M in sm_mats], dtype=torch.int32, device=dev)
            self._dts = torch.tensor([_DT[M.dtype] for M in sm_mats], dtype=torch.int32, device=dev)
            wsb = int(L.pfb_slog_ragged_workspace_bytes(len(sm_mats), ns))
            self._ws_small = torch.empty(wsb, dtype=torch.uint8, device=dev)
            if self._direct:
                self._log_s, self._sign_s = self.log, self.sign
            else:
                self._log_s = torch.empty(len(small), dtype=torch.float64, device=dev)
                self._sign_s = torch.empty(len(small), dtype=torch.float64, device=dev)
                self._idx_s = torch.tensor(small, dtype=torch.int64, device=dev)
            self._small = len(small)
        # the large bin: one pointer-array call per (order, dtype); the calls run
        # one after another on the stream, so they share one workspace
        self._groups = []
        wmax = 0
        for (m, dt), idx in sorted(groups.items(), key=lambda kv: -kv[0][0]):
            ptrs = torch.tensor([self.mats[i].data_ptr() for i in idx], dtype=torch.int64, device=dev)
            lg = torch.empty(len(idx), dtype=torch.float64, device=dev)
            sg = torch.empty(len(idx), dtype=dt, device=dev)
            # float32 signs are widened through a preallocated buffer
            sgd = sg if dt == torch.float64 else torch.empty(len(idx), dtype=torch.float64, device=dev)
            it = torch.tensor(idx, dtype=torch.int64, device=dev)
            gm = resolve_mode(mode, dt, m, len(idx))
            wsb = int(L.pfb_slog_workspace_bytes(_DT[dt], len(idx), m, _MODES[gm]))
            if wsb == 0:
                raise ValueError(f"order {m} is beyond the large path")
            wmax = max(wmax, wsb)
            self._groups.append((m, dt, gm, ptrs, lg, sg, sgd, it, wsb))
        self._ws_large = torch.empty(max(wmax, 1), dtype=torch.uint8, device=dev) if self._groups else None

    @property
    def launches(self) -> int:
        """Kernel launches of one run() (the ragged pair, each large call's
        sequence, and the scatters)."""
        L = _lib.lib()
        k = 2 if self._small else 0
        if self._small and not self._direct:
            k += 2
        for (m, dt, gm, ptrs, lg, sg, sgd, it, wsb) in self._groups:
            nb = int(L.pfb_slog_panel_width(_DT[dt], m))
            npan = (m - 1 + nb - 1) // nb
            per = 2 + npan + (npan - 1) * (2 if gm == "split" else 1)
            k += per * int(L.pfb_slog_stream_ranges(_DT[dt], ptrs.numel(), m, _MODES[gm]))
            k += 2 + (0 if sgd is sg else 1)
        return k

    def run(self):
        L = _lib.lib()
        stream = _stream(self.log)
        if self._small:
            st = L.pfb_slog_pfaffian_ragged(
                self._ptrs.data_ptr(), self._ns.data_ptr(), self._dts.data_ptr(), self._small, self._small_n,
                self.layout, self._log_s.data_ptr(), self._sign_s.data_ptr(), self._ws_small.data_ptr(),
                self._ws_small.numel(), stream)
            _lib.check(st, "pfb_slog_pfaffian_ragged")
            if not self._direct:
                self.log.index_copy_(0, self._idx_s, self._log_s)
                self.sign.index_copy_(0, self._idx_s, self._sign_s)
        for (m, dt, gm, ptrs, lg, sg, sgd, it, wsb) in self._groups:
            st = L.pfb_slog_pfaffian_ptrs(_DT[dt], ptrs.data_ptr(), ptrs.numel(), m, self.layout,
                                          _MODES[gm], lg.data_ptr(), sg.data_ptr(),
                                          self._ws_large.data_ptr(), wsb, stream)
            _lib.check(st, "pfb_slog_pfaffian_ptrs")
            if sgd is not sg:
                sgd.copy_(sg)
            self.log.index_copy_(0, it, lg)
            self.sign.index_copy_(0, it, sgd)
        return self.log, self.sign


def slog_pfaffian_ragged(mats, layout: int = _lib.ROW_MAJOR, mode: str = "auto"):
    """(log|Pf|, sign) for a list of matrices of different orders: orders up to
    544 in one launch, larger ones through the blocked path (RaggedPlan)."""
    plan = RaggedPlan(mats, layout, mode)
    la, sg = plan.run()
    return la.clone(), sg.clone()


# ------------------------------------------------------------- autograd glue
#
# The reference differentiates with forward-mode rules (jax.custom_jvp,
# pfcuda/cuda_api.py:78-107):
#     d log Pf = (1/2) tr(A^-1 dA),   d Pf = Pf * (1/2) tr(A^-1 dA),
# each evaluated with a general inverse (jnp.linalg.inv).  Here both modes run
# through the engine's adjoint kernel, which forms G = (1/2) A^-T from the
# blocked factors (pfcuda_b200.grad); tr(A^-1 dA)/2 is then sum_ij G_ij dA_ij.
# For complex A, log|Pf| = Re(log Pf) and the phase s = Pf/|Pf| = exp(i Im
# log Pf), so d log|Pf| = Re(t) and d s = s * i Im(t) with t = sum G * dA (the
# reference returns a zero sign tangent, which is exact only for real input).
# torch's backward convention for complex tensors is the conjugate Wirtinger
# derivative: a real cotangent g of log|Pf| gives g * conj(G), and a cotangent
# h of the phase adds i Im(h conj(s)) * conj(G).


class _Adjoint(torch.autograd.Function):
    """ct * (1/2) A^-T through the engine's adjoint kernel, as an operation that
    torch's transforms (torch.func.jvp / vjp / grad) can call: they hand its
    forward plain tensors, whose data pointers the C ABI needs.  Its own
    derivatives (second derivatives of log Pf) are not provided."""

    @staticmethod
    def forward(A, ct, mode):
        from .grad import slog_pfaffian_grad
        return slog_pfaffian_grad(A, ct=ct, mode=mode)

    @staticmethod
    def setup_context(ctx, inputs, output):
        pass

    @staticmethod
    def backward(ctx, g):
        raise NotImplementedError("second derivatives of slog_pfaffian / pfaffian are not provided")

    @staticmethod
    def jvp(ctx, dA, dct, dmode):
        raise NotImplementedError("second derivatives of slog_pfaffian / pfaffian are not provided")


def _half_inv_t(A, mode="fp64", ct=None):
    return _Adjoint.apply(A, ct, mode)


def _contract(G, dA):
    """sum_ij G_ij dA_ij per matrix (no conjugation): (1/2) tr(A^-1 dA)."""
    return (G * dA.to(G.dtype)).sum(dim=(-2, -1))


class _PfaffianFn(torch.autograd.Function):
    @staticmethod
    def forward(A):
        return pfaffian_raw(A)

    @staticmethod
    def setup_context(ctx, inputs, output):
        (A,) = inputs
        ctx.save_for_backward(A, output)
        ctx.save_for_forward(A, output)

    @staticmethod
    def backward(ctx, g):
        # dPf/dA = Pf * (1/2) A^-T (pfcuda/cuda_api.py:78-90); torch wants the
        # conjugate for complex A.
        A, pf = ctx.saved_tensors
        G = _half_inv_t(A)
        if A.is_complex():
            G = G.conj()
            pf = pf.conj()
        return (g * pf)[..., None, None] * G

    @staticmethod
    def jvp(ctx, dA):
        # d Pf = Pf * (1/2) tr(A^-1 dA)  (pfcuda/cuda_api.py:78-90)
        A, pf = ctx.saved_tensors
        return pf * _contract(_half_inv_t(A), dA).to(pf.dtype)


class _SlogFn(torch.autograd.Function):
    @staticmethod
    def forward(A, mode):
        return slog_pfaffian_raw(A, mode)

    @staticmethod
    def setup_context(ctx, inputs, output):
        A, mode = inputs
        la, sg = output
        ctx.mode = mode
        ctx.save_for_backward(A, sg)
        ctx.save_for_forward(A, sg)
        if not A.is_complex():
            ctx.mark_non_differentiable(sg)   # +-1: piecewise constant

    @staticmethod
    def backward(ctx, g_log, g_sign):
        # d log|Pf| / dA = (1/2) A^-T  (pfcuda/cuda_api.py:92-107); for real A
        # the engine applies the cotangent in its last kernel.
        A, sg = ctx.saved_tensors
        if not A.is_complex():
            return _half_inv_t(A, ctx.mode, ct=g_log), None
        c = torch.zeros(A.shape[:-2], dtype=A.dtype, device=A.device)
        if g_log is not None:
            c = c + g_log.to(A.dtype)
        if g_sign is not None:
            c = c + 1j * (g_sign * sg.conj()).imag.to(A.dtype)
        return c[..., None, None] * _half_inv_t(A, ctx.mode).conj(), None

    @staticmethod
    def jvp(ctx, dA, _dmode):
        # d log|Pf| = Re (1/2) tr(A^-1 dA)  (pfcuda/cuda_api.py:92-107); the
        # phase of complex A turns by i Im of the same trace.
        A, sg = ctx.saved_tensors
        t = _contract(_half_inv_t(A, ctx.mode), dA)
        if A.is_complex():
            return t.real.to(torch.float64), sg * (1j * t.imag).to(sg.dtype)
        return t.to(torch.float64), None   # the sign of real A is piecewise constant
