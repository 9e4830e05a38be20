"""Reverse-mode derivative of log|Pf| through the engine's own factors.

The reference differentiates with jax.custom_jvp rules that call
jnp.linalg.inv (pfcuda/cuda_api.py:78-107):

    d log Pf = (1/2) tr(A^-1 dA),   so   d log Pf / dA = (1/2) A^-T.

``slog_pfaffian_grad`` returns ct * (1/2) A^-T for a batch in one C-ABI call
(pfb_slog_pfaffian_grad): the blocked skew-LTL^T factorisation of the forward
pass, then the inverse assembled from its factors on the device
(P A P^T = U^T D U  =>  A^-1 = P^T U^-1 D^-1 U^-T P), so the forward values come
out of the same call.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .api import _DT, _MODES, _stream


def grad_workspace_bytes(dtype: torch.dtype, batch: int, n: int, mode: str = "fp64") -> int:
    return int(_lib.lib().pfb_slog_grad_workspace_bytes(_DT[dtype], batch, n, _MODES[mode]))


def grad_min_workspace_bytes(dtype: torch.dtype, n: int, mode: str = "fp64") -> int:
    """The smallest workspace the adjoint accepts: one matrix at a time."""
    return grad_workspace_bytes(dtype, 1, n, mode)


def slog_pfaffian_grad(A: torch.Tensor, ct: torch.Tensor | None = None, mode: str = "fp64",
                       layout: int = _lib.ROW_MAJOR, workspace: torch.Tensor | None = None,
                       return_forward: bool = False, budget_bytes: int | None = None):
    """ct * d log Pf(A) / dA = ct * (1/2) A^-T for a contiguous (..., n, n) CUDA tensor.

    ``ct`` holds one real cotangent per matrix (None: all ones).  The result has
    A's dtype and layout and is holomorphic (not conjugated).  A matrix with
    Pf = 0 gets an all-NaN gradient; odd orders (Pf = 0 identically) give NaN
    without a launch.  With ``return_forward`` the call also returns
    (log|Pf|, sign) of the same factorisation.

    ``budget_bytes`` caps the workspace (about 2 n^2 working elements per
    matrix): the batch then runs in chunks of as many matrices as fit, with
    results identical to an unbounded call.  It cannot go below one matrix's
    need (grad_min_workspace_bytes).  A ``workspace`` tensor given by the caller
    is used as it is, its size being the budget.
    """
    if not isinstance(A, torch.Tensor) or not A.is_cuda:
        raise ValueError("the engine runs on CUDA tensors only (no CPU fallback)")
    if A.dtype not in _DT:
        raise TypeError(f"unsupported dtype {A.dtype}")
    if A.ndim < 2 or A.shape[-1] != A.shape[-2]:
        raise ValueError(f"expected (..., n, n) matrices, got shape {tuple(A.shape)}")
    A = A.contiguous()
    n = A.shape[-1]
    lead = A.shape[:-2]
    B = int(np.prod(lead)) if len(lead) else 1
    G = torch.empty_like(A)
    la = torch.empty(lead, dtype=torch.float64, device=A.device)
    sg = torch.empty(lead, dtype=A.dtype, device=A.device)
    if n == 0 or n & 1:
        G.fill_(float("nan"))
        la.fill_(-float("inf") if n else 0.0)
        sg.fill_(0 if n else 1)
        return (G, la, sg) if return_forward else G
    if ct is not None:
        ct = ct.to(device=A.device, dtype=torch.float64).reshape(-1).contiguous()
        if ct.numel() != B:
            raise ValueError(f"ct must hold one cotangent per matrix ({B}), got {ct.numel()}")
    wsb = grad_workspace_bytes(A.dtype, B, n, mode)
    if wsb == 0:
        raise ValueError(f"order {n} is outside the supported range")
    w1 = grad_min_workspace_bytes(A.dtype, n, mode)
    if budget_bytes is not None:
        if budget_bytes < w1:
            raise ValueError(f"budget_bytes {budget_bytes} is below one matrix's need ({w1} bytes)")
        wsb = min(wsb, int(budget_bytes))
    if workspace is None:
        workspace = torch.empty(wsb, dtype=torch.uint8, device=A.device)
    elif workspace.numel() < w1:
        raise ValueError(f"workspace of {workspace.numel()} bytes is below one matrix's need ({w1} bytes)")
    else:
        wsb = min(wsb, workspace.numel())
    st = _lib.lib().pfb_slog_pfaffian_grad(
        _DT[A.dtype], A.data_ptr(), B, n, layout, _MODES[mode],
        ct.data_ptr() if ct is not None else None, G.data_ptr(), la.data_ptr(), sg.data_ptr(),
        workspace.data_ptr(), wsb, _stream(A))
    _lib.check(st, "pfb_slog_pfaffian_grad")
    return (G, la, sg) if return_forward else G
