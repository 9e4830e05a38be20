"""pfb_slog_pfaffian_noalloc: the large path for callers that cannot allocate.

Callers such as a plugin handed raw device pointers by a framework that owns
every allocation, or a binding with no CUDA allocator, cannot provide the
workspace pfb_slog_pfaffian asks for.  This entry point uses a fixed scratch
array inside the library instead.  Its results must match the allocating entry
point's (same kernels, same inputs) on consecutive calls, which also checks that
nothing left in the shared scratch by one call leaks into the next.  The file
name makes pytest collect it last.
"""
import ctypes

import numpy as np
import pytest
import torch

import pfcuda_b200 as pf
from pfcuda_b200 import _lib

pytestmark = pytest.mark.gpu

DT = {torch.float64: _lib.F64, torch.complex128: _lib.C128, torch.float32: _lib.F32}


def skew(seed, B, n, dtype):
    g = torch.Generator().manual_seed(seed)
    G = torch.randn(B, n, n, generator=g, dtype=torch.float64) / n ** 0.5
    if dtype.is_complex:
        G = torch.complex(G, torch.randn(B, n, n, generator=g, dtype=torch.float64) / n ** 0.5)
    return ((G - G.transpose(-1, -2)) / 2).to(dtype).cuda()


def noalloc(A, mode):
    n = A.shape[-1]
    B = A.shape[0]
    la = torch.full((B,), 7.0, dtype=torch.float64, device=A.device)
    sg = torch.full((B,), 7.0, dtype=A.dtype, device=A.device)
    st = _lib.lib().pfb_slog_pfaffian_noalloc(DT[A.dtype], A.data_ptr(), B, n, _lib.ROW_MAJOR, mode,
                                              la.data_ptr(), sg.data_ptr(),
                                              torch.cuda.current_stream().cuda_stream)
    return st, la, sg


def close(got, want):
    la, sg = got
    wl, ws = want
    la, wl = la.cpu().numpy(), wl.cpu().numpy()
    assert np.all(np.abs(la - wl) <= 1e-10 * np.abs(wl) + 1e-12)
    assert np.all(np.abs(sg.cpu().numpy() - ws.cpu().numpy()) <= 1e-10)


@pytest.mark.parametrize("dtype,n,B,mode", [
    (torch.float64, 256, 3, _lib.MODE_FP64),
    (torch.float64, 200, 2, _lib.MODE_SPLIT),
    (torch.complex128, 130, 2, _lib.MODE_FP64),
    (torch.float32, 96, 4, _lib.MODE_FP64),
    (torch.float64, 20, 5, _lib.MODE_FP64),
])
def test_matches_allocating_entry_point_on_consecutive_calls(dtype, n, B, mode):
    mname = "split" if mode == _lib.MODE_SPLIT else "fp64"
    for call, seed in enumerate((11, 12)):          # two calls in a row, different inputs
        A = skew(seed + n, B, n, dtype)
        st, la, sg = noalloc(A, mode)
        assert st == 0, _lib.lib().pfb_status_string(st)
        torch.cuda.synchronize()
        close((la, sg), pf.slog_pfaffian_raw(A, mode=mname))


def test_rejects_sizes_beyond_the_scratch():
    A = torch.zeros(1, 2048, 2048, dtype=torch.float64, device="cuda")
    st, la, sg = noalloc(A, _lib.MODE_FP64)
    assert st == 2                                    # PFB_ERR_SIZE, nothing launched
    torch.cuda.synchronize()
    assert torch.all(la == 7.0)
