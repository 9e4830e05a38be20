"""The C-ABI library: symbols, status strings and argument checks (no GPU needed).

Every call here returns before any CUDA work is enqueued.
"""
import ctypes
import os
import re

import pytest

from pfcuda_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "pfb200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(pfb_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_functions()
    assert len(names) >= 6
    for name in names:
        assert hasattr(L, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


def test_status_strings():
    L = _lib.lib()
    for st in range(0, 8):
        assert isinstance(L.pfb_status_string(st), bytes)
    assert L.pfb_status_string(0) == b"ok"


def test_argument_checks_without_gpu():
    L = _lib.lib()
    out = ctypes.c_double()
    p = ctypes.addressof(out)
    assert L.pfb_pfaffian(9, p, 1, 8, 0, p, None) == 1          # bad dtype
    assert L.pfb_pfaffian(1, p, 1, 8, 7, p, None) == 1          # bad layout
    assert L.pfb_pfaffian(1, p, -1, 8, 0, p, None) == 1         # negative batch
    assert L.pfb_pfaffian(1, p, 1, 34, 0, p, None) == 2         # order above 32
    assert L.pfb_pfaffian(1, p, 0, 8, 0, p, None) == 0          # empty batch
    assert L.pfb_pfaffian(1, p, 1, 8, 0, None, None) == 1       # no output
    assert L.pfb_slog_pfaffian(1, p, 1, 64, 0, 5, p, p, None, 0, None) == 1   # bad mode
    assert L.pfb_slog_pfaffian(1, p, 1, 64, 0, 0, p, p, None, 0, None) == 3   # no workspace
    assert L.pfb_slog_pfaffian(1, p, 0, 64, 0, 0, p, p, None, 0, None) == 0


@pytest.mark.parametrize("dtype", [0, 1, 2, 3])
def test_workspace_sizes(dtype):
    L = _lib.lib()
    prev = 0
    for n in (34, 64, 128, 1024, 4096):
        for mode in (0, 1):
            w = L.pfb_slog_workspace_bytes(dtype, 1, n, mode)
            assert w > 0 and w % 256 == 0
        w = L.pfb_slog_workspace_bytes(dtype, 1, n, 0)
        assert w >= prev
        prev = w
    assert L.pfb_slog_workspace_bytes(dtype, 2, 1024, 0) > L.pfb_slog_workspace_bytes(dtype, 1, 1024, 0)
    assert L.pfb_slog_workspace_bytes(dtype, 1, 1 << 20, 0) == 0   # beyond the supported order


def test_grad_argument_checks_without_gpu():
    L = _lib.lib()
    out = ctypes.c_double()
    p = ctypes.addressof(out)
    f = L.pfb_slog_pfaffian_grad
    assert f(9, p, 1, 64, 0, 0, None, p, p, p, None, 0, None) == 1      # bad dtype
    assert f(1, p, 1, 64, 3, 0, None, p, p, p, None, 0, None) == 1      # bad layout
    assert f(1, p, 1, 64, 0, 9, None, p, p, p, None, 0, None) == 1      # bad mode
    assert f(1, p, 1, 35, 0, 0, None, p, p, p, None, 0, None) == 2      # odd order
    assert f(1, p, 1, 64, 0, 0, None, p, p, p, None, 0, None) == 3      # no workspace
    assert f(1, p, 1, 64, 0, 0, None, None, p, p, None, 0, None) == 1   # no output
    assert f(1, p, 0, 64, 0, 0, None, p, p, p, None, 0, None) == 0      # empty batch
    for dtype in range(4):
        w1 = L.pfb_slog_grad_workspace_bytes(dtype, 1, 512, 0)
        assert w1 > L.pfb_slog_workspace_bytes(dtype, 1, 512, 0) and w1 % 256 == 0
        assert L.pfb_slog_grad_workspace_bytes(dtype, 1, 35, 0) == 0
        assert L.pfb_slog_grad_workspace_bytes(dtype, 1, 1 << 20, 0) == 0


def test_upload_upper_sizes_and_argument_checks_without_gpu():
    L = _lib.lib()
    # orders <= 32 go whole; above, one rectangle per 256 rows from the diagonal on
    assert L.pfb_upload_upper_bytes(_lib.F64, 3, 32) == 3 * 32 * 32 * 8
    assert L.pfb_upload_upper_bytes(_lib.F32, 2, 300) == 2 * (256 * 300 + 44 * 44) * 4
    n = 4096
    want = sum(256 * (n - r0) for r0 in range(0, n, 256)) * 16
    assert L.pfb_upload_upper_bytes(_lib.C128, 1, n) == want
    assert want < 0.54 * n * n * 16
    assert L.pfb_upload_upper_bytes(99, 1, 64) == 0
    assert L.pfb_upload_upper_bytes(_lib.F64, -1, 64) == 0
    buf = ctypes.create_string_buffer(64)
    assert L.pfb_upload_upper(99, buf, buf, 1, 4, None) == 1           # bad dtype
    assert L.pfb_upload_upper(_lib.F64, None, buf, 1, 4, None) == 1    # no source
    assert L.pfb_upload_upper(_lib.F64, buf, None, 1, 4, None) == 1    # no destination
    assert L.pfb_upload_upper(_lib.F64, None, None, 0, 4, None) == 0   # empty batch
