"""ctypes binding of libpfb200.so (the C ABI declared in include/pfb200.h).

The library is built in-tree by ``python -m pfcuda_b200.build``.  There is no
fallback: if the library is missing, loading raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpfb200.so")

# enums of include/pfb200.h
F32, F64, C64, C128 = 0, 1, 2, 3
ROW_MAJOR, COL_MAJOR = 0, 1
MODE_FP64, MODE_SPLIT = 0, 1
OK = 0

# every function include/pfb200.h declares: name -> (restype, argtypes)
_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_int = ctypes.c_int
_sz = ctypes.c_size_t
SIGNATURES = {
    "pfb_status_string": (ctypes.c_char_p, [_int]),
    "pfb_last_cuda_error": (_int, []),
    "pfb_pfaffian": (_int, [_int, _vp, _i64, _int, _int, _vp, _vp]),
    "pfb_slog_pfaffian": (_int, [_int, _vp, _i64, _int, _int, _int, _vp, _vp, _vp, _sz, _vp]),
    "pfb_slog_workspace_bytes": (_sz, [_int, _i64, _int, _int]),
    "pfb_slog_pivots": (_int, [_i64, _int, _vp, _sz, _vp, _vp]),
    "pfb_slog_pfaffian_timed": (_int, [_int, _vp, _i64, _int, _int, _int, _vp, _vp, _vp, _sz, _vp, _vp]),
    "pfb_slog_panel_width": (_int, [_int, _int]),
    "pfb_slog_max_concurrent": (_int, [_int, _int]),
    "pfb_slog_stream_ranges": (_int, [_int, _i64, _int, _int]),
    "pfb_slog_max_concurrent_form": (_int, [_int, _int, _int]),
    "pfb_slog_config_for": (_int, [_int, _i64, _int, _int, _vp]),
    "pfb_slog_pfaffian_ex": (_int, [_int, _vp, _i64, _int, _int, _int, _vp, _vp, _vp, _sz, _vp, _vp, _vp]),
    "pfb_slog_pfaffian_ptrs": (_int, [_int, _vp, _i64, _int, _int, _int, _vp, _vp, _vp, _sz, _vp]),
    "pfb_slog_pfaffian_ragged": (_int, [_vp, _vp, _vp, _i64, _int, _int, _vp, _vp, _vp, _sz, _vp]),
    "pfb_slog_ragged_workspace_bytes": (_sz, [_i64, _int]),
    "pfb_slog_pfaffian_noalloc": (_int, [_int, _vp, _i64, _int, _int, _int, _vp, _vp, _vp]),
    "pfb_slog_pfaffian_grad": (_int, [_int, _vp, _i64, _int, _int, _int, _vp, _vp, _vp, _vp, _vp, _sz, _vp]),
    "pfb_slog_grad_workspace_bytes": (_sz, [_int, _i64, _int, _int]),
    "pfb_upload_upper": (_int, [_int, _vp, _vp, _i64, _int, _vp]),
    "pfb_upload_upper_bytes": (_sz, [_int, _i64, _int]),
}

class SlogConfig(ctypes.Structure):
    """pfb_slog_config of include/pfb200.h (0 fields: the tuned table's choice)."""
    _fields_ = [("panel", ctypes.c_int), ("slices", ctypes.c_int), ("ranges", ctypes.c_int),
                ("epilogue", ctypes.c_int)]

    def as_dict(self):
        return {"panel": {1: "registers", 2: "half_shared"}.get(self.panel, self.panel),
                "slices": self.slices, "ranges": self.ranges,
                "epilogue": {1: "roundtrip", 2: "reduce", 3: "direct"}.get(self.epilogue, self.epilogue)}


PANEL_REGISTERS, PANEL_HALF_SHARED = 1, 2
EPILOGUE_ROUNDTRIP, EPILOGUE_REDUCE, EPILOGUE_DIRECT = 1, 2, 3


class SlogTiming(ctypes.Structure):
    """pfb_slog_timing of include/pfb200.h."""
    _fields_ = [("panel_events", ctypes.POINTER(ctypes.c_void_p)),
                ("update_events", ctypes.POINTER(ctypes.c_void_p)),
                ("pairs", ctypes.c_int)]


_lib = None


class PfbError(RuntimeError):
    """A C-ABI call returned a non-zero pfb_status."""

    def __init__(self, status: int, what: str):
        msg = lib().pfb_status_string(status).decode()
        if status == 4:
            msg += f" (cudaError {lib().pfb_last_cuda_error()})"
        super().__init__(f"{what}: {msg} [status {status}]")
        self.status = status


def lib():
    """Load libpfb200.so once (raises OSError if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: build it with `python -m pfcuda_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int, what: str):
    if status != OK:
        raise PfbError(status, what)
