"""pfcuda_b200 -- a B200-native Pfaffian engine.

Drop-in for the hot path of PfCUDA (pfcuda/__init__.py:1): ``pfaffian`` for
2n <= 32 and ``slog_pfaffian`` for any even 2n, on float32 / float64 /
complex64 / complex128, computed by hand-written sm_100a kernels behind the C ABI
of include/pfb200.h (libpfb200.so, built in-tree).
"""
from .api import (pfaffian, slog_pfaffian, pfaffian_raw, slog_pfaffian_raw,
                  slog_workspace_bytes, slog_pfaffian_ragged, RaggedPlan, upload_upper,
                  upload_upper_bytes, resolve_mode, slog_config)
from .grad import slog_pfaffian_grad, grad_workspace_bytes

__all__ = ["pfaffian", "slog_pfaffian", "pfaffian_raw", "slog_pfaffian_raw",
           "slog_workspace_bytes", "slog_pfaffian_ragged", "RaggedPlan",
           "slog_pfaffian_grad", "grad_workspace_bytes", "upload_upper", "upload_upper_bytes", "resolve_mode",
           "slog_config"]
