"""Host-side rules of the Python API (pfcuda/cuda_api.py:27-76), on CPU tensors.

These branches never reach a kernel; the kernel branches must refuse CPU tensors
(there is no CPU fallback).
"""
import numpy as np
import pytest
import torch

import pfcuda_b200 as pf


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64, torch.complex64, torch.complex128])
def test_odd_and_empty_give_zero(dtype):
    for n in (0, 1, 3, 5, 11, 15):
        out = pf.pfaffian(torch.ones(2, n, n, dtype=dtype))
        assert out.shape == (2,) and torch.all(out == 0)


def test_closed_forms():
    for a in (0.0, 1.0, -3.5, 1e-12, 1e10):
        A = torch.tensor([[0, a], [-a, 0]], dtype=torch.float64)
        assert pf.pfaffian(A).item() == a
    rng = np.random.default_rng(0)
    G = rng.normal(size=(4, 4))
    A = G - G.T
    want = A[0, 1] * A[2, 3] - A[0, 2] * A[1, 3] + A[0, 3] * A[1, 2]
    assert np.isclose(pf.pfaffian(torch.from_numpy(A)).item(), want)
    assert np.isclose(pf.pfaffian(A), want)          # NumPy in, NumPy out


def test_size_limits():
    with pytest.raises(ValueError, match="32x32"):
        pf.pfaffian(torch.zeros(34, 34, dtype=torch.float64))
    with pytest.raises(ValueError, match="33x33"):
        pf.slog_pfaffian(torch.zeros(32, 32, dtype=torch.float64))


def test_slog_odd():
    la, sg = pf.slog_pfaffian(torch.ones(3, 35, 35, dtype=torch.complex128))
    assert la.dtype == torch.float64 and torch.all(torch.isneginf(la))
    assert sg.dtype == torch.complex128 and torch.all(sg == 0)


def test_no_cpu_fallback():
    with pytest.raises(ValueError, match="CUDA"):
        pf.pfaffian(torch.zeros(8, 8, dtype=torch.float64))
    with pytest.raises(ValueError, match="CUDA"):
        pf.slog_pfaffian(torch.zeros(40, 40, dtype=torch.float64))


def test_bad_inputs():
    with pytest.raises(ValueError):
        pf.pfaffian(torch.zeros(3, 4))
    with pytest.raises(TypeError):
        pf.pfaffian(torch.zeros(8, 8, dtype=torch.int32))


def test_mode_resolution():
    assert pf.resolve_mode("auto", torch.float64) == "split"
    assert pf.resolve_mode("auto", torch.float32) == "split"
    assert pf.resolve_mode("auto", torch.complex128) == "fp64"
    assert pf.resolve_mode("auto", torch.complex64) == "fp64"
    assert pf.resolve_mode("fp64", torch.float64) == "fp64"
    with pytest.raises(ValueError, match="mode"):
        pf.resolve_mode("tf32", torch.float64)
    with pytest.raises(ValueError, match="mode"):
        pf.slog_pfaffian(torch.zeros(40, 40, dtype=torch.float64), mode="tf32")


def test_auto_mode_follows_the_tuned_table(monkeypatch):
    """With measured entries for both modes, "auto" takes the faster one for
    the dtype class, order bin and batch bin; without, the defaults."""
    import pfcuda_b200.api as api
    entries = [
        {"dtype": "complex", "mode": "split", "n_min": 1058, "n_max": 2080, "batch_min": 2, "batch_max": 50, "ms": 30.0},
        {"dtype": "complex", "mode": "fp64", "n_min": 1058, "n_max": 2080, "batch_min": 2, "batch_max": 50, "ms": 40.0},
        {"dtype": "real", "mode": "split", "n_min": 34, "n_max": 544, "batch_min": 1, "batch_max": 1, "ms": 2.0},
        {"dtype": "real", "mode": "fp64", "n_min": 34, "n_max": 544, "batch_min": 1, "batch_max": 1, "ms": 1.5},
    ]
    monkeypatch.setattr(api, "_TUNED", entries)
    assert api.resolve_mode("auto", torch.complex128, 2048, 10) == "split"
    assert api.resolve_mode("auto", torch.complex128, 4096, 10) == "fp64"      # no entry: default
    assert api.resolve_mode("auto", torch.float64, 512, 1) == "fp64"
    assert api.resolve_mode("auto", torch.float64, 512, 7) == "split"          # no entry: default
    assert api.resolve_mode("fp64", torch.float64, 512, 7) == "fp64"
