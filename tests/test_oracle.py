"""The oracle against the reference's own outputs (CPU only).

The oracle (oracle/pf_oracle.c) restates src/pfaffian_cpu.cpp and
pfcuda/pfaffian_py.py.  Before it is trusted as the checker of the CUDA engine
it is pinned here: its as-shipped mode must reproduce the reference's CPU values
bit for bit, and its log-space mode must agree with them and with the
reference's NumPy path and known-answer construction.
"""
import numpy as np
import pytest

from oracle import oracle as O
from golden_io import load, split


def test_as_shipped_bit_exact_vs_golden():
    g = load("cpu_f64.npz")
    mats = split(g["sizes_A"], g["sizes_n"])
    got = np.array([O.pf_product(a, as_shipped=True) for a in mats])
    assert np.array_equal(got, g["sizes_pf"])
    assert np.array_equal(O.pf_product(g["bench_A"], as_shipped=True), g["bench_pf"])
    assert np.array_equal(O.pf_product(g["mid64_A"], as_shipped=True), g["mid64_pf"])
    assert np.array_equal(O.pf_product(g["mid128_A"], as_shipped=True), g["mid128_pf"])


def test_slog_matches_reference_cpu_values():
    g = load("cpu_f64.npz")
    for A, pf in ((g["bench_A"], g["bench_pf"]), (g["mid64_A"], g["mid64_pf"]),
                  (g["mid128_A"], g["mid128_pf"])):
        la, sg = O.slog_pf(A)
        np.testing.assert_allclose(la, np.log(np.abs(pf)), rtol=1e-12, atol=1e-11)
        assert np.array_equal(sg, np.sign(pf))


def test_slog_matches_reference_cpu_large():
    g = load("cpu_large.npz")
    for seed, n, pf in zip(g["seeds"], g["n"], g["pf"]):
        A = O.config_large(int(n), seed=int(seed))[0]
        la, sg = O.slog_pf(A)
        assert abs(la - np.log(abs(pf))) <= 1e-11 * abs(la)
        assert sg == np.sign(pf)


def test_complex_matches_reference_numpy_path():
    g = load("py_c128.npz")
    for A, pf in zip(split(g["A"], g["n"]), g["pf"]):
        la, ph = O.slog_pf(A)
        got = ph * np.exp(la)
        assert abs(got - pf) <= 1e-12 * abs(pf)
        assert abs(O.pf_product(A) - pf) <= 1e-12 * abs(pf)


def test_known_answer_construction():
    g = load("known.npz")
    for A, pf in zip(split(g["A"], g["n"]), g["pf"]):
        la, sg = O.slog_pf(A)
        np.testing.assert_allclose(sg * np.exp(la), pf, rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("n", [34, 64, 100, 256])
def test_pf_squared_is_det(n):
    rng = np.random.default_rng(n)
    A = O.skew_normal(rng, 2, n, scale=1 / np.sqrt(n))
    la, sg = O.slog_pf(A)
    s, ld = np.linalg.slogdet(A)
    np.testing.assert_allclose(2 * la, ld, rtol=1e-12)
    assert np.all(s > 0)


def test_live_reference_cpu_bit_exact():
    if O.ref_cpu() is None:
        pytest.skip("oracle/_ref/libref_cpu.so not built")
    rng = np.random.default_rng(99)
    for n in (6, 10, 32, 50, 96):
        A = O.skew_normal(rng, 8, n)
        assert np.array_equal(O.ref_cpu_pfaffian(A), O.pf_product(A, as_shipped=True))


def test_numpy_restatement_agrees():
    rng = np.random.default_rng(3)
    for cplx in (False, True):
        A = O.skew_normal(rng, 3, 24, complex_=cplx)
        la, sg = O.slog_pf(A)
        for b in range(3):
            l2, s2 = O.slog_pf_numpy(A[b])
            assert abs(la[b] - l2) < 1e-12
            assert abs(sg[b] - s2) < 1e-12


def test_edge_cases():
    for n in (0, 1, 3, 35):
        la, sg = O.slog_pf(np.ones((1, n, n)))
        assert np.isneginf(la[0]) and sg[0] == 0
    la, sg = O.slog_pf(np.zeros((2, 40, 40)))
    assert np.all(np.isneginf(la)) and np.all(sg == 0)
    la, sg, piv = O.slog_pf(O.skew_normal(np.random.default_rng(1), 1, 10), with_pivots=True)
    assert piv.shape == (1, 5) and np.all(piv[0] >= np.arange(1, 10, 2))


@pytest.mark.parametrize("cplx", [False, True])
def test_jvp_rule_matches_central_difference(cplx):
    """The restated rule of pfcuda/cuda_api.py:92-107 against central differences
    (h = 1e-6) of the C restatement of log|Pf|, and its adjoint against the rule."""
    rng = np.random.default_rng(20 + cplx)
    A = O.skew_normal(rng, 3, 48, scale=1 / np.sqrt(48), complex_=cplx)
    E = O.skew_normal(rng, 3, 48, complex_=cplx)
    fd = O.fd_slog(A, E)
    jvp = O.slog_pf_jvp(A, E)
    assert np.all(np.abs(jvp.real - fd) <= 1e-6 * np.abs(fd) + 1e-7)
    G = O.slog_pf_vjp(A, ct=[1.0, 2.0, -1.0])
    assert np.allclose(np.sum(G * E, axis=(-1, -2)), jvp * np.array([1.0, 2.0, -1.0]), rtol=1e-12)
