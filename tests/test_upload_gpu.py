"""The large path reads only the upper triangle (diagonal included) of each
matrix's row-major view, and pfb_upload_upper moves only that part.

Bars: results with garbage below the diagonal are bit-identical to those of
the clean skew matrix (log, sign and pivot sequence); pfb_upload_upper leaves
every entry on and above the diagonal equal to the host's and moves the bytes
pfb_upload_upper_bytes reports.
"""
import numpy as np
import pytest
import torch

import pfcuda_b200 as pf
from pfcuda_b200 import _lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def run(A, mode, layout=_lib.ROW_MAJOR):
    la, sg = pf.slog_pfaffian_raw(A, mode=mode, layout=layout)
    return la.cpu().numpy(), sg.cpu().numpy()


def spoil_lower(M, rng, value=None):
    """M with every entry strictly below the diagonal of its row-major view
    replaced (random values, or `value`)."""
    M = M.copy()
    n = M.shape[-1]
    il = np.tril_indices(n, -1)
    junk = rng.normal(size=(M.shape[0], len(il[0])))
    if np.iscomplexobj(M):
        junk = junk + 1j * rng.normal(size=junk.shape)
    if value is not None:
        junk[:] = value
    M[:, il[0], il[1]] = junk
    return M


@pytest.mark.parametrize("mode", ["fp64", "split"])
@pytest.mark.parametrize("n,cplx", [(34, False), (100, False), (258, False), (1030, False), (66, True), (300, True)])
def test_lower_triangle_is_never_read(mode, n, cplx):
    rng = np.random.default_rng(40 + n)
    A = O.skew_normal(rng, 3, n, scale=1 / np.sqrt(n), complex_=cplx)
    clean = run(torch.from_numpy(A).cuda(), mode)
    for value in (None, np.nan):
        dirty = run(torch.from_numpy(spoil_lower(A, rng, value)).cuda(), mode)
        assert np.array_equal(clean[0], dirty[0]) and np.array_equal(clean[1], dirty[1])


def test_lower_triangle_column_major():
    rng = np.random.default_rng(47)
    M = O.skew_normal(rng, 2, 130, scale=1 / np.sqrt(130))   # memory of column-major matrices
    clean = run(torch.from_numpy(M).cuda(), "split", _lib.COL_MAJOR)
    dirty = run(torch.from_numpy(spoil_lower(M, rng, np.nan)).cuda(), "split", _lib.COL_MAJOR)
    assert np.array_equal(clean[0], dirty[0]) and np.array_equal(clean[1], dirty[1])


@pytest.mark.parametrize("n,dt", [(16, torch.float64), (40, torch.float64), (300, torch.float32),
                                  (600, torch.complex128), (1030, torch.float64)])
def test_upload_upper(n, dt):
    rng = np.random.default_rng(60 + n)
    A = O.skew_normal(rng, 3, n, scale=1 / np.sqrt(n), complex_=dt.is_complex)
    host = torch.from_numpy(A).to(dt).pin_memory()
    dev = torch.full(host.shape, float("nan"), dtype=dt, device="cuda")
    got = pf.upload_upper(host, out=dev)
    torch.cuda.synchronize()
    assert got.data_ptr() == dev.data_ptr()
    back = dev.cpu()
    iu = np.triu_indices(n)
    if n <= 32:
        assert torch.equal(back, host)
    else:
        assert torch.equal(back[:, iu[0], iu[1]], host[:, iu[0], iu[1]])
    # and the factorisation of the uploaded batch equals that of the full copy
    if n > 32:
        full = host.cuda()
        a = pf.slog_pfaffian_raw(dev)
        b = pf.slog_pfaffian_raw(full)
        assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])
    es = host.element_size()
    want = 3 * n * n * es if n <= 32 else 3 * sum(min(256, n - r0) * (n - r0) for r0 in range(0, n, 256)) * es
    assert _lib.lib().pfb_upload_upper_bytes(_lib.F64 if dt == torch.float64 else
                                             {torch.float32: _lib.F32, torch.complex128: _lib.C128}[dt],
                                             3, n) == want
