"""Readers for the fixtures in tests/golden/ (see tests/golden/make_golden.py)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def split(flat, ns):
    """Split a concatenation of flattened n x n matrices back into a list."""
    out, off = [], 0
    for n in ns:
        out.append(flat[off:off + n * n].reshape(n, n))
        off += n * n
    return out
