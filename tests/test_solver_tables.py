"""The library's line-solver tables, checked on the CPU by emulating the warp algorithm."""
import numpy as np
import pytest

from compact_schemes_b200.numerics import line_tables
from solver_emulation import emulate

SIZES = [5, 7, 8, 9, 16, 17, 32, 33, 48, 64, 65, 96, 100, 128, 129, 256, 257, 512, 513, 1000, 1024]


def deriv_matrix(n, ns, ne):
    A = np.eye(n) + np.diag(np.full(n - 1, 1 / 3), 1) + np.diag(np.full(n - 1, 1 / 3), -1)
    if ns == 0:
        A[0, 1] = 2.0
        A[1, 0] = A[1, 2] = 0.25
    if ne == 0:
        A[n - 1, n - 2] = 2.0
        A[n - 2, n - 1] = A[n - 2, n - 3] = 0.25
    return A


def filter_matrix(n, cyclic, af):
    A = np.eye(n)
    for i in range(n):
        if cyclic or 0 < i < n - 1:
            A[i, (i - 1) % n] = af
            A[i, (i + 1) % n] = af
    return A


@pytest.mark.parametrize("n", SIZES)
def test_deriv_tables(n):
    rng = np.random.default_rng(n)
    for ns in (0, 1):
        for ne in (0, 1):
            if (ns or ne) and n < 8:
                continue
            tab = line_tables(n, 0, ns, ne)
            r = rng.normal(size=n)
            x = emulate(tab, r)
            ref = np.linalg.solve(deriv_matrix(n, ns, ne), r)
            assert np.abs(x - ref).max() / np.abs(ref).max() < 1e-13


@pytest.mark.parametrize("n", [s for s in SIZES if s >= 7])
def test_filter_tables(n):
    rng = np.random.default_rng(n + 7)
    for cyc in (0, 1):
        for af in (0.3, 0.45, 0.49):
            tab = line_tables(n, 1, cyc, cyc, af)
            r = rng.normal(size=n)
            x = emulate(tab, r)
            ref = np.linalg.solve(filter_matrix(n, cyc, af), r)
            assert np.abs(x - ref).max() / np.abs(ref).max() < 1e-13


def test_chunking_limits():
    assert line_tables(1024)["lt"] == 32
    assert line_tables(256)["lt"] == 8 and line_tables(256)["p"] == 32
    with pytest.raises(Exception):
        line_tables(1025)
    with pytest.raises(Exception):
        line_tables(4)
