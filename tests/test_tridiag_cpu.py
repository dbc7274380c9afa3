"""The tridiagonal oracle (oracle/src/tridiag.c) against an independent banded
solver. Tridsolver, which the reference calls, is not vendored, so the oracle
is pinned to the mathematics: scipy's LAPACK banded solve on the same lines."""
import ctypes

import numpy as np
import pytest
from scipy.linalg import solve_banded

from ops_b200 import seeded


def oracle_solve(orc, a, b, c, d, solvedim, u=None, pads=None):
    nd = a.ndim
    dims = (ctypes.c_int * 3)(*list(reversed(a.shape)), *([1] * (3 - nd)))
    pads = dims if pads is None else pads
    f = orc.oracle_trid_batch_d if a.dtype == np.float64 else orc.oracle_trid_batch_s
    f(a.ctypes.data, b.ctypes.data, c.ctypes.data, d.ctypes.data, None if u is None else u.ctypes.data, nd,
      solvedim, dims, pads)


@pytest.mark.parametrize("solvedim", [0, 1, 2])
def test_oracle_matches_banded_lapack(orc, solvedim):
    shape = (5, 7, 9)
    a, b, c, d = seeded.trid_system(shape, solvedim, 3)
    x = d.copy()
    oracle_solve(orc, a, b, c, x, solvedim)
    ax = 2 - solvedim
    A, B, C, D, X = (np.moveaxis(t, ax, -1).reshape(-1, shape[ax]) for t in (a, b, c, d, x))
    for l in range(A.shape[0]):
        ab = np.zeros((3, shape[ax]))
        ab[0, 1:] = C[l, :-1]
        ab[1] = B[l]
        ab[2, :-1] = A[l, 1:]
        ref = solve_banded((1, 1), ab, D[l])
        np.testing.assert_allclose(X[l], ref, rtol=1e-12, atol=1e-14)


def test_oracle_inc_adds_and_keeps_d(orc):
    a, b, c, d = seeded.trid_system((4, 6), 0, 5)
    x = d.copy()
    oracle_solve(orc, a, b, c, x, 0)
    u = np.full_like(d, 2.5)
    d0 = d.copy()
    oracle_solve(orc, a, b, c, d, 0, u=u)
    assert np.array_equal(d, d0)
    np.testing.assert_allclose(u, 2.5 + x, rtol=1e-15)
