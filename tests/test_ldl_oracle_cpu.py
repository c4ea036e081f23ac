"""The NumPy restatement of Bunch-Kaufman LDL^T (oracle/ldl_ref.py, the checker of the
device factorisation) against LAPACK's ?sytrf through scipy.linalg.ldl: the library routine
the reference calls when it switches its Schur system to the indefinite solver
(linalg/hdsdp_linsolver.c:1118-1190). Same permutation, same pivot blocks, same factors."""
from __future__ import annotations

import numpy as np
import pytest
import scipy.linalg as sl

from oracle import ldl_ref as R


def _cases():
    rng = np.random.default_rng(2024)
    for n in (1, 2, 5, 20, 60, 150):
        B = rng.standard_normal((n, n))
        yield "random%d" % n, (B + B.T) / 2
        Z = rng.standard_normal((n, n))
        Z = (Z + Z.T) / 2
        np.fill_diagonal(Z, 0.0)
        if n > 1:
            yield "zero_diagonal%d" % n, Z
        W = (B + B.T) / 2
        W[np.diag_indices(n)] *= 0.1
        yield "small_diagonal%d" % n, W
        P = rng.standard_normal((n, n))
        yield "positive_definite%d" % n, P @ P.T + n * np.eye(n)


@pytest.mark.parametrize("name,S", list(_cases()), ids=[c[0] for c in _cases()])
def test_restatement_matches_lapack(name, S):
    perm, sizes, D, L = R.bunch_kaufman(S)
    lu, d, sp = sl.ldl(S, lower=True)
    np.testing.assert_array_equal(perm, sp)
    scale = max(1.0, np.abs(S).max())
    assert np.abs(lu[sp] - L).max() <= 1e-10
    assert np.abs(d - D).max() <= 1e-10 * scale
    # the factorisation and the solve
    assert np.abs(L @ D @ L.T - S[np.ix_(perm, perm)]).max() <= 1e-12 * scale * S.shape[0]
    b = np.arange(1.0, S.shape[0] + 1.0)
    x = R.solve((perm, sizes, D, L), b)
    np.testing.assert_allclose(S @ x, b, rtol=0, atol=1e-9 * np.abs(b).max() * np.linalg.cond(S))
    two, neg, pos = R.inertia((perm, sizes, D, L))
    ev = np.linalg.eigvalsh(S)
    assert (neg, pos) == (int((ev < 0).sum()), int((ev > 0).sum()))
    assert two == sizes.count(2)


def test_zero_pivot_column_is_reported():
    with pytest.raises(ZeroDivisionError):
        R.bunch_kaufman(np.zeros((3, 3)))
