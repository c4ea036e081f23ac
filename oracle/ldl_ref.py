"""NumPy restatement of the symmetric indefinite factorisation the reference switches its Schur
system to when the Cholesky fails.

TEST INFRASTRUCTURE ONLY: the checker for the device LDL^T (hdsdp_b200/csrc/ldl.cu); never
imported by the product package.

The reference calls LAPACK dsytrf / dsytrs on the full Schur matrix
(linalg/hdsdp_linsolver.c:1118-1190; the switch at :1367-1380 and :1407-1420). LAPACK is a
third-party dependency, not part of the reference's sources (the build here links the
OpenBLAS bundled with SciPy). Its published algorithm is the Bunch-Kaufman partial pivoting
of dsytf2, restated here for the lower triangle:

  alpha = (1 + sqrt 17) / 8
  at step k: colmax = max_{i>k} |A(i,k)| at row imax;
    |A(k,k)| >= alpha colmax                          -> 1 x 1 pivot, no interchange
    else rowmax = max_{j in [k,n), j != imax} |A(imax,j)|
      |A(k,k)| >= alpha colmax (colmax / rowmax)      -> 1 x 1 pivot, no interchange
      |A(imax,imax)| >= alpha rowmax                  -> 1 x 1 pivot, interchange k, imax
      otherwise                                       -> 2 x 2 pivot, interchange k+1, imax
  then the rank-1 or rank-2 update of the trailing matrix.

The result is written as P A P^T = L D L^T (perm[a] = the original index of row a, L unit
lower, D block diagonal), the form scipy.linalg.ldl returns (it calls LAPACK ?sytrf), which
pins this restatement to the library the reference calls; tests/test_ldl_oracle_cpu.py holds
that check. Ties in the column search go to the smallest row, as LAPACK's idamax does.
"""
from __future__ import annotations

import numpy as np

ALPHA = (1.0 + np.sqrt(17.0)) / 8.0


def bunch_kaufman(S):
    """Factor the symmetric S (only its lower triangle is read). Returns (perm, sizes, D, L) with
    sizes the pivot block sizes in elimination order, or raises ZeroDivisionError on an exactly
    zero pivot column."""
    A = np.tril(np.array(S, dtype=np.float64))
    A = A + np.tril(A, -1).T           # full symmetric working copy
    n = A.shape[0]
    perm = np.arange(n)
    Lf = np.zeros((n, n))              # multipliers, rows in the current order
    D = np.zeros((n, n))
    sizes = []
    k = 0
    while k < n:
        col = np.abs(A[k + 1:, k])
        colmax = col.max() if col.size else 0.0
        imax = k + 1 + int(np.argmax(col)) if col.size else k
        absakk = abs(A[k, k])
        if max(absakk, colmax) == 0.0:
            raise ZeroDivisionError("zero pivot column at step %d" % (k + 1))
        kp, kstep = k, 1
        if absakk < ALPHA * colmax:
            row = np.abs(A[imax, k:]).copy()
            row[imax - k] = 0.0
            rowmax = row.max()
            if absakk >= ALPHA * colmax * (colmax / rowmax):
                kp = k
            elif abs(A[imax, imax]) >= ALPHA * rowmax:
                kp = imax
            else:
                kp, kstep = imax, 2
        kk = k + kstep - 1
        if kp != kk:
            A[[kk, kp], :] = A[[kp, kk], :]
            A[:, [kk, kp]] = A[:, [kp, kk]]
            Lf[[kk, kp], :k] = Lf[[kp, kk], :k]
            perm[[kk, kp]] = perm[[kp, kk]]
        if kstep == 1:
            d = A[k, k]
            D[k, k] = d
            x = A[k + 1:, k].copy()
            l = x / d
            Lf[k + 1:, k] = l
            A[k + 1:, k + 1:] -= np.outer(l, x)
        else:
            blk = A[k:k + 2, k:k + 2].copy()
            D[k:k + 2, k:k + 2] = blk
            X = A[k + 2:, k:k + 2].copy()
            Lk = X @ np.linalg.inv(blk)
            Lf[k + 2:, k:k + 2] = Lk
            A[k + 2:, k + 2:] -= Lk @ X.T
        sizes.append(kstep)
        k += kstep
    L = Lf + np.eye(n)
    return perm, sizes, D, L


def solve(factor, b):
    """x = S^-1 b from bunch_kaufman's result."""
    perm, _, D, L = factor
    y = np.asarray(b, dtype=np.float64)[perm]
    z = np.linalg.solve(L, y)
    w = np.linalg.solve(D, z)
    v = np.linalg.solve(L.T, w)
    x = np.empty_like(v)
    x[perm] = v
    return x


def inertia(factor):
    """(2 x 2 pivots, negative, positive eigenvalues) of D."""
    _, sizes, D, _ = factor
    neg = pos = two = 0
    k = 0
    for s in sizes:
        ev = np.linalg.eigvalsh(D[k:k + s, k:k + s])
        neg += int((ev < 0).sum())
        pos += int((ev > 0).sum())
        two += s == 2
        k += s
    return two, neg, pos
