"""The host Ritz solve of rsatb_lanczos_extremes (implicit QL on a symmetric
tridiagonal matrix, last row of the eigenvectors only) against numpy's
eigh: eigenvalues to 1e-12 of the spectral radius, |last components| to
1e-10, including split blocks, a 1 x 1 and a 2 x 2 case and a Lanczos-like
matrix with clustered extreme eigenvalues."""
from __future__ import annotations

import numpy as np
import pytest


def dense(d, e):
    return np.diag(d) + np.diag(e, 1) + np.diag(e, -1)


@pytest.mark.parametrize("case", ["random", "split", "one", "two", "clustered", "zero"])
def test_tridiag_eigen_matches_eigh(case):
    from rsatb_b200.bounds import tridiag_eigen
    rng = np.random.default_rng(17)
    if case == "random":
        d, e = rng.standard_normal(60), rng.standard_normal(59)
    elif case == "split":
        d, e = rng.standard_normal(30), rng.standard_normal(29)
        e[[4, 11, 12, 25]] = 0.0
    elif case == "one":
        d, e = np.array([2.5]), np.zeros(0)
    elif case == "two":
        d, e = np.array([1.0, -3.0]), np.array([0.75])
    elif case == "clustered":
        # alpha/beta of a Lanczos run on diag(linspace) with two close extremes
        lam = np.concatenate([[-5.0, -4.999999], np.linspace(-2, 2, 200), [6.0, 6.0000001]])
        n, k = lam.size, 80
        q = rng.standard_normal(n)
        q /= np.linalg.norm(q)
        Q = np.zeros((n, k))
        d, e = np.zeros(k), np.zeros(k - 1)
        for j in range(k):
            Q[:, j] = q
            w = lam * q
            d[j] = q @ w
            for _ in range(2):
                w -= Q[:, :j + 1] @ (Q[:, :j + 1].T @ w)
            if j + 1 < k:
                e[j] = np.linalg.norm(w)
                q = w / e[j]
    else:
        d, e = np.zeros(5), np.zeros(4)
    th, last = tridiag_eigen(d, e)
    w, V = np.linalg.eigh(dense(d, e))
    scale = max(1.0, np.abs(w).max())
    assert np.all(np.diff(th) >= 0)
    assert np.abs(th - w).max() <= 1e-12 * scale
    if case not in ("clustered", "zero"):
        # eigenvectors of (nearly) repeated eigenvalues are not unique
        assert np.abs(np.abs(last) - np.abs(V[-1])).max() <= 1e-10
    else:
        # the residual norms |y_m| over a cluster are invariant: compare sums of squares
        for lo, hi in ((0, 2), (len(w) - 2, len(w))):
            assert abs((last[lo:hi] ** 2).sum() - (V[-1, lo:hi] ** 2).sum()) <= 1e-10


def test_tridiag_eigen_rejects_bad_lengths():
    from rsatb_b200.bounds import tridiag_eigen
    with pytest.raises(ValueError):
        tridiag_eigen(np.zeros(4), np.zeros(4))
