"""Global sparse Newton-Schulz refinement (rsatb_inverse_sqrt_refine) against
the oracle's dense restatement of rsatb::calc::inverse_sqrt's loop
(rsatb/calc/isqrtm.hpp:620-800) and test_isqrtm.cpp's semantics.

* With no drop threshold and X reformed every step, the device iteration is
  the dense one up to FP64 summation order: same steps, factor within 1e-10
  (diamond L = 2, 8x8 blocks, from the same graph-local seed).  With the
  propagation route the factor stays within 1e-9.
* test_isqrtm.cpp's chains: the 2000-site shifted Laplacian converges to
  tol 1e-7 at sptol 1e-8 with an applied residual below 1e-5 that an
  independent probe (numpy, five vectors) confirms within a factor of ten;
  on 24 sites, off-diagonal 0.6 diverges, 0.49 converges, and a one-step cap
  is neither.
* At the default sptol 1e-6 on diamond L = 3 the loop stops at the drop
  floor and Z^T S Z stays within 1e-4 of the identity.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    torch.cuda.set_device(0)
    return torch


def dense(A):
    return A.to_dense()


def run(S_arrays, **opts):
    from rsatb_b200.isqrt import InverseSqrtOptions, inverse_sqrt
    Z, rep = inverse_sqrt(S_arrays, InverseSqrtOptions(**opts))
    return Z.to_arrays(), rep


def csr(S: np.ndarray, rp, ci):
    from rsatb_b200.lattice import BsrArrays
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    return BsrArrays(rp, ci, S[rows, ci].reshape(-1, 1, 1).copy(), 1)


@pytest.mark.parametrize("route", [1, 0])
def test_diamond_refinement_equals_the_dense_iteration(torch_cuda, route):
    from rsatb_b200 import lattice
    from rsatb_b200.isqrt import graph_inverse_sqrt
    _, S = lattice.diamond_lcao(L=2, seed=3)
    seed = graph_inverse_sqrt(S)
    Sd = dense(S)
    Z_ref, r_ref = oracle.ns_refine_dense(Sd, dense(seed), 8, tol=1e-11, maxit=12)
    Z, rep = run(S, tol=1e-11, sptol=0.0, maxit=12, route=route)
    Zd = dense(Z)
    err = np.abs(Zd - Z_ref).max() / np.abs(Z_ref).max()
    assert err <= (1e-10 if route == 1 else 1e-9), err
    assert rep.converged == r_ref["converged"]
    if route == 1:
        assert rep.steps == r_ref["steps"] and rep.propagations == 0
    assert np.abs(Zd.T @ Sd @ Zd - np.eye(Sd.shape[0])).max() < 1e-9


def test_long_chain_converges_like_test_isqrtm(torch_cuda):
    """test_isqrtm.cpp:79-126: 2000 sites, S = Laplacian + I, tol 1e-7,
    sptol 1e-8, maxit 50."""
    S, rp, ci = oracle.chain_overlap(2000, 3.0, -1.0)
    Z, rep = run(csr(S, rp, ci), tol=1e-7, sptol=1e-8, maxit=50)
    assert rep.converged and not rep.hit_maxiter and rep.residual <= 1e-7
    assert np.isfinite(rep.applied_residual) and rep.applied_residual <= 1e-5
    Zd = dense(Z)
    rng = np.random.default_rng(1337)
    worst = 0.0
    for _ in range(5):
        v = rng.uniform(-1.0, 1.0, 2000)
        out = Zd.T @ (S @ (Zd @ v))
        worst = max(worst, np.linalg.norm(out - v) / np.linalg.norm(v))
    assert worst <= 1e-5
    assert 0.1 < rep.applied_residual / worst < 10.0


@pytest.mark.parametrize("off,maxit,tol,want", [(0.60, 20, 1e-10, "diverged"),
                                                (0.49, 20, 1e-10, "converged"),
                                                (0.49, 1, 1e-16, "capped")])
def test_short_chain_verdicts(torch_cuda, off, maxit, tol, want):
    """test_isqrtm.cpp:128-186, sptol 1e-12."""
    S, rp, ci = oracle.chain_overlap(24, 1.0, off)
    _, rep = run(csr(S, rp, ci), tol=tol, sptol=1e-12, maxit=maxit)
    if want == "diverged":
        assert not rep.converged and rep.diverged
    elif want == "converged":
        assert rep.converged and not rep.diverged
    else:
        assert not rep.converged and not rep.diverged and rep.hit_maxiter


def test_default_threshold_on_diamond(torch_cuda):
    from rsatb_b200 import lattice
    _, S = lattice.diamond_lcao(L=3, seed=7)
    Z, rep = run(S)  # tol 1e-7, sptol 1e-6, maxit 20, routes by cost
    assert not rep.diverged and rep.steps >= 1
    Sd, Zd = dense(S), dense(Z)
    assert np.abs(Zd.T @ Sd @ Zd - np.eye(Sd.shape[0])).max() < 1e-4
    assert rep.applied_residual < 1e-4
    print(f"diamond L=3: steps {rep.steps}, residual {rep.residual:.2e}, applied "
          f"{rep.applied_residual:.2e}, nnz {rep.nnz_blocks} ({rep.nnz_blocks / 216:.0f}/row), "
          f"reforms {rep.reforms}, propagations {rep.propagations}")
