"""GPU checks of two entry points against the reference's own test cases and
an exact-diagonalisation oracle: the batched CG on the cases of
rsatb/calc/test/test_solver.cpp, and the orbital-resolved KPM LDOS against
sum_n |U_in|^2 T_m(x_n).  Collected after the main suites."""
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


def _csr_dev(A):
    """A dense matrix as a device BSR of 1x1 blocks (its nonzero pattern)."""
    from rsatb_b200.vbcsr import BlockSpMat
    rows, cols = np.nonzero(A)
    row_ptr = np.zeros(A.shape[0] + 1, dtype=np.int32)
    np.add.at(row_ptr, rows + 1, 1)
    return BlockSpMat(np.cumsum(row_ptr), cols, A[rows, cols].reshape(-1, 1, 1), 1)


def test_cg_reference_cases(torch_cuda):
    """The cases of the reference's test_solver.cpp: S = 2 I gives X = B / 2;
    a 1-D Laplacian with a varying diagonal is solved to the residual
    tolerance, plainly and with a diagonal symmetric preconditioner."""
    torch = torch_cuda
    from rsatb_b200.calc import ISQRTMPreconditioner, cg_solve
    rng = np.random.default_rng(4)
    n = 40
    B = rng.standard_normal((n, 3))
    Bd = torch.as_tensor(B).cuda().contiguous()
    X = torch.zeros_like(Bd)
    it, _ = cg_solve(_csr_dev(2.0 * np.eye(n)), Bd, X, tol=1e-8, max_iter=100)
    assert it == 1 and np.abs(X.cpu().numpy() - B / 2).max() < 1e-13
    A = np.diag(2.0 + 0.1 * (np.arange(n) % 3)) - np.eye(n, k=1) - np.eye(n, k=-1)
    X = torch.zeros_like(Bd)
    it, res = cg_solve(_csr_dev(A), Bd, X, tol=1e-8, max_iter=1000)
    assert res < 1e-8 and np.abs(A @ X.cpu().numpy() - B).max() < 1e-7
    D = np.diag(1.0 / np.sqrt(np.diag(A)))
    X = torch.zeros_like(Bd)
    it2, res2 = cg_solve(_csr_dev(A), Bd, X, tol=1e-10, max_iter=1000,
                         preconditioner=ISQRTMPreconditioner(_csr_dev(D)))
    assert res2 < 1e-10 and np.abs(A @ X.cpu().numpy() - B).max() < 1e-8


@pytest.mark.parametrize("precision,tol", [("f64", 1e-10), ("mixed", 1e-4)])
def test_compute_ldos_matches_exact_diagonalisation(precision, tol):
    """Orbital LDOS: the local moments <e_i|T_n|e_i> against the FP64
    exact-diagonalisation oracle sum_n |U_in|^2 T_m(x_n), and the LDOS
    against the oracle's density of those moments (error peak-normalised,
    as for the DOS)."""
    import torch
    from rsatb_b200 import lattice
    from rsatb_b200.calc import Chebyshev, dos_energy_grid, dos_moment_count, kpm_ldos_moments
    from rsatb_b200.driver import RSATB, SetupOptions
    from rsatb_b200.vbcsr import BlockSpMat
    torch.cuda.set_device(0)
    H, _, _ = lattice.graphene(8, 7)
    emin, emax = -8.6, 8.7
    c, hw = (emax + emin) / 2, (emax - emin) / 2
    w, U = np.linalg.eigh(H.to_dense())
    theta = np.arccos((w - c) / hw)
    orbs = [0, 5, 17, 111]
    M = 64
    mu_ed = np.array([[np.sum(U[i] ** 2 * np.cos(m * theta)) for i in orbs] for m in range(M)])
    cheb = Chebyshev(BlockSpMat(H.row_ptr, H.col_ind, H.values, 1), emin, emax)
    if precision == "mixed":
        cheb = cheb.astype("f32")
    mu = kpm_ldos_moments(cheb, orbs, M)
    assert mu.shape == (M, len(orbs))
    # A single unit column does not average the FP32 rounding away as the
    # stochastic DOS does: mixed-mode local moments to 5e-5, LDOS to 1e-4.
    assert np.abs(mu - mu_ed).max() < (1e-10 if precision == "f64" else 5e-5)
    calc = RSATB(H, SetupOptions(energy_bounds=(emin, emax), precision=precision))
    dE = 0.4
    ldos, omega = calc.compute_ldos(orbs, dE)
    x, _, nt = dos_energy_grid(emin, emax, dE)
    N = dos_moment_count(hw, dE)
    for j, i in enumerate(orbs):
        mu_i = np.array([np.sum(U[i] ** 2 * np.cos(m * theta)) for m in range(N)])
        want = 2.0 * oracle.density(mu_i.astype(np.complex128), x, 0.5 / nt)
        assert np.abs(ldos[0, j] - want).max() < tol * want.max()
