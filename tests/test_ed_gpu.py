"""Errors of the GPU paths against FP64 exact diagonalisation (ED).

The mixed-precision error is stated against ED, not against the GPU's own
FP64 path:

* DOS: KPM moments of the same seeded sample vectors from the eigen-
  decomposition (oracle.kpm_moments_ed) on the orthogonal pz graphene of the
  DOS benchmark at its full size (60 x 60 cells, 7,200 orbitals, R = 8
  random phases, 512 moments) and on a diamond LCAO sandwich Z^H H Z
  (Z the graph-local S^-1/2 by the reference's eigen route on the host),
  the DOS on 2,001 points.  FP64: moments within 1e-10 of mu_0 and DOS
  within 1e-10 of its peak; mixed (FP32 matrices and vectors, FP64 rescale
  and dots): DOS within 1e-5 of its peak.
* Conductivity: the Greenwood sigma(E) of dc_spectrum_fftcheb with the N
  unit vectors as samples (an exact trace) against the ED Kubo-Greenwood
  sum (oracle.kubo_greenwood_ed, pinned to the reference's own ED sum in
  tests/golden/ed_greenwood.npz).  FP64 within 1e-10 of the peak; FP32
  vectors within 1e-5 of the peak.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
X_GRID = np.linspace(-0.999, 0.999, 2001)


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    torch.cuda.set_device(0)
    return torch


def csr(A: np.ndarray):
    """Dense matrix -> scalar-block BSR arrays of its nonzeros."""
    from rsatb_b200.lattice import BsrArrays
    rows, cols = np.nonzero(A)
    n = A.shape[0]
    row_ptr = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=n))]).astype(np.int32)
    return BsrArrays(row_ptr, cols.astype(np.int32), A[rows, cols].reshape(-1, 1, 1).copy(), 1)


def dev(A, imaginary=False):
    from rsatb_b200.vbcsr import BlockSpMat
    return BlockSpMat(A.row_ptr, A.col_ind, A.values, A.block_size, A.n_block_cols,
                      imaginary=imaginary)


def dos_err(mu, mu_ref):
    rho = oracle.density(np.asarray(mu), X_GRID, 1e-3)
    ref = oracle.density(np.asarray(mu_ref), X_GRID, 1e-3)
    return float(np.abs(rho - ref).max() / np.abs(ref).max())


def check_against_ed(torch, cheby, psi, dense_op, n_moments):
    """FP64 and mixed moments of cheby on psi against the ED moments of
    dense_op on the same window; returns (fp64 DOS error, mixed DOS error)."""
    from rsatb_b200.calc import kpm_dos_moments
    c, hw = cheby.center, cheby.half_width
    ref = oracle.kpm_moments_ed(dense_op, psi.cpu().numpy(), c, hw, n_moments)
    mu64 = kpm_dos_moments(cheby, psi, n_moments)
    assert np.abs(mu64 - ref).max() <= 1e-10 * abs(ref[0])
    e64 = dos_err(mu64, ref)
    assert e64 <= 1e-10, e64
    lo = torch.complex64 if psi.is_complex() else torch.float32
    mu32 = kpm_dos_moments(cheby.astype("f32"), psi.to(lo), n_moments)
    e32 = dos_err(mu32, ref)
    assert e32 <= 1e-5, e32
    return e64, e32


def test_graphene_dos_against_ed(torch_cuda):
    """Config 1 at full size: 60 x 60 pz graphene, R = 8, 512 moments."""
    torch = torch_cuda
    from rsatb_b200 import lattice
    from rsatb_b200.calc import Chebyshev
    from rsatb_b200.vbcsr import set_random
    H, _, _ = lattice.graphene(60, 60)
    cheby = Chebyshev(dev(H), -8.6, 8.6)  # |E| <= 3|t| = 8.1 eV, 0.5 eV pad
    psi = torch.empty(H.n_rows, 8, dtype=torch.complex128, device="cuda")
    set_random(psi, 20240917)
    e64, e32 = check_against_ed(torch, cheby, psi, H.to_dense(), 512)
    print(f"graphene 60x60 DOS vs ED: fp64 {e64:.2e}, mixed {e32:.2e}")


def test_diamond_sandwich_dos_against_ed(torch_cuda):
    """Non-orthogonal diamond LCAO (L = 3, 1,728 orbitals), Z^H H Z with
    the graph-local factor, R = 16 Rademacher vectors, 256 moments."""
    torch = torch_cuda
    from rsatb_b200 import lattice
    from rsatb_b200.calc import Chebyshev, ISQRTMPreconditioner
    from rsatb_b200.vbcsr import set_random
    H, S = lattice.diamond_lcao(L=3, seed=7)
    Z = lattice.BsrArrays(S.row_ptr, S.col_ind,
                          oracle.graph_inverse_sqrt_eigen(S.row_ptr, S.col_ind, S.values, 8), 8)
    Zd = Z.to_dense()
    op = Zd.T @ H.to_dense() @ Zd
    w = np.linalg.eigvalsh(op)
    cheby = Chebyshev(dev(H), w[0] - 0.5, w[-1] + 0.5,
                      preconditioner=ISQRTMPreconditioner(dev(Z)))
    psi = torch.empty(H.n_rows, 16, dtype=torch.float64, device="cuda")
    set_random(psi, 20240917, orbitals_per_atom=8)
    e64, e32 = check_against_ed(torch, cheby, psi, op, 256)
    print(f"diamond L=3 sandwich DOS vs ED: fp64 {e64:.2e}, mixed {e32:.2e}")


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_greenwood_sigma_against_ed(torch_cuda, precision):
    torch = torch_cuda
    from rsatb_b200.calc import Chebyshev
    from rsatb_b200.transport import dc_spectrum_fftcheb
    z = np.load(GOLDEN / "ed_greenwood.npz")
    H, V = z["H"], z["V"]
    c, hw, M = float(z["center"]), float(z["half_width"]), int(z["n_moments"])
    N = H.shape[0]
    cheby = Chebyshev(dev(csr(H)), c - hw, c + hw)
    Wd = dev(csr(V.imag.copy()), imaginary=True)  # V = i W, W real antisymmetric
    dt = torch.complex128
    if precision == "f32":
        cheby, Wd, dt = cheby.astype("f32"), Wd.astype("f32"), torch.complex64
    psi = torch.eye(N, dtype=dt, device="cuda").contiguous()  # every unit vector: exact trace
    sigma, energy = dc_spectrum_fftcheb(cheby, Wd, Wd, Wd, psi, M, prefactor=1.0)
    E, K = oracle.kubo_greenwood_ed(H, V, c, hw, M)
    assert np.abs(energy - E).max() < 1e-12
    tol = 1e-10 if precision == "f64" else 1e-5
    for comp in (0, 3, 5):  # xx, yy, zz
        err = float(np.abs(sigma[:, comp] - K).max() / np.abs(K).max())
        assert err <= tol, (comp, err)
    print(f"Greenwood sigma vs ED ({precision}): "
          f"{float(np.abs(sigma[:, 0] - K).max() / np.abs(K).max()):.2e}")
