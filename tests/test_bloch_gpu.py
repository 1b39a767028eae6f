"""Operators at a k-point from real-space images (rsatb_bloch_sum) against
the oracle's dense Bloch sum (BlochPhase / AddLocalBlock,
rsatb/operator/block_assembly.hpp:31-100; the commutator velocity of
rsatb/operator/commutator_velocity.hpp:114-255), the graphene band
structure, and KPM moments of H(k)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from _util import rel_err, to_oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    torch.cuda.set_device(0)
    return torch


def _op_dense(op, M):
    from rsatb_b200.lattice import BsrArrays
    return BsrArrays(op.row_ptr, op.col_ind, M.values_tensor().cpu().numpy(), op.block_size,
                     op.n_block_cols).to_dense()


def _random_images(seed, n_blocks=20, b=3, n_bonds=150, complex_values=True):
    rng = np.random.default_rng(seed)
    rows = rng.integers(0, n_blocks, n_bonds)
    cols = rng.integers(0, n_blocks, n_bonds)
    rows[:20] = 4            # several images of one block
    cols[:20] = 7
    shifts = rng.integers(-2, 3, (n_bonds, 3)).astype(np.float64)
    blocks = rng.standard_normal((n_bonds, b, b))
    if complex_values:
        blocks = blocks + 1j * rng.standard_normal((n_bonds, b, b))
    vecs = rng.standard_normal((n_bonds, 3))
    return rows, cols, shifts, blocks, vecs, n_blocks, b


@pytest.mark.parametrize("complex_values", [True, False])
def test_bloch_sum_matches_oracle(torch_cuda, complex_values):
    from rsatb_b200.bloch import ImageOperator
    rows, cols, shifts, blocks, vecs, n, b = _random_images(3, complex_values=complex_values)
    op = ImageOperator(rows, cols, shifts, blocks, b, n, bond_vectors=vecs)
    for k in ([0.0, 0.0, 0.0], [0.21, -0.37, 0.05], [0.5, 0.5, 0.5]):
        got = _op_dense(op, op.at_k(k))
        want = oracle.bloch_dense(rows, cols, shifts, blocks, n, k)
        assert np.abs(got - want).max() < 1e-13 * np.abs(want).max()
        for a in range(3):
            got_v = _op_dense(op, op.velocity_at_k(k, a))
            want_v = oracle.bloch_dense(rows, cols, shifts, blocks, n, k, weights=vecs[:, a],
                                        imag_unit=True)
            assert np.abs(got_v - want_v).max() < 1e-13 * np.abs(want_v).max()


def test_graphene_bands_and_gamma(torch_cuda):
    """The primitive cell gives +-|t f(k)|; a 3 x 3 supercell at K holds the
    nine folded primitive k-points; k = 0 is graphene()'s supercell H."""
    from rsatb_b200 import lattice
    from rsatb_b200.bloch import ImageOperator
    r, c, sh, bl, bv, n, cell = lattice.graphene_images(1, 1)
    op = ImageOperator(r, c, sh, bl, 1, n, bond_vectors=bv)
    k = np.array([0.2, 0.13, 0.0])
    ev = np.linalg.eigvalsh(_op_dense(op, op.at_k(k)))
    f = 2.7 * abs(1 + np.exp(-2j * np.pi * k[0]) + np.exp(-2j * np.pi * k[1]))
    assert np.allclose(ev, [-f, f], rtol=0, atol=1e-13)
    r, c, sh, bl, bv, n, cell = lattice.graphene_images(3, 3)
    op = ImageOperator(r, c, sh, bl, 1, n, bond_vectors=bv)
    K = np.array([0.3, -0.2, 0.0])
    ev = np.sort(np.linalg.eigvalsh(_op_dense(op, op.at_k(K))))
    want = []
    for m1 in range(3):
        for m2 in range(3):
            kp = (K[:2] + [m1, m2]) / 3
            ff = 2.7 * abs(1 + np.exp(-2j * np.pi * kp[0]) + np.exp(-2j * np.pi * kp[1]))
            want += [ff, -ff]
    assert np.abs(ev - np.sort(want)).max() < 1e-12
    H, _, _ = lattice.graphene(3, 3)
    assert np.abs(_op_dense(op, op.at_k([0, 0, 0])) - H.to_dense()).max() == 0.0


def test_kpm_moments_at_k_match_oracle(torch_cuda):
    """KPM moments of the complex H(k) (complex BSR through the fused step)
    against the oracle's recurrence on the same matrix."""
    torch = torch_cuda
    from rsatb_b200 import lattice
    from rsatb_b200.bloch import ImageOperator
    from rsatb_b200.calc import Chebyshev, kpm_dos_moments
    from rsatb_b200.lattice import BsrArrays
    from rsatb_b200.vbcsr import set_random
    r, c, sh, bl, bv, n, cell = lattice.graphene_images(6, 5)
    op = ImageOperator(r, c, sh, bl, 1, n, bond_vectors=bv)
    Hk = op.at_k([0.17, 0.41, 0.0])
    cheb = Chebyshev(Hk, -8.6, 8.7)
    psi = torch.empty(n, 4, dtype=torch.complex128, device="cuda")
    set_random(psi, 13)
    mu = kpm_dos_moments(cheb, psi, 96)
    A = BsrArrays(op.row_ptr, op.col_ind, Hk.values_tensor().cpu().numpy(), 1)
    want = oracle.kpm_moments(oracle.make_op(to_oracle(A), 0.05, 8.65), psi.cpu().numpy(), 96)
    assert np.abs(mu - want).max() < 1e-10 * abs(want[0])


def test_bad_arguments(torch_cuda):
    from rsatb_b200.bloch import ImageOperator
    rows, cols, shifts, blocks, vecs, n, b = _random_images(1)
    with pytest.raises(ValueError):
        ImageOperator(rows, cols, shifts[:-1], blocks, b, n)
    with pytest.raises(ValueError):
        ImageOperator(rows + n, cols, shifts, blocks, b, n)
    op = ImageOperator(rows, cols, shifts, blocks, b, n)
    with pytest.raises(ValueError):
        op.velocity_at_k([0, 0, 0], 0)
