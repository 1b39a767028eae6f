"""Host side of the k-point assembly: the pattern of H(k) and the bond order
that rsatb_bloch_sum sums in (no GPU needed)."""
from __future__ import annotations

import numpy as np

import oracle
from rsatb_b200 import lattice
from rsatb_b200.bloch import image_pattern
from rsatb_b200.lattice import BsrArrays


def _check(rows, cols, shifts, blocks, nbr, nbc, k):
    order, slot_ptr, row_ptr, col_ind = image_pattern(rows, cols, nbr, nbc)
    assert sorted(order.tolist()) == list(range(len(rows)))
    prow = np.repeat(np.arange(nbr), np.diff(row_ptr))
    assert row_ptr[-1] == col_ind.size == slot_ptr.size - 1
    for i in range(nbr):   # columns sorted and unique within a row
        c = col_ind[row_ptr[i]:row_ptr[i + 1]]
        assert np.all(np.diff(c) > 0)
    vals = np.zeros((col_ind.size,) + blocks.shape[1:], dtype=np.complex128)
    ph = np.exp(-2j * np.pi * (shifts @ np.asarray(k)))
    for s in range(col_ind.size):
        bonds = order[slot_ptr[s]:slot_ptr[s + 1]]
        assert np.all(rows[bonds] == prow[s]) and np.all(cols[bonds] == col_ind[s])
        assert np.all(np.diff(bonds) > 0)     # input order within a block
        vals[s] = np.sum(ph[bonds, None, None] * blocks[bonds], axis=0)
    dense = BsrArrays(row_ptr, col_ind, vals, blocks.shape[1], nbc).to_dense()
    want = oracle.bloch_dense(rows, cols, shifts, blocks, nbr, k, n_block_cols=nbc)
    assert np.abs(dense - want).max() < 1e-13


def test_image_pattern_random_bonds():
    rng = np.random.default_rng(2)
    n = 200
    rows = rng.integers(0, 15, n)
    cols = rng.integers(0, 11, n)
    rows[:30], cols[:30] = 3, 5           # many images of one block
    shifts = rng.integers(-2, 3, (n, 3)).astype(np.float64)
    blocks = rng.standard_normal((n, 2, 2)) + 1j * rng.standard_normal((n, 2, 2))
    _check(rows, cols, shifts, blocks, 15, 11, [0.13, -0.4, 0.27])


def test_image_pattern_graphene_primitive_and_supercell():
    for n1, n2 in ((1, 1), (2, 3), (4, 4)):
        r, c, sh, bl, bv, n, cell = lattice.graphene_images(n1, n2)
        _check(r, c, sh, bl, n, n, [0.21, 0.35, 0.0])
    r, c, sh, bl, bv, n, cell = lattice.graphene_images(1, 1)
    order, slot_ptr, row_ptr, col_ind = image_pattern(r, c, n, n)
    assert col_ind.tolist() == [1, 0] and np.diff(slot_ptr).tolist() == [3, 3]
