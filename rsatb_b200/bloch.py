"""Operators at a k-point from their real-space images, summed on the GPU.

The reference builds H(k) by adding every bond block H_ij(R) times the Bloch
phase exp(-2 pi i k . R) into block (i, j) (rsatb/operator/block_assembly.hpp:
31-100), and the commutator velocity with the extra factor i (R + r_j - r_i)_a
(rsatb/operator/commutator_velocity.hpp:114-255).  ``ImageOperator`` holds the
bonds on the device, sorted by output block, with the pattern of H(k) (the
union of the (i, j) pairs over images) built once; ``at_k`` and
``velocity_at_k`` fill a C128 BlockSpMat with one kernel launch each
(``rsatb_bloch_sum``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _capi
from ._capi import check, lib
from .vbcsr import BlockSpMat, context


def image_pattern(rows, cols, n_block_rows: int, n_block_cols: int):
    """The pattern of H(k) from the bonds (rows[e], cols[e]): returns
    (order, slot_ptr, row_ptr, col_ind) with the bonds in `order` sorted by
    output block (row, col), bonds of one block kept in input order;
    bonds order[slot_ptr[s]:slot_ptr[s + 1]] sum into block s, whose column
    is col_ind[s]; row_ptr is the CSR row pointer over the blocks."""
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    n = rows.size
    order = np.lexsort((cols, rows))
    key = rows[order] * int(n_block_cols) + cols[order]
    first = np.ones(n, dtype=bool)
    first[1:] = key[1:] != key[:-1]
    slot_start = np.flatnonzero(first)
    slot_ptr = np.append(slot_start, n).astype(np.int64)
    prow = rows[order][slot_start]
    col_ind = cols[order][slot_start].astype(np.int32)
    row_ptr = np.zeros(int(n_block_rows) + 1, dtype=np.int32)
    np.add.at(row_ptr, prow + 1, 1)
    row_ptr = np.cumsum(row_ptr).astype(np.int32)
    return order, slot_ptr, row_ptr, col_ind


class ImageOperator:
    """Bonds (rows[e], cols[e], shifts[e]) with blocks[e] (b x b, real or
    complex); shifts in the units k is given against (fractional for integer
    lattice images).  bond_vectors[e] = R + r_j - r_i in Cartesian units
    (needed for velocities only)."""

    def __init__(self, rows, cols, shifts, blocks, block_size: int, n_block_rows: int,
                 bond_vectors=None, n_block_cols: int | None = None, device=None):
        rows = np.asarray(rows, dtype=np.int64)
        cols = np.asarray(cols, dtype=np.int64)
        shifts = np.asarray(shifts, dtype=np.float64).reshape(-1, 3)
        b = int(block_size)
        blocks = np.asarray(blocks)
        n = rows.size
        if cols.size != n or shifts.shape[0] != n or blocks.shape != (n, b, b):
            raise ValueError("rows, cols, shifts and blocks must describe the same bonds")
        nbc = int(n_block_cols) if n_block_cols is not None else int(n_block_rows)
        if n and (rows.min() < 0 or rows.max() >= n_block_rows or cols.min() < 0
                  or cols.max() >= nbc):
            raise ValueError("bond index outside the matrix")
        self.block_size, self.n_block_rows, self.n_block_cols = b, int(n_block_rows), nbc
        # Bonds sorted by output block (row, col); equal blocks keep input order.
        order, slot_ptr, self.row_ptr, self.col_ind = image_pattern(rows, cols,
                                                                    self.n_block_rows, nbc)
        self.nnz_blocks = self.col_ind.size
        self.ctx = context(device)
        dev = f"cuda:{self.ctx.device}"
        cplx = np.iscomplexobj(blocks)
        vals = np.ascontiguousarray(blocks[order], dtype=np.complex128 if cplx else np.float64)
        self._dtype = _capi.C128 if cplx else _capi.F64
        self._slot_ptr = torch.as_tensor(slot_ptr).to(dev)
        self._shifts = torch.as_tensor(np.ascontiguousarray(shifts[order])).to(dev)
        self._vals = torch.as_tensor(vals.view(np.float64).reshape(-1)).to(dev)
        self._bonds = None
        if bond_vectors is not None:
            bv = np.asarray(bond_vectors, dtype=np.float64).reshape(-1, 3)
            if bv.shape[0] != n:
                raise ValueError("bond_vectors must have one row per bond")
            self._bonds = [torch.as_tensor(np.ascontiguousarray(bv[order, a])).to(dev)
                           for a in range(3)]

    @property
    def shape(self):
        return (self.n_block_rows * self.block_size, self.n_block_cols * self.block_size)

    def _empty(self) -> BlockSpMat:
        zeros = np.zeros((self.nnz_blocks, self.block_size, self.block_size), dtype=np.complex128)
        return BlockSpMat(self.row_ptr, self.col_ind, zeros, self.block_size, self.n_block_cols,
                          device=self.ctx.device)

    def _sum(self, k, weights, imag_unit: bool) -> BlockSpMat:
        kk = np.ascontiguousarray(np.asarray(k, dtype=np.float64).reshape(3))
        out = self._empty()
        self.ctx.bind_stream()
        w = C.c_void_p(weights.data_ptr()) if weights is not None else None
        check(lib().rsatb_bloch_sum(self.ctx.handle, out.handle,
                                    C.c_void_p(self._slot_ptr.data_ptr()),
                                    C.c_void_p(self._shifts.data_ptr()),
                                    C.c_void_p(self._vals.data_ptr()), self._dtype, w,
                                    kk.ctypes.data_as(C.POINTER(C.c_double)), int(imag_unit)))
        return out

    def at_k(self, k) -> BlockSpMat:
        """H(k) = sum_R H(R) exp(-2 pi i k . R) as a C128 BlockSpMat."""
        return self._sum(k, None, False)

    def velocity_at_k(self, k, axis: int) -> BlockSpMat:
        """V_a(k) = i sum_R (R + r_j - r_i)_a H(R) exp(-2 pi i k . R)."""
        if self._bonds is None:
            raise ValueError("velocities need the bond vectors")
        if axis not in (0, 1, 2):
            raise ValueError("axis must be 0, 1 or 2")
        return self._sum(k, self._bonds[axis], True)
