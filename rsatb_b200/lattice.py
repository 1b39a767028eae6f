"""Seeded synthetic operators for the benchmark workloads.

The reference builds H and S from model files through vbcsr's AtomicData
(out of scope here); these generators produce the same kinds of operators
directly as uniform-block BSR arrays on the host, with atoms ordered as
generated (cell-major) and neighbour lists from explicit lattice
enumeration.  Every random draw comes from ``numpy.random.default_rng``
with an explicit seed, so the GPU path and the oracle see the same input.

A ``BsrArrays`` holds (row_ptr, col_ind, values[nnzb, b, b], b).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class BsrArrays:
    row_ptr: np.ndarray
    col_ind: np.ndarray
    values: np.ndarray
    block_size: int
    n_block_cols: int | None = None

    @property
    def n_block_rows(self) -> int:
        return self.row_ptr.size - 1

    @property
    def n_rows(self) -> int:
        return self.n_block_rows * self.block_size

    @property
    def nnz_blocks(self) -> int:
        return self.col_ind.size

    def to_dense(self) -> np.ndarray:
        b = self.block_size
        nbc = self.n_block_cols or self.n_block_rows
        A = np.zeros((self.n_block_rows * b, nbc * b), dtype=self.values.dtype)
        rows = np.repeat(np.arange(self.n_block_rows), np.diff(self.row_ptr))
        for k in range(self.nnz_blocks):
            i, j = rows[k], self.col_ind[k]
            A[i * b:(i + 1) * b, j * b:(j + 1) * b] += self.values[k]
        return A

    def with_values(self, values: np.ndarray) -> "BsrArrays":
        return BsrArrays(self.row_ptr, self.col_ind, values, self.block_size, self.n_block_cols)

    def block_index(self) -> dict:
        rows = np.repeat(np.arange(self.n_block_rows), np.diff(self.row_ptr))
        return {(int(i), int(j)): k for k, (i, j) in enumerate(zip(rows, self.col_ind))}


def csr_from_pairs(n: int, rows: np.ndarray, cols: np.ndarray):
    """Sorted, de-duplicated CSR pattern from (row, col) pairs; returns
    (row_ptr, col_ind, order) with order mapping pattern slots to pairs."""
    key = rows.astype(np.int64) * n + cols.astype(np.int64)
    order = np.argsort(key, kind="stable")
    key_sorted = key[order]
    if key_sorted.size and np.any(np.diff(key_sorted) == 0):
        raise ValueError("duplicate (row, col) pairs")
    r = rows[order]
    row_ptr = np.zeros(n + 1, dtype=np.int32)
    np.add.at(row_ptr, r + 1, 1)
    row_ptr = np.cumsum(row_ptr).astype(np.int32)
    return row_ptr, cols[order].astype(np.int32), order


# ------------------------------------------------------------------ graphene

def graphene(n1: int = 60, n2: int = 60, t: float = -2.7, a_cc: float = 1.42):
    """pz graphene n1 x n2 honeycomb supercell, periodic, nearest-neighbour t,
    onsite 0 (S = I).  Atom 2*(i + n1*j) + s, s = 0 (A) / 1 (B).
    Returns (H BsrArrays with b = 1, positions[n, 3], cell[3, 3])."""
    a = math.sqrt(3.0) * a_cc
    a1 = np.array([a, 0.0, 0.0])
    a2 = np.array([a / 2, a * math.sqrt(3.0) / 2, 0.0])
    delta = (a1 + a2) / 3.0
    n = 2 * n1 * n2
    i, j = np.meshgrid(np.arange(n1), np.arange(n2), indexing="ij")
    i = i.ravel(order="F")
    j = j.ravel(order="F")
    cell_id = i + n1 * j
    A = 2 * cell_id
    B = A + 1
    pos = np.zeros((n, 3))
    pos[A] = i[:, None] * a1 + j[:, None] * a2
    pos[B] = pos[A] + delta

    def bidx(ii, jj):
        return 2 * ((ii % n1) + n1 * (jj % n2)) + 1

    rows = np.concatenate([A, A, A])
    cols = np.concatenate([bidx(i, j), bidx(i - 1, j), bidx(i, j - 1)])
    rows, cols = np.concatenate([rows, cols]), np.concatenate([cols, rows])
    row_ptr, col_ind, _ = csr_from_pairs(n, rows, cols)
    vals = np.full((col_ind.size, 1, 1), t)
    cell = np.array([n1 * a1, n2 * a2, [0.0, 0.0, 20.0]])
    return BsrArrays(row_ptr, col_ind, vals, 1), pos, cell


# ------------------------------------------------------------------- diamond

_DIAMOND_BASIS4 = np.array([[0, 0, 0], [0, 2, 2], [2, 0, 2], [2, 2, 0],
                            [1, 1, 1], [1, 3, 3], [3, 1, 3], [3, 3, 1]])


def diamond_pattern(L: int, max_shell_sq: int = 11):
    """Neighbour pattern of an L^3 conventional-cell diamond supercell to the
    shell with |d|^2 <= max_shell_sq in units of (a/4)^2 (3: 1st, 8: 2nd,
    11: 3rd shell).  Atom 8*(cx + L*(cy + L*cz)) + basis.  Returns
    (row_ptr, col_ind, dist2 per pattern slot, int positions[n, 3])."""
    G = 4 * L
    grid = -np.ones((G, G, G), dtype=np.int64)
    cx, cy, cz = np.meshgrid(np.arange(L), np.arange(L), np.arange(L), indexing="ij")
    cells = np.stack([cx.ravel(order="F"), cy.ravel(order="F"), cz.ravel(order="F")], 1)
    n = 8 * L ** 3
    ipos = (4 * cells[:, None, :] + _DIAMOND_BASIS4[None, :, :]).reshape(n, 3)
    grid[ipos[:, 0], ipos[:, 1], ipos[:, 2]] = np.arange(n)
    r = int(math.isqrt(max_shell_sq))
    d = np.array([(x, y, z) for x in range(-r, r + 1) for y in range(-r, r + 1)
                  for z in range(-r, r + 1) if x * x + y * y + z * z <= max_shell_sq])
    rows, cols, dist2 = [], [], []
    for dv in d:
        q = (ipos + dv) % G
        nb = grid[q[:, 0], q[:, 1], q[:, 2]]
        ok = nb >= 0
        rows.append(np.nonzero(ok)[0])
        cols.append(nb[ok])
        dist2.append(np.full(ok.sum(), int(dv @ dv)))
    rows = np.concatenate(rows)
    cols = np.concatenate(cols)
    dist2 = np.concatenate(dist2)
    row_ptr, col_ind, order = csr_from_pairs(n, rows, cols)
    return row_ptr, col_ind, dist2[order], ipos


def _symmetric_blocks(row_ptr, col_ind, gen_block, b):
    """Values for a symmetric pattern with V[j,i] = V[i,j]^T: blocks are drawn
    for i < j (and i == j) in pattern order, then mirrored."""
    n = row_ptr.size - 1
    rows = np.repeat(np.arange(n), np.diff(row_ptr))
    nnz = col_ind.size
    key = rows.astype(np.int64) * n + col_ind
    tkey = col_ind.astype(np.int64) * n + rows
    mirror = np.searchsorted(key, tkey)
    upper = rows <= col_ind
    vals = np.zeros((nnz, b, b))
    idx_upper = np.nonzero(upper)[0]
    vals[idx_upper] = gen_block(idx_upper, rows[idx_upper], col_ind[idx_upper])
    lower = np.nonzero(~upper)[0]
    vals[lower] = np.transpose(vals[mirror[lower]], (0, 2, 1))
    diag = np.nonzero(rows == col_ind)[0]
    vals[diag] = 0.5 * (vals[diag] + np.transpose(vals[diag], (0, 2, 1)))
    return vals


def diamond_lcao(L: int = 16, seed: int = 7, a: float = 3.567, orbitals: int = 8,
                 s_amplitude: float = 0.15, s_scale: float = 1.0):
    """Non-orthogonal LCAO diamond: H blocks N(0,1)*exp(-r/1.5), S = I on the
    diagonal and U(0, s_amplitude)*s_scale*exp(-r/1.2) off it, both
    symmetric, 8x8 blocks to the 3rd shell (29 blocks per row).  Returns
    (H, S) BsrArrays."""
    row_ptr, col_ind, dist2, _ = diamond_pattern(L, 11)
    r = np.sqrt(dist2) * a / 4.0
    b = orbitals
    rng_h = np.random.default_rng(seed)
    rng_s = np.random.default_rng(seed + 1)

    def gen_h(idx, _r, _c):
        blk = rng_h.standard_normal((idx.size, b, b))
        return blk * np.exp(-r[idx] / 1.5)[:, None, None]

    def gen_s(idx, rr, cc):
        blk = rng_s.uniform(0.0, s_amplitude, (idx.size, b, b)) * s_scale
        blk *= np.exp(-r[idx] / 1.2)[:, None, None]
        blk[rr == cc] = np.eye(b)
        return blk

    H = BsrArrays(row_ptr, col_ind, _symmetric_blocks(row_ptr, col_ind, gen_h, b), b)
    S = BsrArrays(row_ptr, col_ind, _symmetric_blocks(row_ptr, col_ind, gen_s, b), b)
    return H, S


def subgraph_problems(P: BsrArrays):
    """The graph-local problems of graph_inverse_sqrt (isqrtm.hpp:149-232):
    for block row i the dense sub-matrix of P on {i} + neighbours(i).
    Returns (members[n, k] sorted atom lists, slot[n] position of i,
    gather[n, k, k] block index into P.values or -1).  Rows must have equal
    neighbour counts (uniform lattices)."""
    n = P.n_block_rows
    deg = np.diff(P.row_ptr)
    if not np.all(deg == deg[0]):
        raise ValueError("subgraph_problems needs a uniform neighbour count")
    k = int(deg[0])
    members = P.col_ind.reshape(n, k).astype(np.int64)
    slot = np.argmax(members == np.arange(n)[:, None], axis=1)
    rows = np.repeat(np.arange(n), k)
    key = rows.astype(np.int64) * n + P.col_ind
    q = members[:, :, None] * n + members[:, None, :]
    pos = np.searchsorted(key, q)
    pos = np.minimum(pos, key.size - 1)
    gather = np.where(key[pos] == q, pos, -1).astype(np.int64)
    return members, slot, gather
