"""Test helpers: the same operator, built for the GPU library and the oracle."""
from __future__ import annotations

import numpy as np

import oracle
from rsatb_b200.lattice import BsrArrays


def random_hermitian_bsr(n_blocks: int, b: int, degree: int, seed: int, complex_values: bool,
                         scale: float = 1.0) -> BsrArrays:
    """A Hermitian BSR with ~degree random off-diagonal blocks per row."""
    rng = np.random.default_rng(seed)
    pairs = set()
    for i in range(n_blocks):
        pairs.add((i, i))
        for j in rng.choice(n_blocks, size=min(degree, n_blocks), replace=False):
            pairs.add((i, int(j)))
            pairs.add((int(j), i))
    pairs = sorted(pairs)
    rows = np.array([p[0] for p in pairs])
    cols = np.array([p[1] for p in pairs])
    row_ptr = np.zeros(n_blocks + 1, dtype=np.int32)
    np.add.at(row_ptr, rows + 1, 1)
    row_ptr = np.cumsum(row_ptr).astype(np.int32)
    index = {p: k for k, p in enumerate(pairs)}
    dt = np.complex128 if complex_values else np.float64
    vals = np.zeros((len(pairs), b, b), dtype=dt)
    for k, (i, j) in enumerate(pairs):
        if i > j:
            continue
        blk = rng.standard_normal((b, b))
        if complex_values:
            blk = blk + 1j * rng.standard_normal((b, b))
        blk *= scale
        if i == j:
            blk = 0.5 * (blk + blk.conj().T)
            vals[k] = blk
        else:
            vals[k] = blk
            vals[index[(j, i)]] = blk.conj().T
    return BsrArrays(row_ptr, cols.astype(np.int32), vals, b)


def to_oracle(A: BsrArrays, imag: bool = False) -> oracle.Bsr:
    nbc = A.n_block_cols or A.n_block_rows
    return oracle.Bsr(A.n_block_rows, nbc, A.block_size, A.row_ptr, A.col_ind, A.values, imag=imag)


def adjoint_arrays(A: BsrArrays) -> BsrArrays:
    """A^H on the host (for the oracle's sandwich)."""
    n = A.n_block_rows
    nbc = A.n_block_cols or n
    rows = np.repeat(np.arange(n), np.diff(A.row_ptr))
    cols = A.col_ind
    order = np.lexsort((rows, cols))
    t_rows = cols[order]
    row_ptr = np.zeros(nbc + 1, dtype=np.int32)
    np.add.at(row_ptr, t_rows + 1, 1)
    row_ptr = np.cumsum(row_ptr).astype(np.int32)
    vals = np.conj(np.transpose(A.values[order], (0, 2, 1)))
    return BsrArrays(row_ptr, rows[order].astype(np.int32), np.ascontiguousarray(vals),
                     A.block_size, n)


def rel_err(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
