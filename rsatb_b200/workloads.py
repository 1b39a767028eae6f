"""Benchmark workloads: seeded operators, factors, bounds and sample vectors.

``diamond_sandwich`` is the non-orthogonal LCAO diamond DOS run: 16^3
conventional cells (32,768 atoms x 8 orbitals, N = 262,144), 8x8 BSR blocks
to the 3rd neighbour shell (29 per row), H ~ N(0,1) exp(-r/1.5),
S = I + U(0,0.15) exp(-r/1.2), the operator Z^H H Z with Z the graph-local
S^-1/2, 128 Rademacher vectors and 1024 moments.  ``graphene_dos`` is the
orthogonal pz graphene DOS run (60x60 cells, R = 8 random phases, 512
moments).
"""
from __future__ import annotations

import dataclasses
import time

import numpy as np
import torch

from . import lattice
from .bounds import estimate_spectral_bounds
from .calc import Chebyshev, ISQRTMPreconditioner
from .isqrt import graph_inverse_sqrt
from .vbcsr import BlockSpMat, set_random

SAMPLE_SEED = 20240917  # SetupOptions::sample_seed default (model/setup.hpp:72)


@dataclasses.dataclass
class KpmWorkload:
    name: str
    H: lattice.BsrArrays
    Z: lattice.BsrArrays | None
    cheby64: Chebyshev
    cheby32: Chebyshev
    emin: float
    emax: float
    n_moments: int
    R: int
    orbitals: int
    first_column: int
    complex_vectors: bool
    setup_seconds: dict

    @property
    def n_rows(self) -> int:
        return self.H.n_rows

    def psi(self, dtype) -> torch.Tensor:
        t = torch.empty(self.n_rows, self.R, dtype=dtype, device="cuda")
        kind = 0 if self.complex_vectors else 1
        set_random(t, SAMPLE_SEED, normalize=True, orbitals_per_atom=self.orbitals, kind=kind,
                   first_column=self.first_column)
        return t

    def vec_dtype(self, precision: str) -> torch.dtype:
        if self.complex_vectors:
            return torch.complex128 if precision == "f64" else torch.complex64
        return torch.float64 if precision == "f64" else torch.float32


def _dev(A: lattice.BsrArrays, imaginary: bool = False) -> BlockSpMat:
    return BlockSpMat(A.row_ptr, A.col_ind, A.values, A.block_size, A.n_block_cols,
                      imaginary=imaginary)


def diamond_sandwich(L: int = 16, R: int = 128, n_moments: int = 1024, seed: int = 7,
                     rank: int = 0, isqrt_method: str = "ns_fp64") -> KpmWorkload:
    t = {}
    t0 = time.perf_counter()
    H, S = lattice.diamond_lcao(L=L, seed=seed)
    t["generate"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    Z = graph_inverse_sqrt(S, method=isqrt_method)
    torch.cuda.synchronize()
    t["graph_inverse_sqrt"] = time.perf_counter() - t0
    del S
    t0 = time.perf_counter()
    pre = ISQRTMPreconditioner(_dev(Z))
    c = Chebyshev(_dev(H), -1.0, 1.0, preconditioner=pre)
    emin, emax = estimate_spectral_bounds(c)
    c64 = Chebyshev(c.H, emin, emax, preconditioner=pre)
    c32 = c64.astype("f32")
    torch.cuda.synchronize()
    t["upload_bounds"] = time.perf_counter() - t0
    return KpmWorkload("diamond_sandwich", H, Z, c64, c32, emin, emax, n_moments, R, 8,
                       rank * R, False, t)


def graphene_dos(n1: int = 60, n2: int = 60, R: int = 8, n_moments: int = 512,
                 rank: int = 0) -> KpmWorkload:
    t = {}
    t0 = time.perf_counter()
    H, _, _ = lattice.graphene(n1, n2)
    c = Chebyshev(_dev(H), -1.0, 1.0)
    emin, emax = estimate_spectral_bounds(c)
    c64 = Chebyshev(c.H, emin, emax)
    c32 = c64.astype("f32")
    torch.cuda.synchronize()
    t["setup"] = time.perf_counter() - t0
    return KpmWorkload("graphene_dos", H, None, c64, c32, emin, emax, n_moments, R, 1,
                       rank * R, True, t)


def spmm_bytes(A: BlockSpMat, n_vectors: int, vec_itemsize: int) -> int:
    """Algorithmic HBM bytes of one Y = A X: values + indices once, X read
    once, Y written once."""
    n_rows, n_cols = A.shape
    return A.value_bytes() + A.index_bytes() + (n_rows + n_cols) * n_vectors * vec_itemsize


def spmm_flops(A: BlockSpMat, n_vectors: int, complex_vectors: bool) -> float:
    """Real FLOPs of one Y = A X (2 per multiply-add; a complex matrix times
    a complex panel is 4 real multiply-adds per entry)."""
    per = 2.0 * A.nnz_blocks * A.block_size ** 2 * n_vectors
    if A.is_complex:
        per *= 4.0
    elif complex_vectors:
        per *= 2.0
    return per
