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
                     rank: int = 0, isqrt_method: str = "ns") -> KpmWorkload:
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


@dataclasses.dataclass
class SpdBatch:
    """A batch of dense SPD problems packed for rsatb_isqrt_columns_batched:
    problem p is the n[p] x n[p] matrix at element offset[p] of `flat`
    (symmetric, so row- and column-major agree)."""
    flat: torch.Tensor
    n: np.ndarray
    offset: np.ndarray
    kappa: np.ndarray
    seed: int

    def matrix(self, p: int) -> np.ndarray:
        n = int(self.n[p])
        o = int(self.offset[p])
        return self.flat[o:o + n * n].reshape(n, n).cpu().numpy()


def batched_spd(n_problems: int = 100_000, n_min: int = 40, n_max: int = 400,
                kappa_min: float = 1e2, kappa_max: float = 1e5, family: str = "continuous",
                seed: int = 7, device="cuda") -> SpdBatch:
    """Seeded batched inverse-sqrt problems: sizes uniform in [n_min, n_max],
    condition numbers log-uniform in [kappa_min, kappa_max], A = Q diag(l) Q^T
    with Q from the QR of a Gaussian matrix and l the reference benchmark's
    spectrum families (rsatb/calc/test/benchmark_isqrt_action.cpp:53-85):
    "continuous" (log-spread over [1/kappa, 1]) or "gapped" (n/20 values in
    [1/kappa, 10/kappa], the rest in [0.2, 2])."""
    rng = np.random.default_rng(seed)
    n = np.sort(rng.integers(n_min, n_max + 1, size=n_problems)).astype(np.int32)
    kappa = np.exp(rng.uniform(np.log(kappa_min), np.log(kappa_max), size=n_problems))
    offset = np.concatenate([[0], np.cumsum(n.astype(np.int64) ** 2)[:-1]]).astype(np.int64)
    flat = torch.empty(int((n.astype(np.int64) ** 2).sum()), dtype=torch.float64, device=device)
    gen = torch.Generator(device=device)
    for size in np.unique(n):
        idx = np.flatnonzero(n == size)
        gen.manual_seed(seed * 1_000_003 + int(size))
        for start in range(0, idx.size, 512):
            part = idx[start:start + 512]
            c = part.size
            G = torch.randn(c, size, size, dtype=torch.float64, device=device, generator=gen)
            Q, _ = torch.linalg.qr(G)
            lk = torch.as_tensor(np.log(kappa[part]), device=device)[:, None]
            t = torch.linspace(0.0, 1.0, int(size), dtype=torch.float64, device=device)[None, :]
            if family == "continuous":
                lam = torch.exp(-lk + t * lk)
            else:
                u = torch.rand(c, int(size), dtype=torch.float64, device=device, generator=gen)
                n_low = max(1, int(size) // 20)
                lam = 0.2 + 1.8 * u
                lam[:, :n_low] = torch.exp(-lk) * torch.exp(u[:, :n_low] * np.log(10.0))
            A = (Q * lam[:, None, :]) @ Q.transpose(1, 2)
            A = 0.5 * (A + A.transpose(1, 2))
            o = int(offset[part[0]])  # equal sizes are contiguous (n is sorted)
            flat[o:o + c * int(size) ** 2] = A.reshape(-1)
    return SpdBatch(flat, n, offset, kappa, seed)
