"""Graph-local inverse square root S^-1/2 (the seed of rsatb's inverse_sqrt).

``graph_inverse_sqrt`` follows rsatb::calc::graph_inverse_sqrt
(rsatb/calc/isqrtm.hpp:149-232): for every block row i, the dense overlap
sub-matrix M_i on {i} + neighbours(i) is formed, its inverse square root is
taken, and block row i of M_i^{-1/2} becomes block row i of Z (Z keeps S's
pattern).  The per-problem action is selected by ``method``:

* ``"eigen"``  -- the clamped eigendecomposition route of
  isqrt::eigen_action (rsatb/calc/isqrt_action.hpp:766-795), x -> x^-1/2 for
  x > 1e-12 else 0, which the reference takes for every n <= 256;
* ``"ns"``     -- the batched Newton-Schulz kernels of the rsatb_b200
  library (``rsatb_b200.ns``), when built.

The problems are gathered and solved on the GPU in chunks.
"""
from __future__ import annotations

import numpy as np
import torch

from .lattice import BsrArrays, subgraph_problems

EIGEN_CLAMP = 1.0e-12  # isqrt::Options::eigen_clamp (isqrt_action.hpp:126)


def _gather_dense(vals: torch.Tensor, gather: torch.Tensor, b: int) -> torch.Tensor:
    """(P, k, k) block indices -> (P, k*b, k*b) dense matrices."""
    P, k, _ = gather.shape
    g = gather.clamp(min=0)
    blocks = vals[g.reshape(-1)].reshape(P, k, k, b, b)
    blocks = blocks * (gather >= 0).reshape(P, k, k, 1, 1).to(vals.dtype)
    return blocks.permute(0, 1, 3, 2, 4).reshape(P, k * b, k * b)


def clamped_inverse_sqrt_rows(M: torch.Tensor, rows: torch.Tensor, b: int) -> torch.Tensor:
    """Block row `rows` (per problem) of the clamped M^{-1/2} (eigen route)."""
    w, V = torch.linalg.eigh(M)
    f = torch.where(w > EIGEN_CLAMP, w.clamp(min=EIGEN_CLAMP).rsqrt(), torch.zeros_like(w))
    P, n, _ = M.shape
    idx = rows[:, None] * b + torch.arange(b, device=M.device)[None, :]
    Vr = torch.gather(V, 1, idx[:, :, None].expand(P, b, n))  # (P, b, n)
    return (Vr * f[:, None, :]) @ V.transpose(1, 2)           # (P, b, n)


def newton_schulz_rows_fp64(M: torch.Tensor, rows: torch.Tensor, b: int, max_iter: int = 40,
                            tol: float = 1e-14) -> torch.Tensor:
    """Block row `rows` of M^{-1/2} by the coupled Newton-Schulz iteration
    Y <- Y T, Z <- T Z, T = (3I - Z Y)/2 from Y0 = M/s, Z0 = I (Higham,
    Functions of Matrices, 2008, eq. 6.35), s a Gershgorin bound of
    lambda_max, in FP64 batched GEMMs."""
    P, n, _ = M.shape
    s = M.abs().sum(-1).amax(-1)                        # >= lambda_max
    Y = M / s[:, None, None]
    I = torch.eye(n, dtype=M.dtype, device=M.device).expand(P, n, n)
    Z = I.clone()
    for _ in range(max_iter):
        T = 1.5 * I - 0.5 * (Z @ Y)
        Y = Y @ T
        Z = T @ Z
        err = (T - I).abs().amax().item()
        if err < tol:
            break
    idx = rows[:, None] * b + torch.arange(b, device=M.device)[None, :]
    Zr = torch.gather(Z, 1, idx[:, :, None].expand(P, b, n))
    return Zr / s.sqrt()[:, None, None]


def graph_inverse_sqrt(S: BsrArrays, method: str = "eigen", device="cuda",
                       chunk: int = 2048) -> BsrArrays:
    """Z with S's pattern, block row i = row block of (S restricted to the
    neighbourhood of i)^{-1/2}."""
    members, slot, gather = subgraph_problems(S)
    n, k = members.shape
    b = S.block_size
    vals = torch.as_tensor(np.ascontiguousarray(S.values), dtype=torch.float64, device=device)
    out = torch.empty((n, k, b, b), dtype=torch.float64, device=device)
    g_all = torch.as_tensor(gather, device=device)
    s_all = torch.as_tensor(slot, device=device)
    for start in range(0, n, chunk):
        stop = min(n, start + chunk)
        M = _gather_dense(vals, g_all[start:stop], b)
        if method == "eigen":
            X = clamped_inverse_sqrt_rows(M, s_all[start:stop], b)
        elif method == "ns_fp64":
            X = newton_schulz_rows_fp64(M, s_all[start:stop], b)
        elif method == "ns":
            from . import ns
            X = ns.inverse_sqrt_rows(M, s_all[start:stop], b)
        else:
            raise ValueError(f"unknown isqrt method {method!r}")
        # (P, b, k*b) -> (P, k, b, b): block j of row i
        out[start:stop] = X.reshape(stop - start, b, k, b).permute(0, 2, 1, 3)
        del M, X
    # members[i] is sorted and equals S's column list of row i, so the blocks
    # land in S's pattern order.
    zvals = out.reshape(n * k, b, b).cpu().numpy()
    return BsrArrays(S.row_ptr, S.col_ind, zvals, b)


def graph_inverse_sqrt_host(S: BsrArrays) -> BsrArrays:
    """numpy version of the eigen route (small systems, tests)."""
    members, slot, gather = subgraph_problems(S)
    n, k = members.shape
    b = S.block_size
    zvals = np.zeros((n * k, b, b))
    for i in range(n):
        g = gather[i]
        M = np.zeros((k * b, k * b))
        for p in range(k):
            for q in range(k):
                if g[p, q] >= 0:
                    M[p * b:(p + 1) * b, q * b:(q + 1) * b] = S.values[g[p, q]]
        w, V = np.linalg.eigh(M)
        f = np.where(w > EIGEN_CLAMP, 1.0 / np.sqrt(np.maximum(w, EIGEN_CLAMP)), 0.0)
        X = (V[slot[i] * b:(slot[i] + 1) * b] * f) @ V.T
        zvals[i * k:(i + 1) * k] = X.reshape(b, k, b).transpose(1, 0, 2)
    return BsrArrays(S.row_ptr, S.col_ind, zvals, b)
