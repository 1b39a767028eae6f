"""Inverse square root S^-1/2 of a sparse overlap: rsatb's inverse_sqrt.

``graph_inverse_sqrt`` follows rsatb::calc::graph_inverse_sqrt
(rsatb/calc/isqrtm.hpp:149-232): for every block row i, the dense overlap
sub-matrix M_i on {i} + neighbours(i) is formed, its inverse square root is
taken, and block row i of M_i^{-1/2} becomes block row i of Z (Z keeps S's
pattern).  The per-problem action is selected by ``method``:

* ``"eigen"``  -- the clamped eigendecomposition route of
  isqrt::eigen_action (rsatb/calc/isqrt_action.hpp:766-795), x -> x^-1/2 for
  x > 1e-12 else 0, which the reference takes for every n <= 256;
* ``"ns"``, ``"ns_tf32x3"``, ``"ns_tf32"`` -- the batched Newton-Schulz
  solve of the rsatb_b200 library (``inverse_sqrt_columns_batched``): FP64
  throughout, or a tcgen05 tensor-core phase (split or plain TF32) finished
  by FP64 iterations.

The problems are gathered and solved on the GPU in chunks.

``inverse_sqrt`` is rsatb::calc::inverse_sqrt (rsatb/calc/isqrtm.hpp:262):
that seed refined by the global sparse Newton-Schulz purification, every
product a block SpGEMM on the device (``rsatb_inverse_sqrt_refine``).
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np
import torch

from . import _capi
from ._capi import check, lib
from .lattice import BsrArrays, subgraph_problems
from .vbcsr import context

EIGEN_CLAMP = 1.0e-12  # isqrt::Options::eigen_clamp (isqrt_action.hpp:126)

NS_METHODS = {"ns": "fp64", "ns_tf32x3": "tf32x3", "ns_tf32": "tf32"}
PRECISIONS = {"fp64": _capi.NS_FP64, "tf32x3": _capi.NS_TF32X3, "tf32": _capi.NS_TF32}


def inverse_sqrt_columns_batched(M: torch.Tensor, n, in_offset, col_start=None, k_cols=None,
                                 out_offset=None, precision: str = "tf32x3",
                                 max_iter: int = 0, max_fp64_iter: int = 0, tol: float = 0.0,
                                 accept: float = 0.0, workspace_bytes: int = 0,
                                 graph: bool = True, out: torch.Tensor | None = None,
                                 tiles: "TileTable | None" = None):
    """Columns [col_start, col_start + k) of M_p^{-1/2} for every problem p
    (isqrt::inverse_sqrt_columns_inplace, rsatb/calc/isqrt_action.hpp:1343,
    for a batch), by the library's batched Newton-Schulz solve.

    M: 1-D float64 CUDA tensor holding the matrices, problem p's n_p x n_p
    column-major matrix at element in_offset[p] (upper triangle read).
    Returns (out, status, stats): out a 1-D float64 CUDA tensor with problem
    p's n_p x k_p column-major block at out_offset[p] (packed in problem
    order when out_offset is None), status one rsatb_status per problem,
    stats a dict of the call's counters.  tiles: the tensor-core kernel and
    N tiles picked by autotune_tiles (None: the built-in choice).
    """
    if not (M.is_cuda and M.dtype == torch.float64 and M.dim() == 1 and M.is_contiguous()):
        raise ValueError("M must be a contiguous 1-D float64 CUDA tensor")
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
    n = np.ascontiguousarray(np.asarray(n, dtype=np.int32))
    P = n.size
    in_offset = np.ascontiguousarray(np.asarray(in_offset, dtype=np.int64))
    col_start = np.zeros(P, np.int32) if col_start is None else np.ascontiguousarray(
        np.asarray(col_start, dtype=np.int32))
    k = n.copy() if k_cols is None else np.ascontiguousarray(np.asarray(k_cols, dtype=np.int32))
    k = np.where(k > 0, k, n).astype(np.int32)
    if out_offset is None:
        sizes = n.astype(np.int64) * k
        out_offset = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
        total = int(sizes.sum())
    else:
        out_offset = np.ascontiguousarray(np.asarray(out_offset, dtype=np.int64))
        total = int((out_offset + n.astype(np.int64) * k).max()) if P else 0
    if out is None:
        out = torch.zeros(max(total, 1), dtype=torch.float64, device=M.device)
    opt = _capi.IsqrtOptions(PRECISIONS[precision], max_iter, max_fp64_iter, tol, accept,
                             workspace_bytes, 0 if graph else 1)
    if tiles is not None:
        t_np = np.ascontiguousarray(np.asarray(list(tiles.nt.keys()), dtype=np.int32))
        t_nt = np.ascontiguousarray(np.asarray(list(tiles.nt.values()), dtype=np.int32))
        opt.tc_kernel = tiles.tc_kernel
        opt.n_tiles = int(t_np.size)
        opt.tile_n_pad = t_np.ctypes.data
        opt.tile_nt = t_nt.ctypes.data
    stats = _capi.IsqrtStats()
    status = np.zeros(P, dtype=np.int32)
    ctx = context(M.device.index)
    ctx.bind_stream()
    vp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    check(lib().rsatb_isqrt_columns_batched(
        ctx.handle, P, vp(n), vp(col_start), vp(k), vp(in_offset), C.c_void_p(M.data_ptr()),
        vp(out_offset), C.c_void_p(out.data_ptr()), C.byref(opt), vp(status),
        C.byref(stats)))
    return out, status, {f: getattr(stats, f) for f, _ in stats._fields_}


class TileTable:
    """Tensor-core kernel (1 warp-specialised, 2 single-role) and N tile per
    padded size for inverse_sqrt_columns_batched, as autotune_tiles picks
    them; ms holds every candidate's measured time per size."""

    def __init__(self, tc_kernel: int, nt: dict, ms: dict | None = None):
        self.tc_kernel = int(tc_kernel)
        self.nt = {int(k): int(v) for k, v in nt.items()}
        self.ms = ms or {}

    def __repr__(self):
        kind = "warp-specialised" if self.tc_kernel == 1 else "single-role"
        return f"TileTable({kind}, nt={self.nt})"


def autotune_tiles(sizes, precision: str = "tf32x3", problems_per_size: int = 16,
                   device: int | None = None) -> TileTable:
    """Times the tensor-core kernel and N-tile candidates of the batched solve
    on seeded well-conditioned SPD samples of each size (a fixed-length
    solve, device time from CUDA events) and returns the fastest choice."""
    if PRECISIONS.get(precision) not in (_capi.NS_TF32X3, _capi.NS_TF32):
        raise ValueError("autotuning needs a tensor-core precision ('tf32x3' or 'tf32')")
    pads = sorted({(int(s) + 31) // 32 * 32 for s in np.asarray(sizes).ravel()})
    sz = np.ascontiguousarray(np.asarray(pads, dtype=np.int32))
    nt = np.zeros(sz.size, dtype=np.int32)
    ms = np.zeros(sz.size * 8, dtype=np.float64)
    kern = C.c_int(0)
    ctx = context(device if device is not None else torch.cuda.current_device())
    ctx.bind_stream()
    check(lib().rsatb_isqrt_autotune(ctx.handle, PRECISIONS[precision], int(sz.size),
                                     sz.ctypes.data_as(C.c_void_p), int(problems_per_size),
                                     C.byref(kern), nt.ctypes.data_as(C.c_void_p),
                                     ms.ctypes.data_as(C.c_void_p)))
    table = {int(p): int(t) for p, t in zip(sz, nt)}
    times = {int(p): ms[8 * i:8 * i + 8].reshape(2, 4).tolist() for i, p in enumerate(sz)}
    return TileTable(kern.value, table, times)


def inverse_sqrt_rows_batched(M: torch.Tensor, rows: torch.Tensor, b: int,
                              precision: str = "tf32x3") -> torch.Tensor:
    """Block row `rows[p]` of M[p]^{-1/2} for a (P, n, n) batch of symmetric
    matrices, through inverse_sqrt_columns_batched (the columns of a
    symmetric matrix are its rows)."""
    P, n, _ = M.shape
    flat = M.contiguous().reshape(-1)
    offs = np.arange(P, dtype=np.int64) * n * n
    cs = (rows.to("cpu").numpy().astype(np.int64) * b).astype(np.int32)
    out, status, _ = inverse_sqrt_columns_batched(flat, np.full(P, n, np.int32), offs, cs,
                                                  np.full(P, b, np.int32), precision=precision)
    bad = np.flatnonzero(status != 0)
    if bad.size:
        raise _capi.RsatbError(int(status[bad[0]]),
                               f"{bad.size} of {P} subgraph problems failed (first: {bad[0]})")
    return out[:P * n * b].reshape(P, b, n)


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
        elif method in NS_METHODS:
            X = inverse_sqrt_rows_batched(M, s_all[start:stop], b, NS_METHODS[method])
        else:
            raise ValueError(f"unknown isqrt method {method!r}")
        # (P, b, k*b) -> (P, k, b, b): block j of row i
        out[start:stop] = X.reshape(stop - start, b, k, b).permute(0, 2, 1, 3)
        del M, X
    # members[i] is sorted and equals S's column list of row i, so the blocks
    # land in S's pattern order.
    zvals = out.reshape(n * k, b, b).cpu().numpy()
    return BsrArrays(S.row_ptr, S.col_ind, zvals, b)


def _seed_ragged(S: BsrArrays, device="cuda") -> BsrArrays:
    """graph_inverse_sqrt for patterns whose rows have different neighbour
    counts (chains with ends, unstructured graphs): the rows are grouped by
    neighbour count and each group takes the clamped eigen route."""
    n, b = S.n_block_rows, S.block_size
    rp = np.asarray(S.row_ptr, dtype=np.int64)
    ci = np.asarray(S.col_ind, dtype=np.int64)
    deg = np.diff(rp)
    key = np.repeat(np.arange(n), deg) * n + ci
    vals = torch.as_tensor(np.ascontiguousarray(S.values), dtype=torch.float64, device=device)
    zvals = np.zeros((ci.size, b, b))
    for k in np.unique(deg):
        rows = np.flatnonzero(deg == k)
        members = ci[rp[rows][:, None] + np.arange(k)[None, :]]
        slot = np.argmax(members == rows[:, None], axis=1)
        q = members[:, :, None] * n + members[:, None, :]
        pos = np.minimum(np.searchsorted(key, q), key.size - 1)
        gather = torch.as_tensor(np.where(key[pos] == q, pos, -1), device=device)
        M = _gather_dense(vals, gather, b)
        X = clamped_inverse_sqrt_rows(M, torch.as_tensor(slot, device=device), b)
        blocks = X.reshape(rows.size, b, int(k), b).permute(0, 2, 1, 3).cpu().numpy()
        for r, i in enumerate(rows):
            zvals[rp[i]:rp[i] + k] = blocks[r]
    return BsrArrays(S.row_ptr, S.col_ind, zvals, b)


@dataclasses.dataclass
class InverseSqrtOptions:
    """rsatb::calc::InverseSqrtOptions (rsatb/calc/isqrtm.hpp:235-240), and
    the route rule of the X update (0: propagate P X P when its first product
    is smaller, every fifth step and residuals >= 0.1 reform; 1: always
    reform)."""
    tol: float = 1e-7
    sptol: float = 1e-6
    maxit: int = 20
    route: int = 0


@dataclasses.dataclass
class InverseSqrtReport:
    """rsatb::calc::InverseSqrtReport (rsatb/calc/isqrtm.hpp:243-258)."""
    steps: int
    converged: bool
    hit_maxiter: bool
    diverged: bool
    last_advance_propagated: bool
    residual: float
    applied_residual: float
    nnz_blocks: int
    reforms: int
    propagations: int


def inverse_sqrt(S, options: InverseSqrtOptions | None = None, seed=None):
    """S^-1/2 of the FP64 BSR overlap S (BsrArrays): the graph-local seed
    (``graph_inverse_sqrt``, or ``seed`` if given) refined on the device by
    the sparse Newton-Schulz purification of inverse_sqrt
    (rsatb/calc/isqrtm.hpp:262-900).  Returns (Z as a device BlockSpMat, its
    pattern grown by the products; InverseSqrtReport)."""
    from .vbcsr import BlockSpMat
    opt = options or InverseSqrtOptions()
    if seed is None:
        deg = np.diff(np.asarray(S.row_ptr))
        seed = graph_inverse_sqrt(S) if np.all(deg == deg[0]) else _seed_ragged(S)
    Sd = BlockSpMat(S.row_ptr, S.col_ind, S.values, S.block_size, dtype=np.float64)
    Zd = BlockSpMat(seed.row_ptr, seed.col_ind, seed.values, seed.block_size, dtype=np.float64)
    copt = _capi.NsRefineOptions(float(opt.tol), float(opt.sptol), int(opt.maxit),
                                 int(opt.route))
    rep = _capi.NsRefineReport()
    h = C.c_void_p()
    ctx = Sd.ctx
    ctx.bind_stream()
    check(lib().rsatb_inverse_sqrt_refine(ctx.handle, Sd.handle, Zd.handle, C.byref(copt),
                                          C.byref(h), C.byref(rep)))
    Z = BlockSpMat(None, None, None, 0, device=ctx.device, _handle=h)
    report = InverseSqrtReport(rep.steps, bool(rep.converged), bool(rep.hit_maxiter),
                               bool(rep.diverged), bool(rep.last_advance_propagated),
                               rep.residual, rep.applied_residual, rep.nnz_blocks, rep.reforms,
                               rep.propagations)
    return Z, report


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
