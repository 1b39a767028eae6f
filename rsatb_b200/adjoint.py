"""Differentiable KPM density of states on the GPU.

``kpm_moments_vjp`` calls the library's adjoint Chebyshev recurrence
(rsatb_kpm_moments_vjp): the gradient of sum_n dmu_n mu_n with respect to
every stored block value of H, t_n recomputed from sqrt(N) checkpoints.
``KpmDosLoss`` wraps forward (plain moments -> Jackson-smoothed DOS -> L2
loss against a target DOS) and backward (dL/dmu on the host, then the
device VJP) in a ``torch.autograd.Function`` whose input is the tensor of
H's block values.  The reference has no differentiation code; the forward
quantities follow Chebyshev::compute_moments (rsatb/calc/cheby.hpp:479-514),
evaluate_kpm_density (rsatb/calc/kpm.hpp:206-241) and ComputeDos's factor 2
(rsatb/calc/observables.hpp:389-441).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _capi
from ._capi import check, lib
from .calc import Chebyshev, KpmKernel, kpm_dos_moments_plain, kpm_kernel_weights
from .vbcsr import BlockSpMat, dtype_code


def kpm_moments_vjp(cheby: Chebyshev, psi: torch.Tensor, n_moments: int, dmu,
                    checkpoint_stride: int = 0):
    """(grad[nnz, b, b] float64 CUDA tensor, mu[n_moments], stats)."""
    if cheby.M is not None:
        raise NotImplementedError("the adjoint runs for the Orthogonal form only")
    if not psi.is_cuda or psi.dim() != 2 or not psi.is_contiguous() or psi.is_complex():
        raise ValueError("psi must be a contiguous real (N, R) CUDA tensor")
    H = cheby.H
    dmu = np.ascontiguousarray(np.asarray(dmu, dtype=np.float64))
    if dmu.size != n_moments:
        raise ValueError("dmu needs n_moments entries")
    b = H.block_size
    grad = torch.empty((H.nnz_blocks, b, b), dtype=torch.float64, device=psi.device)
    mu = np.zeros(n_moments)
    stats = _capi.AdjointStats()
    ctx = H.ctx
    ctx.bind_stream()
    op = cheby.c_op()
    P = C.POINTER(C.c_double)
    check(lib().rsatb_kpm_moments_vjp(
        ctx.handle, C.byref(op), C.c_void_p(psi.data_ptr()), psi.shape[1],
        dtype_code(psi.dtype), int(n_moments), dmu.ctypes.data_as(P), int(checkpoint_stride),
        mu.ctypes.data_as(P), C.c_void_p(grad.data_ptr()), C.byref(stats)))
    return grad, mu, {f: getattr(stats, f) for f, _ in stats._fields_}


def dos_basis(n_moments: int, x: np.ndarray, kernel: KpmKernel = KpmKernel.Jackson) -> np.ndarray:
    """D[j, n] with rho(x_j) = sum_n D[j, n] mu_n: ComputeDos's 2 * (g_0 mu_0 +
    2 sum g_n mu_n T_n(x)) / (pi sqrt(1 - x^2))."""
    g = kpm_kernel_weights(kernel, n_moments)
    n = np.arange(n_moments)
    T = np.cos(np.outer(np.arccos(x), n))
    w = np.where(n == 0, 1.0, 2.0) * g
    return 2.0 * T * w[None, :] / (math.pi * np.sqrt(1.0 - x * x))[:, None]


class KpmDosLoss(torch.autograd.Function):
    """L(values) = sum_j (rho_j(values) - target_j)^2 for the Jackson DOS of
    H(values) on the grid x (bounds held fixed), rho from the plain moments of
    the real sample panel psi.  ``values``: (nnz, b, b) float64 CUDA tensor of
    H's block values in H's pattern order."""

    @staticmethod
    def forward(ctx, values, H: BlockSpMat, psi, emin, emax, n_moments, x, target,
                checkpoint_stride=0):
        H.set_values(values)
        cheby = Chebyshev(H, emin, emax)
        mu = kpm_dos_moments_plain(cheby, psi, n_moments).real
        D = dos_basis(n_moments, np.asarray(x, dtype=np.float64))
        rho = D @ mu
        resid = rho - np.asarray(target, dtype=np.float64)
        ctx.saved = (H, psi, emin, emax, n_moments, D, resid, checkpoint_stride)
        return torch.tensor(float(resid @ resid), dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        H, psi, emin, emax, n_moments, D, resid, stride = ctx.saved
        dmu = float(grad_out) * 2.0 * (resid @ D)
        grad, _, _ = kpm_moments_vjp(Chebyshev(H, emin, emax), psi, n_moments, dmu, stride)
        return (grad,) + (None,) * 8


def kpm_moments_vjp_sandwich(cheby: Chebyshev, psi: torch.Tensor, n_moments: int, dmu,
                             checkpoint_stride: int = 0):
    """Sandwich form A = (Z^T H Z - c) / hw: (grad_h[nnz_H, b, b],
    grad_z[nnz_Z, b, b] float64 CUDA tensors, mu[n_moments], stats) from
    rsatb_kpm_moments_vjp_sandwich."""
    if cheby.M is None:
        raise ValueError("kpm_moments_vjp_sandwich needs the sandwich form (a preconditioner)")
    if not psi.is_cuda or psi.dim() != 2 or not psi.is_contiguous() or psi.is_complex():
        raise ValueError("psi must be a contiguous real (N, R) CUDA tensor")
    H, Z = cheby.H, cheby.M.Z
    dmu = np.ascontiguousarray(np.asarray(dmu, dtype=np.float64))
    if dmu.size != n_moments:
        raise ValueError("dmu needs n_moments entries")
    b = H.block_size
    gh = torch.empty((H.nnz_blocks, b, b), dtype=torch.float64, device=psi.device)
    gz = torch.empty((Z.nnz_blocks, b, b), dtype=torch.float64, device=psi.device)
    mu = np.zeros(n_moments)
    stats = _capi.AdjointStats()
    ctx = H.ctx
    ctx.bind_stream()
    op = cheby.c_op()
    P = C.POINTER(C.c_double)
    check(lib().rsatb_kpm_moments_vjp_sandwich(
        ctx.handle, C.byref(op), C.c_void_p(psi.data_ptr()), psi.shape[1],
        dtype_code(psi.dtype), int(n_moments), dmu.ctypes.data_as(P), int(checkpoint_stride),
        mu.ctypes.data_as(P), C.c_void_p(gh.data_ptr()), C.c_void_p(gz.data_ptr()),
        C.byref(stats)))
    return gh, gz, mu, {f: getattr(stats, f) for f, _ in stats._fields_}


def grad_s_from_grad_z(S, grad_z: torch.Tensor) -> torch.Tensor:
    """dL/dS on S's stored blocks from dL/dZ, for Z the graph-local factor of
    S by the clamped eigen route (rsatb/calc/isqrtm.hpp:149-232,
    isqrt_action.hpp:766-795; Z keeps S's pattern).  Block row i of Z is
    block row i of f(M_i), M_i = S on {i} + neighbours(i), f(x) = x^-1/2 for
    x > 1e-12 else 0.  The adjoint of the Frechet derivative of f at
    M = U diag(w) U^T is E -> U (F o (U^T E U)) U^T with F_kl the divided
    differences of f, here -1 / (sqrt(w_k) sqrt(w_l) (sqrt(w_k) + sqrt(w_l))),
    which has no cancellation and equals f'(w) on the diagonal.  Its
    symmetric part is the gradient under perturbations that keep S
    symmetric, split over the two stored copies of each off-diagonal block
    (perturbing blocks (p, q) and (q, p) = (p, q)^T together changes L by
    <grad_pq + grad_qp^T, delta>).  Runs on the device (batched eigh per
    neighbour count)."""
    from .isqrt import EIGEN_CLAMP, _gather_dense
    dev = grad_z.device
    n, b = S.n_block_rows, S.block_size
    rp = np.asarray(S.row_ptr, dtype=np.int64)
    ci = np.asarray(S.col_ind, dtype=np.int64)
    deg = np.diff(rp)
    key = np.repeat(np.arange(n), deg) * n + ci
    vals = torch.as_tensor(np.ascontiguousarray(S.values), dtype=torch.float64, device=dev)
    gs = torch.zeros_like(vals)
    for k in np.unique(deg):
        k = int(k)
        rows = np.flatnonzero(deg == k)
        members = ci[rp[rows][:, None] + np.arange(k)[None, :]]
        slot = np.argmax(members == rows[:, None], axis=1)
        q = members[:, :, None] * n + members[:, None, :]
        pos = np.minimum(np.searchsorted(key, q), key.size - 1)
        gather = torch.as_tensor(np.where(key[pos] == q, pos, -1), device=dev)
        M = _gather_dense(vals, gather, b)
        w, U = torch.linalg.eigh(M)
        live = w > EIGEN_CLAMP
        sw = torch.where(live, w.clamp(min=EIGEN_CLAMP).sqrt(), torch.ones_like(w))
        F = -1.0 / (sw[:, :, None] * sw[:, None, :] * (sw[:, :, None] + sw[:, None, :]))
        f = torch.where(live, 1.0 / sw, torch.zeros_like(w))
        both = live[:, :, None] & live[:, None, :]
        dw = w[:, :, None] - w[:, None, :]
        df = f[:, :, None] - f[:, None, :]
        one = live[:, :, None] ^ live[:, None, :]  # one side clamped to 0
        F = torch.where(both, F, torch.where(one, df / torch.where(dw == 0, torch.ones_like(dw),
                                                                     dw), torch.zeros_like(F)))
        P_ = rows.size
        gz_rows = grad_z[torch.as_tensor(rp[rows][:, None] + np.arange(k)[None, :], device=dev)]
        E = torch.zeros_like(M)
        ridx = torch.as_tensor(slot[:, None] * b + np.arange(b)[None, :], device=dev)  # (P, b)
        E.scatter_(1, ridx[:, :, None].expand(P_, b, k * b),
                   gz_rows.permute(0, 2, 1, 3).reshape(P_, b, k * b))
        D = U @ (F * (U.transpose(1, 2) @ E @ U)) @ U.transpose(1, 2)
        D = 0.5 * (D + D.transpose(1, 2))
        blocks = D.reshape(P_, k, b, k, b).permute(0, 1, 3, 2, 4)  # (P, k, k, b, b)
        ok = gather >= 0
        gs.index_add_(0, gather[ok], blocks[ok])
    return gs


class KpmDosLossSandwich(torch.autograd.Function):
    """L(h_values, s_values) = sum_j (rho_j - target_j)^2 for the Jackson DOS
    of the non-orthogonal operator Z^T H Z, Z the graph-local S^-1/2 of S
    (eigen route), from the plain moments of the real sample panel psi
    (bounds held fixed).  h_values, s_values: (nnz, b, b) float64 CUDA
    tensors in H's and S's pattern order (``Hp``, ``Sp``: lattice.BsrArrays
    giving the patterns).  Backward: the device VJP for H and Z, then the
    local Frechet adjoint from Z to S (grad_s_from_grad_z)."""

    @staticmethod
    def forward(ctx, h_values, s_values, Hp, Sp, psi, emin, emax, n_moments, x, target,
                checkpoint_stride=0):
        from .calc import ISQRTMPreconditioner
        from .isqrt import graph_inverse_sqrt
        from .lattice import BsrArrays
        S = BsrArrays(Sp.row_ptr, Sp.col_ind, s_values.detach().cpu().numpy(), Sp.block_size)
        Z = graph_inverse_sqrt(S)
        b = Hp.block_size
        H = BlockSpMat(Hp.row_ptr, Hp.col_ind, h_values.detach().cpu().numpy(), b)
        Zd = BlockSpMat(Z.row_ptr, Z.col_ind, Z.values, b)
        cheby = Chebyshev(H, emin, emax, preconditioner=ISQRTMPreconditioner(Zd))
        mu = kpm_dos_moments_plain(cheby, psi, n_moments).real
        D = dos_basis(n_moments, np.asarray(x, dtype=np.float64))
        resid = D @ mu - np.asarray(target, dtype=np.float64)
        ctx.saved = (cheby, S, psi, n_moments, D, resid, checkpoint_stride)
        return torch.tensor(float(resid @ resid), dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        cheby, S, psi, n_moments, D, resid, stride = ctx.saved
        dmu = float(grad_out) * 2.0 * (resid @ D)
        gh, gz, _, _ = kpm_moments_vjp_sandwich(cheby, psi, n_moments, dmu, stride)
        return (gh, grad_s_from_grad_z(S, gz)) + (None,) * 9
