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
