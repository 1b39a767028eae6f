"""Spectral bounds of the Chebyshev operator by Lanczos on the GPU.

The reference estimates the extreme eigenvalues with PRIMME and pads them by
BoundsOptions::padding = 0.5 eV (rsatb/setup/spectral_bounds.hpp:67-76,
311-490).  PRIMME is not available, so this runs Lanczos (full
reorthogonalisation, FP64) on the unscaled operator, applied through the
rsatb_b200 kernels, and widens each extreme Ritz value by its residual norm
|beta_m s_m| as well as the padding.  Two modes:

* a fixed number of steps (the benchmark workloads' window, 20 steps);
* with ``tol`` the reference's contract: steps until both extreme Ritz
  pairs have residual <= tol * max|theta| (PRIMME's 1e-3 of the
  spectral_bounds call), at most ``max_matvecs`` applications; a Hamiltonian
  with max|H| <= zero_tol is the zero operator (window (0, 0) before the
  padding); a solve that does not converge falls back to +-||H||_F for an
  orthogonal basis and raises otherwise, as ExtremalEigenvalues does.
"""
from __future__ import annotations

import numpy as np
import torch

from .calc import Chebyshev
from .vbcsr import set_random

PADDING = 0.5  # eV, spectral_bounds.hpp:75
MAX_KRYLOV = 400  # Lanczos vectors kept (full reorthogonalisation)


def lanczos_extremes(cheby: Chebyshev, steps: int = 20, seed: int = 2, tol: float | None = None,
                     max_matvecs: int = 10000, info: dict | None = None):
    """(theta_min, theta_max, res_min, res_max) of the operator cheby iterates
    (its window is ignored: the operator is applied unscaled).  For the
    Solve form S^-1 H the Lanczos basis is S-orthonormal (S^-1 H is
    self-adjoint in the S inner product), the generalised problem
    H x = lambda S x that the reference hands to PRIMME."""
    S = getattr(cheby, "S", None)
    unit = Chebyshev(cheby.H, -1.0, 1.0, preconditioner=cheby.M, overlap=S,
                     cg_tol=getattr(cheby, "cg_tol", 1e-8),
                     cg_max_iter=getattr(cheby, "cg_max_iter", 1000))  # center 0, half_width 1
    n = cheby.n_rows
    dt = torch.complex128 if cheby.H.is_complex or cheby.H.imaginary else torch.float64
    if not cheby.H.is_double:
        dt = torch.complex64 if dt == torch.complex128 else torch.float32
    dev = f"cuda:{cheby.H.ctx.device}"
    real = not dt.is_complex
    wdt = torch.float64 if real else torch.complex128   # FP64 Lanczos arithmetic
    v = torch.empty(n, 1, dtype=dt, device=dev)
    set_random(v, seed, normalize=True)
    v = v.to(wdt)
    m = min(steps, n)

    def metric(x):  # S x for the Solve form, x otherwise
        if S is None:
            return x
        out = torch.empty_like(x.to(dt).contiguous())
        S.mult_dense(x.to(dt).contiguous(), out)
        return out.to(wdt)

    if tol is not None:
        m = min(n, max(1, max_matvecs), MAX_KRYLOV)
    converged = tol is None
    v = v / torch.sqrt(torch.vdot(v[:, 0], metric(v)[:, 0]).real)
    Q = torch.zeros(n, m, dtype=wdt, device=dev)
    SQ = torch.zeros(n, m, dtype=wdt, device=dev)
    alpha = np.zeros(m)
    beta = np.zeros(m)
    w = torch.zeros_like(v.to(dt))
    q = v
    for j in range(m):
        Q[:, j] = q[:, 0]
        SQ[:, j] = metric(q)[:, 0]
        w.zero_()
        unit.apply_op(q.to(dt).contiguous(), w)
        wc = w.to(wdt)
        a = torch.vdot(SQ[:, j], wc[:, 0]).real.item()
        alpha[j] = a
        for _ in range(2):  # full reorthogonalisation in the (S) inner product
            wc = wc - Q[:, :j + 1] @ (SQ[:, :j + 1].conj().T @ wc)
        b = torch.sqrt(torch.vdot(wc[:, 0], metric(wc)[:, 0]).real.clamp(min=0.0)).item()
        beta[j] = b
        if b < 1e-12 * max(1.0, abs(a)):
            m = j + 1
            converged = True
            break
        if tol is not None and j >= 3 and j % 2 == 1:
            Tj = (np.diag(alpha[:j + 1]) + np.diag(beta[:j], 1) + np.diag(beta[:j], -1))
            th, Yj = np.linalg.eigh(Tj)
            rj = np.abs(b * Yj[-1, :])
            scale = max(abs(th[0]), abs(th[-1]), 1e-300)
            if rj[0] <= tol * scale and rj[-1] <= tol * scale:
                m = j + 1
                converged = True
                break
        q = wc / b
    T = np.diag(alpha[:m]) + np.diag(beta[:m - 1], 1) + np.diag(beta[:m - 1], -1)
    theta, Y = np.linalg.eigh(T)
    res = np.abs(beta[m - 1] * Y[-1, :])
    if info is not None:
        info.update(matvecs=m, converged=converged)
    return float(theta[0]), float(theta[-1]), float(res[0]), float(res[-1])


def estimate_spectral_bounds(cheby: Chebyshev, steps: int = 20, padding: float = PADDING,
                             seed: int = 2, tol: float | None = None,
                             zero_tol: float | None = None, max_matvecs: int = 10000,
                             info: dict | None = None):
    """(emin, emax) to pass to Chebyshev; EstimateSpectralBounds analogue
    (fixed steps, or with tol the converging solve described above)."""
    if zero_tol is not None:
        hmax = float(cheby.H.values_tensor().abs().max()) if cheby.H.nnz_blocks else 0.0
        if not np.isfinite(hmax):
            raise RuntimeError("Automatic bounds estimation found a non-finite Hamiltonian "
                               "entry.")
        if hmax <= zero_tol:
            return -padding, padding
    inf = {} if info is None else info
    tmin, tmax, rmin, rmax = lanczos_extremes(cheby, steps, seed, tol, max_matvecs, inf)
    if tol is not None and not inf["converged"]:
        if cheby.M is not None or getattr(cheby, "S", None) is not None:
            raise RuntimeError("Automatic bounds estimation failed: the extreme eigenvalues "
                               f"did not converge within {max_matvecs} matvecs. Provide "
                               "explicit energy bounds or increase max_matvecs.")
        fro = float(cheby.H.values_tensor().abs().pow(2).sum().sqrt())
        return -fro - padding, fro + padding
    return tmin - padding - rmin, tmax + padding + rmax
