"""Spectral bounds of the Chebyshev operator by Lanczos on the GPU.

The reference estimates the extreme eigenvalues with PRIMME and pads them by
BoundsOptions::padding = 0.5 eV (rsatb/setup/spectral_bounds.hpp:67-76,
311-490).  PRIMME is not available, so rsatb_lanczos_extremes runs Lanczos
(full FP64 reorthogonalisation on the device, the tridiagonal Ritz problem
on the host) on the unscaled operator, and each extreme Ritz value is
widened by its residual norm |beta_m y_m| as well as the padding.  Two
modes:

* a fixed number of steps (the benchmark workloads' window, 20 steps);
* with ``tol`` the reference's contract: steps until both extreme Ritz
  pairs have residual <= tol * max|theta| (PRIMME's 1e-3 of the
  spectral_bounds call), at most ``max_matvecs`` applications; a Hamiltonian
  with max|H| <= zero_tol is the zero operator (window (0, 0) before the
  padding); a solve that does not converge falls back to +-||H||_F for an
  orthogonal basis and raises otherwise, as ExtremalEigenvalues does.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import check, lib
from .calc import Chebyshev

PADDING = 0.5  # eV, spectral_bounds.hpp:75
MAX_KRYLOV = 400  # Lanczos vectors kept (full reorthogonalisation)


def lanczos_extremes(cheby: Chebyshev, steps: int = 20, seed: int = 2, tol: float | None = None,
                     max_matvecs: int = 10000, info: dict | None = None):
    """(theta_min, theta_max, res_min, res_max) of the operator cheby iterates
    (its window is ignored: the operator is applied unscaled).  For the
    Solve form S^-1 H the Lanczos basis is S-orthonormal (S^-1 H is
    self-adjoint in the S inner product), the generalised problem
    H x = lambda S x that the reference hands to PRIMME."""
    ctx = cheby.H.ctx
    ctx.bind_stream()
    op = cheby.c_op()
    opts = _capi.LanczosOptions(steps=int(steps), tol=float(tol) if tol is not None else 0.0,
                                max_matvecs=int(max(1, max_matvecs)), seed=int(seed))
    res = _capi.LanczosResult()
    check(lib().rsatb_lanczos_extremes(ctx.handle, C.byref(op), C.byref(opts), C.byref(res)))
    if info is not None:
        info.update(matvecs=int(res.matvecs), converged=bool(res.converged))
    return float(res.theta_min), float(res.theta_max), float(res.res_min), float(res.res_max)


def tridiag_eigen(diag, off):
    """(eigenvalues ascending, last components of the eigenvectors) of the
    symmetric tridiagonal matrix: the Ritz solve of the Lanczos above."""
    d = np.ascontiguousarray(diag, dtype=np.float64)
    e = np.ascontiguousarray(off, dtype=np.float64)
    m = d.size
    if e.size != max(m - 1, 0):
        raise ValueError("off-diagonal length must be len(diag) - 1")
    th = np.empty(m)
    last = np.empty(m)
    ptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    check(lib().rsatb_tridiag_eigen(m, ptr(d), ptr(e if e.size else np.zeros(1)), ptr(th),
                                    ptr(last)))
    return th, last


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
