"""FFT-Chebyshev Kubo-Greenwood transport on the GPU.

``dc_spectrum_fftcheb`` mirrors rsatb::calc::dc_spectrum_fftcheb
(rsatb/calc/fftcheb_transport.hpp:543-660): same arguments (Chebyshev
operator, three velocity matrices, sample block, moment count, formulation,
prefactor, partition sections, workspace bound, kernel) and results
(sigma[n_moments, 6] on the ascending energy grid).  The recurrences, the
per-row DCT-III and the contraction run in the rsatb_b200 library
(rsatb_dc_spectrum_fftcheb); this module validates arguments and moves
handles.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _capi
from ._capi import check, lib
from .calc import Chebyshev, KpmKernel
from .vbcsr import BlockSpMat, dtype_code

GREENWOOD, BASTIN = 0, 1


def dc_spectrum_fftcheb(cheby: Chebyshev, Vx: BlockSpMat, Vy: BlockSpMat, Vz: BlockSpMat,
                        psi: torch.Tensor, n_moments: int, formulation: int = GREENWOOD,
                        prefactor: float = 1.0, partition_sections: int = 0,
                        max_workspace_mb: float = 0.0, kernel: KpmKernel = KpmKernel.Jackson,
                        return_stats: bool = False):
    """Returns (sigma[n_moments, 6], energy[n_moments]) and, with
    return_stats, the call's counters.  Greenwood: the zero-temperature
    sigma(E) (diagonal components); Bastin: sigma(mu, T = 0), the cumulative
    energy integral of the six-component zeta kernel.  psi: (N, R) complex CUDA tensor
    (complex128, or complex64 for FP32 vectors)."""
    if n_moments <= 0:
        raise ValueError("n_moments must be positive")
    if not psi.is_cuda or psi.dim() != 2 or not psi.is_contiguous() or not psi.is_complex():
        raise ValueError("psi must be a contiguous (N, R) complex CUDA tensor")
    if psi.shape[0] != cheby.n_rows:
        raise ValueError("psi rows differ from the operator size")
    if formulation not in (GREENWOOD, BASTIN):
        raise ValueError("formulation must be GREENWOOD (0) or BASTIN (1)")
    ctx = cheby.H.ctx
    ctx.bind_stream()
    op = cheby.c_op()
    sigma = np.zeros(n_moments * 6)
    energy = np.zeros(n_moments)
    stats = _capi.FftchebStats()
    P = C.POINTER(C.c_double)
    check(lib().rsatb_dc_spectrum_fftcheb(
        ctx.handle, C.byref(op), Vx.handle, Vy.handle, Vz.handle, C.c_void_p(psi.data_ptr()),
        psi.shape[1], dtype_code(psi.dtype), int(n_moments), int(formulation), float(prefactor),
        int(partition_sections), int(max_workspace_mb * (1 << 20)), int(kernel),
        sigma.ctypes.data_as(P), energy.ctypes.data_as(P), C.byref(stats)))
    out = (sigma.reshape(n_moments, 6), energy)
    if return_stats:
        return out + ({f: getattr(stats, f) for f, _ in stats._fields_},)
    return out


def dc_spectrum_qe(cheby: Chebyshev, Vx: BlockSpMat, Vy: BlockSpMat, Vz: BlockSpMat,
                   psi: torch.Tensor, n_moments: int, prefactor: float = 1.0,
                   kernel: KpmKernel = KpmKernel.Jackson, nodes_ascending=None):
    """rsatb::calc::dc_spectrum_qe (rsatb/calc/fftcheb_transport.hpp:
    662-884): the Greenwood sigma at the nodes_ascending window of the
    ascending grid (all nodes when None) by quasi-eigenstates, without the
    row store; same (sigma[n_moments, 6], energy[n_moments]) as
    dc_spectrum_fftcheb, sigma zero outside the window."""
    if n_moments <= 0:
        raise ValueError("n_moments must be positive")
    if not psi.is_cuda or psi.dim() != 2 or not psi.is_contiguous() or not psi.is_complex():
        raise ValueError("psi must be a contiguous (N, R) complex CUDA tensor")
    if psi.shape[0] != cheby.n_rows:
        raise ValueError("psi rows differ from the operator size")
    nodes = (np.zeros(0, np.int32) if nodes_ascending is None else
             np.ascontiguousarray(np.asarray(nodes_ascending, dtype=np.int32)))
    ctx = cheby.H.ctx
    ctx.bind_stream()
    op = cheby.c_op()
    sigma = np.zeros(n_moments * 6)
    energy = np.zeros(n_moments)
    P = C.POINTER(C.c_double)
    check(lib().rsatb_dc_spectrum_qe(
        ctx.handle, C.byref(op), Vx.handle, Vy.handle, Vz.handle, C.c_void_p(psi.data_ptr()),
        psi.shape[1], dtype_code(psi.dtype), int(n_moments), float(prefactor), int(kernel),
        nodes.ctypes.data if nodes.size else None, int(nodes.size), sigma.ctypes.data_as(P),
        energy.ctypes.data_as(P)))
    return sigma.reshape(n_moments, 6), energy


def integrate_dc_spectrum(sigma, energy, mu: float, temp: float, device=None) -> np.ndarray:
    """sigma(mu, T) (6 components) from a zero-temperature spectrum
    sigma[n_energy, 6] on `energy` (fftcheb_transport.hpp:950-1040), on the
    GPU: linear interpolation at T <= 0, the exact integral of the
    piecewise-linear spectrum against -df/dE at T > 0 (kelvin)."""
    from .vbcsr import context
    s = np.ascontiguousarray(np.asarray(sigma, dtype=np.float64).reshape(-1, 6))
    e = np.ascontiguousarray(np.asarray(energy, dtype=np.float64).reshape(-1))
    if s.shape[0] != e.size:
        raise ValueError("sigma must hold 6 values per energy")
    out = np.zeros(6)
    P = C.POINTER(C.c_double)
    check(lib().rsatb_integrate_dc_spectrum(context(device).handle, s.ctypes.data_as(P),
                                            e.ctypes.data_as(P), e.size, float(mu), float(temp),
                                            out.ctypes.data_as(P)))
    return out
