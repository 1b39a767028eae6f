"""The KPM engine of rsatb/calc, on the GPU.

Mirrors the reference's calc-layer interface for the DOS path:

* ``Chebyshev`` -- rsatb::calc::Chebyshev<T> (rsatb/calc/cheby.hpp:147-668):
  the rescaled operator (H - center)/half_width in the Orthogonal or the
  Sandwich (Z^H H Z) form, ``apply_op``, ``op_is_hermitian``,
  ``compute_moments``.
* ``kpm_dos_moments`` -- rsatb/calc/dos.hpp:125-190.
* ``jackson_kernel``, ``kpm_kernel_weights``, ``evaluate_kpm_density`` --
  rsatb/calc/kpm.hpp:18-85, 206-241.
* ``ISQRTMPreconditioner`` (borrowing form) -- rsatb/calc/preconditioner.hpp:
  169-240, holding Z and Z^H for the sandwich.

Every numerical step runs in the rsatb_b200 CUDA library; this module only
validates arguments and moves handles.
"""
from __future__ import annotations

import ctypes as C
import enum
import math

import numpy as np
import torch

from . import _capi
from ._capi import check, lib
from .vbcsr import BlockSpMat, context, dtype_code


class ChebyMode(enum.IntEnum):
    """rsatb::calc::ChebyMode (cheby.hpp:58)."""
    NORMAL = 0
    ADJOINT = 1


class ChebyOpForm(enum.IntEnum):
    """rsatb::calc::ChebyOpForm (cheby.hpp:78-82)."""
    Orthogonal = 0
    Solve = 1
    Sandwich = 2


class KpmKernel(enum.IntEnum):
    """rsatb::calc::KpmKernel (kpm.hpp:49)."""
    None_ = _capi.KPM_NONE
    Jackson = _capi.KPM_JACKSON
    CosTaper = _capi.KPM_COSTAPER
    VpTaper = _capi.KPM_VPTAPER


def parse_kpm_kernel(name: str) -> KpmKernel:
    """kpm.hpp:104-111."""
    table = {"jackson": KpmKernel.Jackson, "costaper": KpmKernel.CosTaper,
             "vptaper": KpmKernel.VpTaper, "none": KpmKernel.None_}
    if name not in table:
        raise ValueError(f"Unknown KPM kernel '{name}' (expected jackson, costaper, vptaper, or none)")
    return table[name]


class ISQRTMPreconditioner:
    """Borrowing ISQRTMPreconditioner: applies a given factor Z and Z^H.

    The reference's computing constructor runs inverse_sqrt (isqrtm.hpp:262);
    here the factor comes from ``rsatb_b200.isqrt`` and is passed in.
    ``adjoint`` defaults to Z.adjoint() built once on the device.
    """

    def __init__(self, factor: BlockSpMat, adjoint: BlockSpMat | None = None):
        self.Z = factor
        self.ZH = adjoint if adjoint is not None else factor.adjoint()

    def factor(self) -> BlockSpMat:
        return self.Z

    def astype(self, precision: str) -> "ISQRTMPreconditioner":
        return ISQRTMPreconditioner(self.Z.astype(precision), self.ZH.astype(precision))


class Chebyshev:
    """Rescaled operator Op~ = (Op - center)/half_width on the GPU.

    ``Chebyshev(H, emin, emax)`` is the Orthogonal form;
    ``Chebyshev(H, emin, emax, preconditioner=pre)`` the Sandwich form
    Z^H H Z;  ``Chebyshev(H, emin, emax, overlap=S)`` the Solve form S^-1 H,
    one batched CG with S per application (cheby.hpp:188-192; tolerance
    ``cg_tol`` 1e-8 and at most ``cg_max_iter`` 1000 iterations, as
    LinearSolver's defaults), preconditioned by the factor of
    ``preconditioner`` when one is given as well.  The Solve form serves
    ``apply_op`` (NORMAL), ``apply_dual`` (both modes), ``propagate`` and
    the plain moment recurrence.
    """

    def __init__(self, H: BlockSpMat, emin: float, emax: float,
                 preconditioner: ISQRTMPreconditioner | None = None, verbose: bool = False,
                 overlap: BlockSpMat | None = None, cg_tol: float = 1e-8,
                 cg_max_iter: int = 1000):
        if H.shape[0] != H.shape[1]:
            raise ValueError("H must be square")
        if overlap is not None and overlap.shape != H.shape:
            raise ValueError("S and H shapes differ")
        self.H = H
        self.M = preconditioner
        self.S = overlap
        self.cg_tol, self.cg_max_iter = float(cg_tol), int(cg_max_iter)
        if overlap is not None:
            # With a preconditioner too: its factor preconditions the CG
            # symmetrically (cheby.hpp:195-199), the operator stays S^-1 H.
            self.form = ChebyOpForm.Solve
        else:
            self.form = ChebyOpForm.Sandwich if preconditioner is not None else ChebyOpForm.Orthogonal
        self.verbose = verbose
        self.set_window(emin, emax)

    def set_window(self, emin: float, emax: float) -> None:
        """cheby.hpp:517-520."""
        self.center = (emax + emin) / 2.0
        self.half_width = (emax - emin) / 2.0

    @property
    def n_rows(self) -> int:
        return self.H.shape[0]

    @property
    def is_double(self) -> bool:
        return self.H.is_double

    def op_is_hermitian(self) -> bool:
        """cheby.hpp:222: Orthogonal and Sandwich are Hermitian, Solve is not."""
        return self.form != ChebyOpForm.Solve

    def astype(self, precision: str) -> "Chebyshev":
        """A copy whose matrices are stored in 'f64' or 'f32'."""
        pre = self.M.astype(precision) if self.M is not None else None
        S = self.S.astype(precision) if self.S is not None else None
        c = Chebyshev(self.H.astype(precision), self.center - self.half_width,
                      self.center + self.half_width, preconditioner=pre, overlap=S,
                      cg_tol=self.cg_tol, cg_max_iter=self.cg_max_iter)
        return c

    def c_op(self) -> _capi.ChebOp:
        op = _capi.ChebOp()
        op.form = {ChebyOpForm.Sandwich: _capi.FORM_SANDWICH, ChebyOpForm.Solve: _capi.FORM_SOLVE,
                   ChebyOpForm.Orthogonal: _capi.FORM_ORTHOGONAL}[self.form]
        op.H = self.H.handle
        if self.M is not None:
            op.Z = self.M.Z.handle
            op.ZH = self.M.ZH.handle
        if self.S is not None:
            op.S = self.S.handle
            op.cg_tol = self.cg_tol
            op.cg_max_iter = self.cg_max_iter
        op.center = self.center
        op.half_width = self.half_width
        return op

    def apply_op(self, X: torch.Tensor, Y: torch.Tensor, mode: ChebyMode = ChebyMode.NORMAL):
        """Y = Op~ X (cheby.hpp:232-235); ADJOINT equals NORMAL for the
        Hermitian forms.  Solve form: Y's contents start the CG."""
        if self.form == ChebyOpForm.Solve and mode == ChebyMode.ADJOINT:
            raise NotImplementedError("the Solve form serves NORMAL applications only")
        ctx = self.H.ctx
        ctx.bind_stream()
        op = self.c_op()
        check(lib().rsatb_cheb_apply_op(ctx.handle, C.byref(op), C.c_void_p(X.data_ptr()),
                                        C.c_void_p(Y.data_ptr()), X.shape[1],
                                        dtype_code(X.dtype)))
        return Y

    def apply_dual(self, V: BlockSpMat, X: torch.Tensor, Y: torch.Tensor,
                   mode: ChebyMode = ChebyMode.NORMAL, scale: float = 1.0) -> torch.Tensor:
        """Y = scale * (V dressed by the form) X: V X (Orthogonal), Z^H V Z X
        (Sandwich), S^-1 V X (Solve; ADJOINT: V S^-1 X) (cheby.hpp:249-291);
        mode is immaterial for the two Hermitian forms."""
        ctx = self.H.ctx
        ctx.bind_stream()
        op = self.c_op()
        fn = (lib().rsatb_cheb_apply_dual_adjoint if mode == ChebyMode.ADJOINT
              else lib().rsatb_cheb_apply_dual)
        check(fn(ctx.handle, C.byref(op), V.handle,
                                          C.c_void_p(X.data_ptr()), C.c_void_p(Y.data_ptr()),
                                          X.shape[1], dtype_code(X.dtype), float(scale)))
        return Y

    def propagate(self, V_in: torch.Tensor, V_out: torch.Tensor, coeffs,
                  mode: ChebyMode = ChebyMode.NORMAL) -> torch.Tensor:
        """V_out = sum_n c_n T_n(Op~) V_in (cheby.hpp:367-441); coeffs complex
        (a real panel takes their real parts).  The Solve form runs a CG per
        application (NORMAL only, as its apply_op)."""
        if self.form == ChebyOpForm.Solve and mode == ChebyMode.ADJOINT:
            raise NotImplementedError("the Solve form serves NORMAL applications only")
        c = np.ascontiguousarray(np.asarray(coeffs, dtype=np.complex128))
        flat = np.ascontiguousarray(np.stack([c.real, c.imag], axis=-1).reshape(-1))
        ctx = self.H.ctx
        ctx.bind_stream()
        op = self.c_op()
        check(lib().rsatb_cheb_propagate(ctx.handle, C.byref(op), C.c_void_p(V_in.data_ptr()),
                                         C.c_void_p(V_out.data_ptr()), V_in.shape[1],
                                         dtype_code(V_in.dtype),
                                         flat.ctypes.data_as(C.POINTER(C.c_double)), int(c.size)))
        return V_out

    def compute_moments(self, V: torch.Tensor, N: int) -> np.ndarray:
        """Per-column plain moments <v|T_n|v>, shape (N, R) (cheby.hpp:479-514)."""
        _, col = _moments(self, V, N, doubled=False, per_column=True)
        return col


def _moments(cheby: Chebyshev, psi: torch.Tensor, n_moments: int, doubled: bool,
             per_column: bool = False):
    if n_moments <= 0:
        raise ValueError("n_moments must be positive")
    if not psi.is_cuda or psi.dim() != 2 or not psi.is_contiguous():
        raise ValueError("psi must be a contiguous (N, R) CUDA tensor")
    if psi.shape[0] != cheby.n_rows:
        raise ValueError("psi rows differ from the operator size")
    ctx = cheby.H.ctx
    ctx.bind_stream()
    op = cheby.c_op()
    R = psi.shape[1]
    mu = np.zeros(2 * n_moments)
    col = np.zeros(2 * n_moments * R) if per_column else None
    check(lib().rsatb_kpm_dos_moments(
        ctx.handle, C.byref(op), C.c_void_p(psi.data_ptr()), R, dtype_code(psi.dtype),
        int(n_moments), int(bool(doubled)), mu.ctypes.data_as(C.POINTER(C.c_double)),
        col.ctypes.data_as(C.POINTER(C.c_double)) if per_column else None))
    m = mu.view(np.complex128)
    if per_column:
        return m, col.view(np.complex128).reshape(n_moments, R)
    return m, None


def kpm_dos_moments(cheby: Chebyshev, psi_in: torch.Tensor, n_moments: int) -> np.ndarray:
    """KPM trace moments averaged over the columns of psi_in (dos.hpp:125).

    Doubled (two moments per matvec) since every form here is Hermitian;
    ``kpm_dos_moments_plain`` runs the plain recurrence.
    """
    m, _ = _moments(cheby, psi_in, n_moments, doubled=cheby.op_is_hermitian())
    return m


def kpm_ldos_moments(cheby: Chebyshev, orbitals, n_moments: int) -> np.ndarray:
    """Local moments mu_n(i) = <e_i|T_n(Op~)|e_i> of the orbitals i, one
    unit column each (KPM local density of states; Weisse et al., Rev. Mod.
    Phys. 78, 275, sec. II.C), through the same recurrence as
    kpm_dos_moments (doubled for the Hermitian forms).  Returns
    (n_moments, len(orbitals)), real."""
    idx = np.asarray(orbitals, dtype=np.int64).reshape(-1)
    if idx.size == 0:
        raise ValueError("no orbitals given")
    if idx.min() < 0 or idx.max() >= cheby.n_rows:
        raise ValueError("orbital index outside the operator")
    cplx = cheby.H.is_complex or cheby.H.imaginary
    if cheby.is_double:
        dt = torch.complex128 if cplx else torch.float64
    else:
        dt = torch.complex64 if cplx else torch.float32
    psi = torch.zeros(cheby.n_rows, idx.size, dtype=dt, device=f"cuda:{cheby.H.ctx.device}")
    psi[torch.as_tensor(idx, device=psi.device), torch.arange(idx.size, device=psi.device)] = 1.0
    _, col = _moments(cheby, psi, n_moments, doubled=cheby.op_is_hermitian(), per_column=True)
    return col.real.copy()


def kpm_dos_moments_plain(cheby: Chebyshev, psi_in: torch.Tensor, n_moments: int) -> np.ndarray:
    m, _ = _moments(cheby, psi_in, n_moments, doubled=False)
    return m


def jackson_kernel(n: int) -> np.ndarray:
    """kpm.hpp:18-33 (host FP64)."""
    return kpm_kernel_weights(KpmKernel.Jackson, n)


def kpm_kernel_weights(kernel: KpmKernel, n: int) -> np.ndarray:
    """kpm.hpp:52-85 (host FP64)."""
    if n <= 0:
        raise ValueError("kpm_kernel_weights: n must be positive")
    g = np.ones(n)
    if kernel == KpmKernel.Jackson:
        denom = float(n + 1)
        theta = math.pi / denom
        cot = math.cos(theta) / math.sin(theta)
        i = np.arange(1, n)
        g[1:] = ((denom - i) * np.cos(theta * i) + cot * np.sin(theta * i)) / denom
    elif kernel == KpmKernel.CosTaper:
        n0 = n // 2
        s = (np.arange(n0, n) - n0) / (n - n0)
        g[n0:] = 0.5 * (1.0 + np.cos(math.pi * s))
    elif kernel == KpmKernel.VpTaper:
        n0 = n // 2
        g[n0:] = (n - np.arange(n0, n)) / (n - n0)
    return g


def evaluate_kpm_density(moments, x_values, edge_inset: float,
                         kernel: KpmKernel = KpmKernel.Jackson, device=None) -> np.ndarray:
    """rho(x) from moments on the GPU (kpm.hpp:206-241)."""
    mu = np.ascontiguousarray(np.asarray(moments, dtype=np.complex128))
    x = np.ascontiguousarray(np.asarray(x_values, dtype=np.float64))
    rho = np.zeros_like(x)
    ctx = context(device)
    P = C.POINTER(C.c_double)
    check(lib().rsatb_evaluate_kpm_density(ctx.handle, mu.view(np.float64).ctypes.data_as(P),
                                           mu.size, x.ctypes.data_as(P), x.size,
                                           float(edge_inset), int(kernel), rho.ctypes.data_as(P)))
    return rho


def dos_moment_count(half_width: float, de_ev: float) -> int:
    """Moments for a Jackson FWHM of dE (observables.hpp:346-349)."""
    jackson_fwhm = math.sqrt(8.0 * math.log(2.0)) * math.pi
    return max(1, int(math.ceil(jackson_fwhm * half_width / de_ev)))


def timeprop_coeff(time_step: float, precision: float = 1e-14, forward: bool = True,
                   device=None) -> np.ndarray:
    """Chebyshev coefficients of exp(-+i x t) (cheby.hpp:85-106, truncated as
    bessel.hpp:9-52), computed on the GPU."""
    ctx = context(device)
    n = C.c_int(0)
    check(lib().rsatb_timeprop_coeff(ctx.handle, float(time_step), float(precision),
                                     int(bool(forward)), 0, None, C.byref(n)))
    out = np.zeros(n.value, dtype=np.complex128)
    P = C.POINTER(C.c_double)
    check(lib().rsatb_timeprop_coeff(ctx.handle, float(time_step), float(precision),
                                     int(bool(forward)), n.value,
                                     out.view(np.float64).ctypes.data_as(P), C.byref(n)))
    return out


def corr_moment_count(nt: int, precision: float = 1e-14, device=None) -> int:
    """Moments the correlation DOS needs: the expansion length of the longest
    time nt*pi (observables.hpp:354-357)."""
    return timeprop_coeff(nt * math.pi, precision, True, device).size


def corr_dos(moments, nt: int, precision: float = 1e-14, device=None):
    """corr_from_moments (dos.hpp:30-46) and the windowed inverse FFT of
    ComputeDos "corr" (observables.hpp:393-428) on the GPU.  Returns
    (dos[2 nt], cdos[nt + 1])."""
    if nt < 1:
        raise ValueError("nt must be positive")
    mu = np.ascontiguousarray(np.asarray(moments, dtype=np.complex128))
    if mu.size < 1:
        raise ValueError("corr_dos needs at least one moment")
    cdos = np.zeros(nt + 1, dtype=np.complex128)
    dos = np.zeros(2 * nt)
    ctx = context(device)
    P = C.POINTER(C.c_double)
    check(lib().rsatb_corr_dos(ctx.handle, mu.view(np.float64).ctypes.data_as(P), mu.size,
                               int(nt), float(precision),
                               cdos.view(np.float64).ctypes.data_as(P), dos.ctypes.data_as(P)))
    return dos, cdos


def cg_solve(S: BlockSpMat, B: torch.Tensor, X: torch.Tensor, tol: float = 1e-8,
             max_iter: int = 1000, preconditioner: "ISQRTMPreconditioner | None" = None):
    """X = S^-1 B column by column by batched CG from X's contents
    (LinearSolver::solve, solver.hpp:216-312), or with the graph-local
    factor as symmetric preconditioner (solver.hpp:329-338).  Returns
    (iterations, largest column residual)."""
    for T in (B, X):
        if not T.is_cuda or T.dim() != 2 or not T.is_contiguous():
            raise ValueError("B and X must be contiguous (N, R) CUDA tensors")
    if B.shape != X.shape or B.dtype != X.dtype:
        raise ValueError("B and X must have one shape and dtype")
    ctx = S.ctx
    ctx.bind_stream()
    it, res = C.c_int(0), C.c_double(0.0)
    Z = preconditioner.Z.handle if preconditioner is not None else None
    ZH = preconditioner.ZH.handle if preconditioner is not None else None
    check(lib().rsatb_cg_solve(ctx.handle, S.handle, Z, ZH, C.c_void_p(B.data_ptr()),
                               C.c_void_p(X.data_ptr()), B.shape[1], dtype_code(B.dtype),
                               float(tol), int(max_iter), C.byref(it), C.byref(res)))
    return it.value, res.value


def dos_energy_grid(emin: float, emax: float, de_ev: float):
    """The uniform 2*nt grid of ComputeDos (observables.hpp:336, 370-375,
    438-443): returns (x_grid, omega, nt)."""
    span = emax - emin
    nt = max(1, int(math.ceil(span / de_ev)))
    i = np.arange(nt)
    x = np.concatenate([(i - nt) / nt, i / nt])
    scale, shift = span / 2.0, (emax + emin) / 2.0
    omega = np.concatenate([(i - nt) * scale / nt + shift, i * scale / nt + shift])
    return x, omega, nt
