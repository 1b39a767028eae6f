"""The DOS and transport surface of RSATB's Python object (rsatb/pybind_rsatb.cpp:
549-603, 813-825; rsatb/calc/observables.hpp:311-441, 691-780) over operators
the caller has already built.

Model construction (structures, Slater-Koster / LCAO models) is outside this
package, so ``RSATB`` is constructed from the operators themselves: H, the
optional graph-local factor Z of the overlap, the velocity matrices and the
cell.  ``SetupOptions`` keeps the reference's field names.  Everything below
runs on the device through the C ABI; no result is computed on the host
except the small grids and the final scalings.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import lattice
from .bloch import ImageOperator
from .bounds import estimate_spectral_bounds
from .calc import (Chebyshev, ISQRTMPreconditioner, corr_dos, corr_moment_count,
                   dos_energy_grid, dos_moment_count, evaluate_kpm_density, kpm_dos_moments,
                   kpm_ldos_moments, parse_kpm_kernel)
from .shard import gather_kpoint_results, partition_kpoints, torch_all_reduce_sum
from .transport import BASTIN, GREENWOOD, dc_spectrum_fftcheb, integrate_dc_spectrum
from ._capi import RANDOM_PHASE
from .vbcsr import BlockSpMat, set_random


@dataclass
class PreconditionerOptions:
    """rsatb::model::PreconditionerOptions (rsatb/model/setup.hpp:33-51):
    operator_form 'solve' (S^-1 H, a CG with S per application) or
    'sandwich' (Z^H H Z).  tol, sptol and maxiter configure the construction
    of Z from S when the sandwich form is given S rather than Z, as the
    reference's build_preconditioner does (rsatb/model/operator_set.hpp:369):
    the graph-local seed, then maxiter Newton-Schulz steps on the device
    (isqrt.inverse_sqrt); cg_tol and cg_max_iter are the Solve form's CG
    settings (LinearSolver's 1e-8 and 1000)."""
    operator_form: str = "solve"
    tol: float = 1e-7
    sptol: float = 1e-5
    maxiter: int = 0
    cg_tol: float = 1e-8
    cg_max_iter: int = 1000


@dataclass
class SetupOptions:
    """rsatb::model::SetupOptions (pybind_rsatb.cpp:263-341): k-points,
    sampling and spectral bounds.  k-points other than Gamma need the
    operator as real-space images (bloch.ImageOperator), from which H(k) is
    summed on the device; bounds_zero_tol and bounds_max_matvecs drive the
    Lanczos window estimate as BoundsOptions does.  ``precision`` ('f64' or
    'mixed': FP32 vectors and operators, FP64 dots) is this package's
    addition."""
    kpoints: list = field(default_factory=lambda: [[0.0, 0.0, 0.0]])
    nsamples: int = 1
    sample_seed: int = 20240917
    compute_bounds: bool = True
    energy_bounds: tuple | None = None
    bounds_zero_tol: float = 1e-12
    bounds_max_matvecs: int = 10000
    preconditioner: PreconditionerOptions = field(default_factory=PreconditionerOptions)
    precision: str = "f64"


def _as_device(A) -> BlockSpMat:
    if isinstance(A, BlockSpMat):
        return A
    if isinstance(A, lattice.BsrArrays):
        return BlockSpMat(A.row_ptr, A.col_ind, A.values, A.block_size, A.n_block_cols)
    raise TypeError("operators are BlockSpMat or lattice.BsrArrays")


def _volume(cell: np.ndarray, axis: str) -> float:
    """TransportNormalizationVolume (observables.hpp:277-285): the cell vector
    length for one axis, the area for two, the volume for three."""
    idx = ["abc".index(a) for a in axis]
    vecs = [np.asarray(cell[i], dtype=np.float64) for i in idx]
    if len(vecs) == 1:
        return float(np.linalg.norm(vecs[0]))
    if len(vecs) == 2:
        return float(np.linalg.norm(np.cross(vecs[0], vecs[1])))
    return float(abs(np.dot(vecs[0], np.cross(vecs[1], vecs[2]))))


class RSATB:
    """``_rsatb.RSATB`` for prebuilt operators.

    H: Hamiltonian, either one matrix (BlockSpMat or lattice.BsrArrays: the
    Gamma point) or a ``bloch.ImageOperator`` of real-space images, summed on
    the device at every k-point of ``options.kpoints`` (fractional, against
    the image shifts).  Z: graph-local factor of the overlap (non-orthogonal
    basis: the sandwich form Z^H H Z; one matrix only), or None.  velocities:
    (Vx, Vy, Vz) real matrices W_a of the velocities i W_a (for
    compute_dc_spectrum with one matrix H; with images they are summed from
    the bond vectors).  cell: 3 x 3 lattice vectors in
    Angstrom (rows a, b, c).  orbitals_per_atom / atom_index key the seeded
    sample vectors by atom, as SampleVectors::initialize does.
    """

    def __init__(self, H, options: SetupOptions | None = None, Z=None, velocities=None,
                 cell=None, orbitals_per_atom: int = 1, atom_index=None,
                 spin_degeneracy: float = 2.0, S=None, npar: int | None = None):
        self.options = options or SetupOptions()
        self.npar = npar
        if self.options.precision not in ("f64", "mixed"):
            raise ValueError("precision must be 'f64' or 'mixed'")
        self.kpoints = [np.asarray(k, dtype=np.float64).reshape(3) for k in self.options.kpoints]
        if not self.kpoints:
            raise ValueError("kpoints must hold at least one k-point")
        self.images = H if isinstance(H, ImageOperator) else None
        if self.images is None:
            if any(np.any(k != 0.0) for k in self.kpoints):
                raise ValueError("k-points other than Gamma need the operator's images "
                                 "(bloch.ImageOperator)")
            self.H = _as_device(H)
        else:
            if Z is not None:
                raise NotImplementedError("the sandwich form takes one matrix, not images")
            self.H = self.images.at_k(self.kpoints[0])
        self.Z = _as_device(Z) if Z is not None else None
        self.factor_report = None  # InverseSqrtReport when Z is built from S
        self.S = _as_device(S) if S is not None else None
        form = self.options.preconditioner.operator_form.strip().lower()
        if form not in ("solve", "sandwich"):
            raise ValueError(f"Unknown operator form '{form}' (expected solve or sandwich)")
        # An orthogonal basis passes neither matrix; otherwise the form picks
        # which of S and Z the operator uses (ParseOperatorForm, setup.hpp:54).
        # 'solve' takes S (and Z, if given, preconditions its CG, the
        # reference's default route); 'sandwich' takes Z alone.
        if self.S is not None and form == "sandwich":
            # build_preconditioner: Z from S (seed + maxiter refinement steps);
            # the sandwich never references S itself.
            if self.Z is None:
                self.Z, self.factor_report = self._factor_from_overlap(S)
            self.S = None
        if self.Z is not None and self.S is None and form != "sandwich":
            raise ValueError("operator_form 'solve' needs S (Z alone gives the sandwich form)")
        if self.S is not None and self.images is not None:
            raise NotImplementedError("the solve form takes one matrix, not images")
        self.V = None
        if velocities is not None and self.images is not None:
            raise ValueError("with images the velocities come from the bond vectors")
        if velocities is not None:
            self.V = [v if isinstance(v, BlockSpMat) else
                      BlockSpMat(v.row_ptr, v.col_ind, v.values, v.block_size, v.n_block_cols,
                                 imaginary=True)
                      for v in velocities]
        self.cell = None if cell is None else np.asarray(cell, dtype=np.float64)
        self.orbitals_per_atom = int(orbitals_per_atom)
        self.atom_index = atom_index
        self.spin_degeneracy = float(spin_degeneracy)
        self._bounds = None
        if self.options.energy_bounds is not None:
            lo, hi = self.options.energy_bounds
            self._bounds = (float(lo), float(hi))
        elif self.options.compute_bounds:
            self._bounds = self._estimate_bounds()

    # -- operators --------------------------------------------------------

    def _factor_from_overlap(self, S):
        from .isqrt import InverseSqrtOptions, inverse_sqrt
        po = self.options.preconditioner
        arrays = S.to_arrays() if isinstance(S, BlockSpMat) else S
        return inverse_sqrt(arrays, InverseSqrtOptions(tol=po.tol, sptol=po.sptol,
                                                       maxit=po.maxiter))

    def _operator(self, kidx: int) -> BlockSpMat:
        if self.images is None or kidx == 0:
            return self.H
        return self.images.at_k(self.kpoints[kidx])

    def _cheby(self, emin: float, emax: float, mixed: bool, kidx: int = 0) -> Chebyshev:
        pre = ISQRTMPreconditioner(self.Z) if self.Z is not None else None
        po = self.options.preconditioner
        c = Chebyshev(self._operator(kidx), emin, emax, preconditioner=pre, overlap=self.S,
                      cg_tol=po.cg_tol, cg_max_iter=po.cg_max_iter)
        return c.astype("f32") if mixed else c

    # -- k-point distribution over ranks ------------------------------------
    # Under torch.distributed the k-points are spread over npar colours
    # (default: one per rank) as PartitionKPoints does; every rank computes
    # its own k-points with all samples, and the per-k-point results are
    # gathered as GatherKPointResults does.  One process: everything local.

    def _dist(self):
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            return dist.get_rank(), dist.get_world_size()
        return 0, 1

    def _local_kidx(self):
        rank, world = self._dist()
        return [i for i, _ in partition_kpoints(self.kpoints, self.npar or world, rank, world)]

    def _all_reduce(self):
        import torch.distributed as dist
        dev = f"cuda:{self.H.ctx.device}" if dist.get_backend() == "nccl" else None
        return torch_all_reduce_sum(device=dev)

    def _gather(self, per_k: np.ndarray) -> np.ndarray:
        rank, world = self._dist()
        if world == 1:
            return per_k
        return gather_kpoint_results(per_k, self.npar or world, rank, world, self._all_reduce())

    def _estimate_bounds(self):
        """The widest padded Lanczos window over the k-points (the reference
        keeps one window for all of them, OperatorSet::emin/emax)."""
        lo, hi = np.inf, -np.inf
        for kidx in self._local_kidx():
            opt = self.options
            a, b = estimate_spectral_bounds(self._cheby(-1.0, 1.0, False, kidx), tol=1e-3,
                                            zero_tol=opt.bounds_zero_tol,
                                            max_matvecs=opt.bounds_max_matvecs)
            lo, hi = min(lo, a), max(hi, b)
        if self._dist()[1] > 1:
            import torch.distributed as dist
            dev = f"cuda:{self.H.ctx.device}" if dist.get_backend() == "nccl" else "cpu"
            t = torch.tensor([-lo, hi], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            lo, hi = -float(t[0]), float(t[1])
        return lo, hi

    def energy_bounds(self):
        """(emin, emax) of the operator, padded as the reference pads its
        Lanczos estimate (spectral_bounds.hpp:75)."""
        if self._bounds is None:
            raise RuntimeError("Spectral bound is not computed yet. Set it true during Setup "
                               "stage for random state method support.")
        return self._bounds

    def _samples(self, dtype) -> torch.Tensor:
        n = self.H.shape[0]
        psi = torch.empty(n, self.options.nsamples, dtype=dtype,
                          device=f"cuda:{self.H.ctx.device}")
        set_random(psi, int(self.options.sample_seed), normalize=True,
                   atom_index=self.atom_index, orbitals_per_atom=self.orbitals_per_atom,
                   kind=RANDOM_PHASE)
        return psi

    # -- observables ------------------------------------------------------

    def compute_dos(self, dE: float, method: str = "kpm"):
        """ComputeDos (observables.hpp:311-441).  'kpm': the Jackson moment
        count for a FWHM of dE, the KPM density on the 2 nt grid, scaled by
        2.  'corr': the moments of the longest time nt*pi, the correlation
        series, Hann window and inverse FFT.  Returns (dos, omega)."""
        if method != "kpm" and method != "corr":
            raise ValueError(f"dos method must be 'kpm' or 'corr', got '{method}'")
        if not dE > 0.0:
            raise ValueError("dos dE must be a positive energy resolution in eV")
        emin, emax = self.energy_bounds()
        x, omega, nt = dos_energy_grid(emin, emax, dE)
        dev = self.H.ctx.device
        if method == "kpm":
            N = dos_moment_count((emax - emin) / 2.0, dE)
        else:
            N = corr_moment_count(nt, device=dev)
        mixed = self.options.precision == "mixed"
        psi = self._samples(torch.complex64 if mixed else torch.complex128)
        # One DOS of 2 nt points per k-point, in k-point order
        # (observables.hpp:368, 383-386: offset k_idx * 2 nt).
        out = np.zeros((len(self.kpoints), 2 * nt))
        for kidx in self._local_kidx():
            mu = kpm_dos_moments(self._cheby(emin, emax, mixed, kidx), psi, N)
            if method == "corr":
                out[kidx] = corr_dos(mu, nt, device=dev)[0]
            else:
                out[kidx] = 2.0 * evaluate_kpm_density(mu, x, 0.5 / nt, device=dev)
        return self._gather(out).reshape(-1), omega

    def compute_ldos(self, orbitals, dE: float):
        """Orbital-resolved KPM local DOS on ComputeDos's grid: for every
        orbital i, 2 rho_i(x) with rho_i from the moments <e_i|T_n|e_i> and
        the Jackson moment count of compute_dos (the same factor 2 and the
        same per-unit-x convention as compute_dos).  Returns
        (ldos[n_k, n_orbitals, 2 nt], omega)."""
        if not dE > 0.0:
            raise ValueError("dE must be a positive energy resolution in eV")
        emin, emax = self.energy_bounds()
        x, omega, nt = dos_energy_grid(emin, emax, dE)
        N = dos_moment_count((emax - emin) / 2.0, dE)
        idx = np.asarray(orbitals, dtype=np.int64).reshape(-1)
        mixed = self.options.precision == "mixed"
        dev = self.H.ctx.device
        out = np.zeros((len(self.kpoints), idx.size, 2 * nt))
        for kidx in self._local_kidx():
            mu = kpm_ldos_moments(self._cheby(emin, emax, mixed, kidx), idx, N)
            for j in range(idx.size):
                out[kidx, j] = 2.0 * evaluate_kpm_density(mu[:, j], x, 0.5 / nt, device=dev)
        return self._gather(out), omega

    def compute_dc_spectrum(self, n_moments: int, formulation: str = "greenwood",
                            axis: str = "abc", partition_sections: int = 0,
                            max_workspace_mb: float = 0, kernel: str = "jackson",
                            method: str = "fftcheb"):
        """ComputeDcSpectrum (observables.hpp:691-780) with the fftcheb method:
        prefactor pi g_s (4 Greenwood, 8 Bastin) norb / volume(axis).  With
        images, H(k) and the commutator velocities V_a(k) are summed on the
        device for every k-point.  Returns (sigma[n_k * n_moments * 6],
        energy[n_moments]), one block of sigma per k-point in k-point order."""
        if method != "fftcheb":
            raise NotImplementedError(f"dc method '{method}': only 'fftcheb' is served")
        if self.V is None and self.images is None:
            raise ValueError("compute_dc_spectrum needs the velocity matrices")
        if self.cell is None:
            raise ValueError("compute_dc_spectrum needs the cell for its normalisation")
        if self.S is not None:
            raise NotImplementedError("compute_dc_spectrum: the solve form is not served; use "
                                      "operator_form 'sandwich' with Z")
        forms = {"greenwood": GREENWOOD, "bastin": BASTIN}
        if formulation not in forms:
            raise ValueError(f"Unknown dc formulation: {formulation}")
        if not axis or any(a not in "abc" for a in axis) or len(set(axis)) != len(axis):
            raise ValueError(f"axis must be a subset of 'abc', got '{axis}'")
        emin, emax = self.energy_bounds()
        mixed = self.options.precision == "mixed"
        psi = self._samples(torch.complex64 if mixed else torch.complex128)
        norb = self.H.shape[0]
        trace_prefactor = norb / _volume(self.cell, axis)
        prefactor = (math.pi * self.spin_degeneracy *
                     (4.0 if formulation == "greenwood" else 8.0) * trace_prefactor)
        sigmas = np.zeros((len(self.kpoints), int(n_moments) * 6))
        energy = None
        for kidx in self._local_kidx():
            k = self.kpoints[kidx]
            c = self._cheby(emin, emax, mixed, kidx)
            if self.images is not None:
                V = [self.images.velocity_at_k(k, a) for a in range(3)]
            else:
                V = self.V
            if mixed:
                V = [v.astype("f32") for v in V]
            sigma, en = dc_spectrum_fftcheb(
                c, *V, psi, int(n_moments), forms[formulation], prefactor,
                int(partition_sections), float(max_workspace_mb), parse_kpm_kernel(kernel))
            sigmas[kidx] = sigma.reshape(-1)
            if energy is None:
                energy = en
        rank, world = self._dist()
        if world > 1:
            # The grid is the same for every k-point; rank 0 owns k-point 0
            # (BroadcastSharedGrid, observables.hpp:156-175).
            mine = energy if rank == 0 else np.zeros(int(n_moments))
            energy = self._all_reduce()(np.asarray(mine, dtype=np.float64))
        return self._gather(sigmas).reshape(-1), energy

    def compute_dc(self, n_moments: int, mu: float, temp: float, formulation: str = "greenwood",
                   axis: str = "abc", partition_sections: int = 0, max_workspace_mb: float = 0,
                   kernel: str = "jackson", method: str = "fftcheb"):
        """ComputeDc (observables.hpp:791-850): the spectrum of
        compute_dc_spectrum integrated against -df/dE at (mu, temp) per
        k-point.  Returns 6 values per k-point."""
        sigma, energy = self.compute_dc_spectrum(n_moments, formulation, axis, partition_sections,
                                                 max_workspace_mb, kernel, method)
        dev = self.H.ctx.device
        per_k = sigma.reshape(len(self.kpoints), n_moments, 6)
        return np.concatenate([integrate_dc_spectrum(sk, energy, mu, temp, device=dev)
                               for sk in per_k])
