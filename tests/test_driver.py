"""The RSATB facade (rsatb_b200.driver): ComputeDos and ComputeDcSpectrum
(rsatb/calc/observables.hpp:311-441, 691-780) over prebuilt operators,
checked against the oracle's moments, density and fftcheb on the same
seeded sample vectors."""
from __future__ import annotations

import math

import numpy as np
import pytest

import oracle
from _util import rel_err, to_oracle


def test_normalisation_volume():
    from rsatb_b200.driver import _volume
    cell = np.array([[2.0, 0.0, 0.0], [1.0, 3.0, 0.0], [0.0, 0.0, 5.0]])
    assert _volume(cell, "a") == pytest.approx(2.0)
    assert _volume(cell, "b") == pytest.approx(math.sqrt(10.0))
    assert _volume(cell, "ab") == pytest.approx(6.0)
    assert _volume(cell, "abc") == pytest.approx(30.0)
    assert _volume(cell, "ac") == pytest.approx(10.0)


def test_setup_options_defaults():
    """SetupOptions and PreconditionerOptions defaults of the reference
    (pybind_rsatb.cpp:292-299, rsatb/model/setup.hpp:33-51)."""
    from rsatb_b200.driver import SetupOptions
    o = SetupOptions()
    assert o.nsamples == 1 and o.sample_seed == 20240917 and o.compute_bounds
    assert o.kpoints == [[0.0, 0.0, 0.0]] and o.energy_bounds is None
    assert o.bounds_zero_tol == 1e-12 and o.bounds_max_matvecs == 10000
    p = o.preconditioner
    assert (p.operator_form, p.tol, p.sptol, p.maxiter) == ("solve", 1e-7, 1e-5, 0)
    assert (p.cg_tol, p.cg_max_iter) == (1e-8, 1000)


def _oracle_samples(n, nsamples, seed):
    return oracle.set_random(seed, 0, True, np.arange(n), 1, n, nsamples, True)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_compute_dos_matches_oracle(precision):
    import torch
    from rsatb_b200 import lattice
    from rsatb_b200.calc import dos_energy_grid, dos_moment_count
    from rsatb_b200.driver import RSATB, SetupOptions
    torch.cuda.set_device(0)
    H, _, _ = lattice.graphene(12, 12)
    emin, emax = -8.6, 8.7
    opts = SetupOptions(nsamples=3, sample_seed=77, energy_bounds=(emin, emax),
                        precision=precision)
    calc = RSATB(H, opts)
    assert calc.energy_bounds() == (emin, emax)
    dE = 0.25
    dos, omega = calc.compute_dos(dE)
    N = dos_moment_count((emax - emin) / 2, dE)
    x, omega_o, nt = dos_energy_grid(emin, emax, dE)
    psi = _oracle_samples(H.n_rows, 3, 77)
    op = oracle.make_op(to_oracle(H), (emax + emin) / 2, (emax - emin) / 2)
    mu = oracle.kpm_moments(op, psi, N)
    want = 2.0 * oracle.density(mu, x, 0.5 / nt)
    assert dos.shape == (2 * nt,) and np.array_equal(omega, omega_o)
    assert rel_err(dos, want) < (1e-10 if precision == "f64" else 1e-5)
    # ComputeDos returns 2 rho(x) per unit of the rescaled energy x (grid
    # step 1 / nt): it integrates to 2 (spin) over [-1, 1].
    assert abs(np.sum(dos) / nt - 2.0) < 0.05


@pytest.mark.gpu
def test_compute_dos_bounds_and_errors():
    import torch
    from rsatb_b200 import lattice
    from rsatb_b200.driver import RSATB, SetupOptions
    torch.cuda.set_device(0)
    H, _, _ = lattice.graphene(8, 8)
    calc = RSATB(H, SetupOptions())
    lo, hi = calc.energy_bounds()
    w = np.linalg.eigvalsh(H.to_dense())
    assert lo < w[0] and hi > w[-1]
    with pytest.raises(ValueError):
        calc.compute_dos(0.0)
    with pytest.raises(ValueError):
        calc.compute_dos(0.1, method="lanczos")
    # Both estimators share the grid and integrate to 2 per unit of x (grid
    # step 1 / nt); their integrated DOS curves agree to the broadening.
    d_kpm, w_kpm = calc.compute_dos(0.3)
    d_corr, w_corr = calc.compute_dos(0.3, method="corr")
    nt = d_kpm.size // 2
    assert np.array_equal(w_kpm, w_corr)
    assert abs(d_kpm.sum() / nt - 2.0) < 0.05 and abs(d_corr.sum() / nt - 2.0) < 1e-9
    assert np.abs(np.cumsum(d_kpm) - np.cumsum(d_corr)).max() / nt < 0.25
    none = RSATB(H, SetupOptions(compute_bounds=False))
    with pytest.raises(RuntimeError):
        none.energy_bounds()
    with pytest.raises(ValueError):
        calc.compute_dc_spectrum(16)


@pytest.mark.gpu
@pytest.mark.parametrize("formulation", ["greenwood", "bastin"])
def test_compute_dc_spectrum_matches_oracle(formulation):
    import torch
    from rsatb_b200 import lattice
    from rsatb_b200.driver import RSATB, SetupOptions, _volume
    torch.cuda.set_device(0)
    H, pos, cell, disp = lattice.twisted_bilayer_graphene(m=1, tiles=(4, 4))
    V = lattice.commutator_velocity(H, disp)
    w = np.linalg.eigvalsh(H.to_dense())
    emin, emax = w[0] - 0.5, w[-1] + 0.5
    opts = SetupOptions(nsamples=2, sample_seed=9, energy_bounds=(emin, emax))
    calc = RSATB(H, opts, velocities=V, cell=cell)
    M = 48
    sigma, energy = calc.compute_dc_spectrum(M, formulation=formulation, axis="ab")
    psi = _oracle_samples(H.n_rows, 2, 9)
    op = oracle.make_op(to_oracle(H), (emax + emin) / 2, (emax - emin) / 2)
    Vo = [to_oracle(v, imag=True) for v in V]
    pref = math.pi * 2.0 * (4.0 if formulation == "greenwood" else 8.0) * H.n_rows / _volume(cell, "ab")
    sig_o, en_o = oracle.fftcheb(op, Vo, psi, M, formulation=0 if formulation == "greenwood" else 1,
                                 prefactor=pref)
    assert sigma.shape == (6 * M,)
    assert np.allclose(energy, en_o, rtol=0, atol=1e-13)
    assert rel_err(sigma, sig_o.reshape(-1)) < 1e-10
    with pytest.raises(ValueError):
        calc.compute_dc_spectrum(M, formulation="kubo")
    with pytest.raises(ValueError):
        calc.compute_dc_spectrum(M, axis="xy")


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_compute_dos_corr_matches_oracle(precision):
    import torch
    from rsatb_b200 import lattice
    from rsatb_b200.calc import dos_energy_grid
    from rsatb_b200.driver import RSATB, SetupOptions
    torch.cuda.set_device(0)
    H, _, _ = lattice.graphene(12, 12)
    emin, emax = -8.6, 8.7
    calc = RSATB(H, SetupOptions(nsamples=2, sample_seed=5, energy_bounds=(emin, emax),
                                 precision=precision))
    dE = 0.4
    dos, omega = calc.compute_dos(dE, method="corr")
    x, omega_o, nt = dos_energy_grid(emin, emax, dE)
    N = oracle.timeprop_coeff(nt * np.pi).size
    psi = _oracle_samples(H.n_rows, 2, 5)
    op = oracle.make_op(to_oracle(H), (emax + emin) / 2, (emax - emin) / 2)
    want, _ = oracle.corr_dos(oracle.kpm_moments(op, psi, N), nt)
    assert dos.shape == (2 * nt,) and np.array_equal(omega, omega_o)
    assert np.abs(dos - want).max() < (1e-10 if precision == "f64" else 1e-5) * np.abs(want).max()


@pytest.mark.gpu
def test_compute_dos_kpoints_matches_oracle():
    """k-points from real-space images: one DOS of 2 nt points per k-point,
    in k-point order (observables.hpp:368-386), each equal to the oracle's
    KPM density of the oracle's dense Bloch sum; the estimated window holds
    every band of every k-point."""
    import torch
    from rsatb_b200 import lattice
    from rsatb_b200.bloch import ImageOperator
    from rsatb_b200.calc import dos_energy_grid, dos_moment_count
    from rsatb_b200.driver import RSATB, SetupOptions
    from rsatb_b200.lattice import BsrArrays
    torch.cuda.set_device(0)
    r, c, sh, bl, bv, n, cell = lattice.graphene_images(6, 6)
    op = ImageOperator(r, c, sh, bl, 1, n, bond_vectors=bv)
    kpts = [[0.0, 0.0, 0.0], [0.25, 0.1, 0.0], [0.5, 0.5, 0.0]]
    emin, emax = -8.6, 8.7
    calc = RSATB(op, SetupOptions(kpoints=kpts, nsamples=2, sample_seed=3,
                                  energy_bounds=(emin, emax)))
    dE = 0.3
    dos, omega = calc.compute_dos(dE)
    x, _, nt = dos_energy_grid(emin, emax, dE)
    N = dos_moment_count((emax - emin) / 2, dE)
    psi = _oracle_samples(n, 2, 3)
    assert dos.shape == (3 * 2 * nt,)
    rows = np.repeat(np.arange(n), np.diff(op.row_ptr))
    for q, k in enumerate(kpts):
        Hd = oracle.bloch_dense(r, c, sh, bl, n, k)
        A = BsrArrays(op.row_ptr, op.col_ind, Hd[rows, op.col_ind].reshape(-1, 1, 1), 1)
        mu = oracle.kpm_moments(oracle.make_op(to_oracle(A), (emax + emin) / 2,
                                               (emax - emin) / 2), psi, N)
        want = 2.0 * oracle.density(mu, x, 0.5 / nt)
        assert rel_err(dos[q * 2 * nt:(q + 1) * 2 * nt], want) < 1e-10
    est = RSATB(op, SetupOptions(kpoints=kpts))
    lo, hi = est.energy_bounds()
    for k in kpts:
        w = np.linalg.eigvalsh(oracle.bloch_dense(r, c, sh, bl, n, k))
        assert lo < w[0] and hi > w[-1]
    with pytest.raises(ValueError):
        RSATB(lattice.graphene(6, 6)[0], SetupOptions(kpoints=kpts))


@pytest.mark.gpu
@pytest.mark.parametrize("formulation", ["greenwood", "bastin"])
def test_compute_dc_spectrum_kpoints_matches_oracle(formulation):
    """Transport at k-points from images: H(k) and V_a(k) (complex, summed
    on the device) per k-point, one sigma block each (observables.hpp:
    741-772), against the oracle's fftcheb on its own dense Bloch sums."""
    import torch
    from rsatb_b200 import lattice
    from rsatb_b200.bloch import ImageOperator
    from rsatb_b200.driver import RSATB, SetupOptions, _volume
    from rsatb_b200.lattice import BsrArrays
    torch.cuda.set_device(0)
    r, c, sh, bl, bv, n, cell = lattice.graphene_images(6, 5)
    op = ImageOperator(r, c, sh, bl, 1, n, bond_vectors=bv)
    kpts = [[0.0, 0.0, 0.0], [0.2, 0.35, 0.0]]
    emin, emax = -8.7, 8.8
    calc = RSATB(op, SetupOptions(kpoints=kpts, nsamples=2, sample_seed=21,
                                  energy_bounds=(emin, emax)), cell=cell)
    M = 40
    sigma, energy = calc.compute_dc_spectrum(M, formulation=formulation, axis="ab")
    assert sigma.shape == (2 * M * 6,)
    dc = calc.compute_dc(M, 0.3, 300.0, formulation=formulation, axis="ab")
    want_dc = np.concatenate([oracle.integrate_dc_spectrum(sigma[q * M * 6:(q + 1) * M * 6],
                                                           energy, 0.3, 300.0) for q in range(2)])
    assert dc.shape == (12,) and np.abs(dc - want_dc).max() <= 1e-10 * np.abs(want_dc).max()
    psi = _oracle_samples(n, 2, 21)
    rows = np.repeat(np.arange(n), np.diff(op.row_ptr))

    def at(dense, imag=False):
        vals = dense[rows, op.col_ind].reshape(-1, 1, 1)
        return to_oracle(BsrArrays(op.row_ptr, op.col_ind, vals, 1))

    pref = np.pi * 2.0 * (4.0 if formulation == "greenwood" else 8.0) * n / _volume(cell, "ab")
    for q, k in enumerate(kpts):
        Ho = at(oracle.bloch_dense(r, c, sh, bl, n, k))
        Vo = [at(oracle.bloch_dense(r, c, sh, bl, n, k, weights=bv[:, a], imag_unit=True))
              for a in range(3)]
        oop = oracle.make_op(Ho, (emax + emin) / 2, (emax - emin) / 2)
        sig_o, en_o = oracle.fftcheb(oop, Vo, psi, M,
                                     formulation=0 if formulation == "greenwood" else 1,
                                     prefactor=pref)
        assert rel_err(sigma[q * M * 6:(q + 1) * M * 6], sig_o.reshape(-1)) < 1e-10
        assert np.allclose(energy, en_o, rtol=0, atol=1e-13)
    with pytest.raises(ValueError):
        RSATB(op, SetupOptions(kpoints=kpts, energy_bounds=(emin, emax)), cell=cell,
              velocities=(None, None, None))


@pytest.mark.gpu
def test_compute_dos_solve_form():
    """PreconditionerOptions(operator_form='solve'): the DOS of S^-1 H by the
    plain recurrence with a CG per application, against a dense FP64
    recurrence on S^-1 H with the same samples; the estimated window (an
    S-orthonormal Lanczos) holds the generalised spectrum."""
    import torch
    from rsatb_b200 import lattice
    from rsatb_b200.calc import dos_energy_grid, dos_moment_count
    from rsatb_b200.driver import PreconditionerOptions, RSATB, SetupOptions
    torch.cuda.set_device(0)
    H, S = lattice.diamond_lcao(L=2, seed=3)
    Hd, Sd = H.to_dense(), S.to_dense()
    A = np.linalg.solve(Sd, Hd)
    w = np.sort(np.linalg.eigvals(A).real)
    est = RSATB(H, SetupOptions(preconditioner=PreconditionerOptions(cg_tol=1e-12)), S=S)
    lo, hi = est.energy_bounds()
    assert lo < w[0] and hi > w[-1]
    emin, emax = w[0] - 0.5, w[-1] + 0.5
    calc = RSATB(H, SetupOptions(nsamples=2, sample_seed=4, energy_bounds=(emin, emax),
                                 preconditioner=PreconditionerOptions(cg_tol=1e-12)), S=S)
    dE = 0.6
    dos, omega = calc.compute_dos(dE)
    x, _, nt = dos_energy_grid(emin, emax, dE)
    N = dos_moment_count((emax - emin) / 2, dE)
    psi = _oracle_samples(H.n_rows, 2, 4)
    c, hw = (emax + emin) / 2, (emax - emin) / 2
    At = (A - c * np.eye(A.shape[0])) / hw
    t0, t1 = psi, At @ psi
    mu = np.zeros(N, dtype=np.complex128)
    mu[0] = np.sum(psi.conj() * t0) / 2
    mu[1] = np.sum(psi.conj() * t1) / 2
    for n in range(2, N):
        t0, t1 = t1, 2 * At @ t1 - t0
        mu[n] = np.sum(psi.conj() * t1) / 2
    want = 2.0 * oracle.density(mu, x, 0.5 / nt)
    assert rel_err(dos, want) < 1e-8
    with pytest.raises(ValueError):
        PreconditionerOptions(operator_form="cg") and RSATB(
            H, SetupOptions(preconditioner=PreconditionerOptions(operator_form="cg"),
                            energy_bounds=(emin, emax)))



@pytest.mark.gpu
def test_sandwich_factor_built_from_overlap():
    """operator_form='sandwich' given S (and no Z) builds Z as the
    reference's build_preconditioner does: the graph-local seed, then
    maxiter Newton-Schulz steps on the device.  maxiter = 0 is the seed: the
    DOS equals the one with the seed passed in as Z.  With maxiter > 0 the
    refined factor's congruence Z^T S Z is closer to the identity."""
    import torch
    from rsatb_b200 import lattice
    from rsatb_b200.driver import PreconditionerOptions, RSATB, SetupOptions
    from rsatb_b200.isqrt import graph_inverse_sqrt
    torch.cuda.set_device(0)
    H, S = lattice.diamond_lcao(L=2, seed=3)
    Sd = S.to_dense()

    def opts(maxiter):
        return SetupOptions(nsamples=2, sample_seed=4, energy_bounds=(-12.0, 12.0),
                            preconditioner=PreconditionerOptions(operator_form="sandwich",
                                                                 maxiter=maxiter, tol=1e-9,
                                                                 sptol=1e-9))

    seeded = RSATB(H, opts(0), S=S)
    assert seeded.factor_report.steps == 0 and seeded.S is None
    given = RSATB(H, opts(0), Z=graph_inverse_sqrt(S))
    d0, _ = seeded.compute_dos(0.8)
    d1, _ = given.compute_dos(0.8)
    assert rel_err(d0, d1) < 1e-12
    refined = RSATB(H, opts(3), S=S)
    assert 1 <= refined.factor_report.steps <= 3

    def congruence(Zm):
        Zd = Zm.to_arrays().to_dense()
        return np.abs(Zd.T @ Sd @ Zd - np.eye(Sd.shape[0])).max()

    assert congruence(refined.Z) < 0.1 * congruence(seeded.Z)


@pytest.mark.gpu
def test_converging_bounds_follow_the_reference_contract():
    """estimate_spectral_bounds with tol (the facade's mode): Lanczos until
    both extreme Ritz pairs reach residual 1e-3 of the spectral scale, the
    0.5 eV padding outside; a zero operator gives (-0.5, 0.5); a solve that
    cannot converge within max_matvecs falls back to +-||H||_F (orthogonal)
    or raises (sandwich), as ExtremalEigenvalues does
    (rsatb/setup/spectral_bounds.hpp:311-400)."""
    import torch
    from rsatb_b200 import lattice
    from rsatb_b200.bounds import estimate_spectral_bounds
    from rsatb_b200.calc import Chebyshev, ISQRTMPreconditioner
    from rsatb_b200.isqrt import graph_inverse_sqrt
    from rsatb_b200.vbcsr import BlockSpMat
    torch.cuda.set_device(0)
    H, _, _ = lattice.graphene(20, 20)
    w = np.linalg.eigvalsh(H.to_dense())
    A = BlockSpMat(H.row_ptr, H.col_ind, H.values, 1)
    info = {}
    lo, hi = estimate_spectral_bounds(Chebyshev(A, -1, 1), tol=1e-3, zero_tol=1e-12, info=info)
    assert info["converged"] and info["matvecs"] < 400
    assert lo < w[0] and hi > w[-1] and w[0] - lo < 0.6 and hi - w[-1] < 0.6
    Z0 = BlockSpMat(H.row_ptr, H.col_ind, 0.0 * H.values, 1)
    assert estimate_spectral_bounds(Chebyshev(Z0, -1, 1), tol=1e-3, zero_tol=1e-12) == (-0.5, 0.5)
    fro = float(np.sqrt((H.values ** 2).sum()))
    lo, hi = estimate_spectral_bounds(Chebyshev(A, -1, 1), tol=1e-3, max_matvecs=2)
    assert abs(lo + fro + 0.5) < 1e-9 and abs(hi - fro - 0.5) < 1e-9
    Hd, S = lattice.diamond_lcao(L=2, seed=3)
    Z = graph_inverse_sqrt(S)
    c = Chebyshev(BlockSpMat(Hd.row_ptr, Hd.col_ind, Hd.values, 8), -1, 1,
                  preconditioner=ISQRTMPreconditioner(BlockSpMat(Z.row_ptr, Z.col_ind, Z.values, 8)))
    with pytest.raises(RuntimeError, match="max_matvecs"):
        estimate_spectral_bounds(c, tol=1e-3, max_matvecs=2)
