"""FFT-Chebyshev Kubo-Greenwood transport (rsatb_dc_spectrum_fftcheb)
against the oracle's restatement of dc_spectrum_fftcheb
(rsatb/calc/fftcheb_transport.hpp:270-660), itself pinned to the reference's
O(M^2) moment reference and DCT-III checks (tests/test_oracle_golden.py)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from _util import adjoint_arrays, rel_err, to_oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    torch.cuda.set_device(0)
    return torch


def _dev(A, imaginary=False, precision="f64"):
    from rsatb_b200.vbcsr import BlockSpMat
    M = BlockSpMat(A.row_ptr, A.col_ind, A.values, A.block_size, A.n_block_cols,
                   imaginary=imaginary)
    return M.astype("f32") if precision == "f32" else M


def _tbg(m=1, tiles=(4, 4)):
    from rsatb_b200 import lattice
    H, pos, cell, disp = lattice.twisted_bilayer_graphene(m=m, tiles=tiles)
    V = lattice.commutator_velocity(H, disp)
    return H, V


def _phases(n, R, seed=5):
    rng = np.random.default_rng(seed)
    return np.exp(2j * np.pi * rng.random((n, R))) / np.sqrt(n)


def _bounds(H):
    w = np.linalg.eigvalsh(H.to_dense())
    return w[0] - 0.5, w[-1] + 0.5


def _gpu(torch, H, V, psi, M, emin, emax, precision="f64", Z=None, **kw):
    from rsatb_b200.calc import Chebyshev, ISQRTMPreconditioner
    from rsatb_b200.transport import dc_spectrum_fftcheb
    pre = ISQRTMPreconditioner(_dev(Z)) if Z is not None else None
    c = Chebyshev(_dev(H), emin, emax, preconditioner=pre)
    Vd = [_dev(v, imaginary=True) for v in V]
    dt = torch.complex128
    if precision == "f32":
        c = c.astype("f32")
        Vd = [v.astype("f32") for v in Vd]
        dt = torch.complex64
    p = torch.as_tensor(psi).cuda().to(dt).contiguous()
    return dc_spectrum_fftcheb(c, *Vd, p, M, return_stats=True, **kw)


def _oracle(H, V, psi, M, emin, emax, Z=None, sections=1, formulation=0):
    c, hw = (emax + emin) / 2, (emax - emin) / 2
    if Z is None:
        op = oracle.make_op(to_oracle(H), c, hw)
    else:
        op = oracle.make_op(to_oracle(H), c, hw, to_oracle(Z), to_oracle(adjoint_arrays(Z)))
    Vo = [to_oracle(v, imag=True) for v in V]
    return oracle.fftcheb(op, Vo, psi, M, formulation=formulation, prefactor=1.0,
                          sections=sections)


@pytest.mark.parametrize("M", [1, 2, 17, 64])
def test_greenwood_matches_oracle_tbg(torch_cuda, M):
    H, V = _tbg()
    emin, emax = _bounds(H)
    psi = _phases(H.n_rows, 3)
    (sig, en, st) = _gpu(torch_cuda, H, V, psi, M, emin, emax)
    sig_o, en_o = _oracle(H, V, psi, M, emin, emax)
    assert np.allclose(en, en_o, rtol=0, atol=1e-13)
    assert rel_err(sig, sig_o) < 1e-10
    assert np.all(sig[:, [1, 2, 4]] == 0.0)   # Greenwood fills the diagonal only


def test_sections_and_workspace_do_not_change_sigma(torch_cuda):
    H, V = _tbg()
    emin, emax = _bounds(H)
    psi = _phases(H.n_rows, 2, seed=9)
    s1, _, st1 = _gpu(torch_cuda, H, V, psi, 40, emin, emax)
    s3, _, st3 = _gpu(torch_cuda, H, V, psi, 40, emin, emax, partition_sections=3)
    s_small, _, st_s = _gpu(torch_cuda, H, V, psi, 40, emin, emax, max_workspace_mb=6.0)
    assert st1["sections"] == 1 and st3["sections"] >= 3 and st_s["fft_chunks"] > 1
    assert rel_err(s3, s1) < 1e-12 and rel_err(s_small, s1) < 1e-12


def test_fp32_vectors_against_fp64(torch_cuda):
    """FP32 vectors and matrices, FP64 transform and contraction."""
    H, V = _tbg()
    emin, emax = _bounds(H)
    psi = _phases(H.n_rows, 4, seed=3)
    s64, _, _ = _gpu(torch_cuda, H, V, psi, 64, emin, emax)
    s32, _, _ = _gpu(torch_cuda, H, V, psi, 64, emin, emax, precision="f32")
    assert rel_err(s32, s64) < 1e-4


def test_sandwich_form_matches_oracle(torch_cuda):
    """Non-orthogonal sandwich Z^H H Z with dressed currents Z^H V Z."""
    from rsatb_b200 import lattice
    H, V = _tbg(m=1, tiles=(3, 3))
    # S = I + 0.015 |H|: SPD and non-orthogonal; Z = S^-1/2 as a dense BSR
    n = H.n_rows
    Sd = np.eye(n) + 0.015 * np.abs(H.to_dense())
    w, Q = np.linalg.eigh(Sd)
    Zfull = (Q / np.sqrt(w)) @ Q.T
    rp = (np.arange(n + 1) * n).astype(np.int32)
    ci = np.tile(np.arange(n), n).astype(np.int32)
    Z = lattice.BsrArrays(rp, ci, Zfull.reshape(-1, 1, 1), 1)
    Zd = Z.to_dense()
    Hs = Zd.T @ H.to_dense() @ Zd
    w = np.linalg.eigvalsh(0.5 * (Hs + Hs.T))
    emin, emax = w[0] - 0.5, w[-1] + 0.5
    psi = _phases(H.n_rows, 2, seed=4)
    sig, _, _ = _gpu(torch_cuda, H, V, psi, 24, emin, emax, Z=Z)
    sig_o, _ = _oracle(H, V, psi, 24, emin, emax, Z=Z)
    assert rel_err(sig, sig_o) < 1e-10


def test_graphene_is_isotropic_in_plane(torch_cuda):
    from rsatb_b200 import lattice
    H, pos, cell = lattice.graphene(12, 12)
    d = lattice.graphene_displacements(H, pos, cell)
    V = lattice.commutator_velocity(H, d)
    psi = _phases(H.n_rows, 8, seed=1)
    sig, en, _ = _gpu(torch_cuda, H, V, psi, 64, -9.2, 9.2)
    xx, yy, zz = sig[:, 0], sig[:, 3], sig[:, 5]
    assert np.abs(zz).max() == 0.0
    assert xx.max() > 0
    assert rel_err(yy, xx) < 0.3   # stochastic trace with 8 samples


@pytest.mark.parametrize("M", [1, 2, 17, 48])
def test_bastin_matches_oracle_tbg(torch_cuda, M):
    """Bastin: phi1, phi2 (zero-padded inverse FFTs with the complex phase
    weights) beside phi3, all six tensor components, then the cumulative
    energy integral (fftcheb_transport.hpp:443-519, 635-659)."""
    H, V = _tbg()
    emin, emax = _bounds(H)
    psi = _phases(H.n_rows, 3, seed=7)
    sig, en, _ = _gpu(torch_cuda, H, V, psi, M, emin, emax, formulation=1)
    sig_o, en_o = _oracle(H, V, psi, M, emin, emax, formulation=1)
    assert np.allclose(en, en_o, rtol=0, atol=1e-13)
    assert rel_err(sig, sig_o) < 1e-10


def test_bastin_sections_and_fp32(torch_cuda):
    H, V = _tbg()
    emin, emax = _bounds(H)
    psi = _phases(H.n_rows, 2, seed=2)
    s1, _, _ = _gpu(torch_cuda, H, V, psi, 32, emin, emax, formulation=1)
    s3, _, st3 = _gpu(torch_cuda, H, V, psi, 32, emin, emax, formulation=1,
                      partition_sections=3, max_workspace_mb=6.0)
    s32, _, _ = _gpu(torch_cuda, H, V, psi, 32, emin, emax, formulation=1, precision="f32")
    assert st3["sections"] >= 3
    assert rel_err(s3, s1) < 1e-12
    assert rel_err(s32, s1) < 1e-4


def test_bad_arguments_refused(torch_cuda):
    from rsatb_b200._capi import RsatbError
    from rsatb_b200.calc import Chebyshev
    from rsatb_b200.transport import dc_spectrum_fftcheb
    H, V = _tbg()
    c = Chebyshev(_dev(H), -10, 10)
    Vd = [_dev(v, imaginary=True) for v in V]
    p = torch_cuda.as_tensor(_phases(H.n_rows, 1)).cuda()
    with pytest.raises(ValueError):
        dc_spectrum_fftcheb(c, *Vd, p, 8, formulation=2)
    with pytest.raises(RsatbError):   # FP32 vectors with FP64 matrices
        dc_spectrum_fftcheb(c, *Vd, p.to(torch_cuda.complex64), 8)


@pytest.mark.parametrize("temp", [0.0, 1e-3, 77.0, 300.0, 5000.0])
def test_integrate_dc_spectrum_matches_oracle(torch_cuda, temp):
    """sigma(mu, T) from a spectrum (fftcheb_transport.hpp:950-1040) on the
    device against the oracle's restatement, for mu inside, between and
    outside the grid."""
    from rsatb_b200.transport import integrate_dc_spectrum
    rng = np.random.default_rng(3)
    e = np.sort(rng.uniform(-6.0, 6.0, 300))
    s = rng.standard_normal((300, 6))
    for mu in (-7.0, e[10], 0.123, 6.5):
        got = integrate_dc_spectrum(s, e, mu, temp)
        want = oracle.integrate_dc_spectrum(s, e, mu, temp)
        # The interval moment F(e1) - F(e0) - f(e1) de cancels to a small
        # difference of O(|E|) terms, and random spectra (no smoothness)
        # divide it by de: 1e-10 of the O(1) spectrum values.
        assert np.abs(got - want).max() <= 1e-10 * np.abs(s).max()
    if temp > 0:
        with pytest.raises(Exception):
            integrate_dc_spectrum(s, e[::-1].copy(), 0.0, temp)


# ------------------------------------------------------------------ QE route

@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_qe_route_matches_oracle_and_fftcheb(torch_cuda, precision):
    """dc_spectrum_qe on a window of nodes: the oracle's dense restatement
    of accumulate_qe_block (1e-10 of the window's peak in FP64, 1e-4 with
    FP32 vectors) and the fftcheb Greenwood route on the same nodes, which
    is the same bilinear form (the reference's note: they agree to
    rounding); zero outside the window."""
    torch = torch_cuda
    from rsatb_b200.calc import Chebyshev
    from rsatb_b200.transport import dc_spectrum_fftcheb, dc_spectrum_qe
    H, V = _tbg()
    emin, emax = _bounds(H)
    M, R = 64, 3
    psi = _phases(H.n_rows, R, seed=8)
    nodes = np.arange(20, 34)
    c = Chebyshev(_dev(H), emin, emax)
    Vd = [_dev(v, imaginary=True) for v in V]
    dt = torch.complex128
    if precision == "f32":
        c, Vd, dt = c.astype("f32"), [v.astype("f32") for v in Vd], torch.complex64
    p = torch.as_tensor(psi).cuda().to(dt).contiguous()
    sig, en = dc_spectrum_qe(c, *Vd, p, M, nodes_ascending=nodes)
    Vo = [1j * v.to_dense() for v in V]
    want, en_o = oracle.qe_dense(H.to_dense(), Vo, psi, (emax + emin) / 2, (emax - emin) / 2, M,
                                 nodes)
    assert np.abs(en - en_o).max() < 1e-12
    tol = 1e-10 if precision == "f64" else 1e-4
    assert rel_err(sig, want) < tol
    outside = np.setdiff1d(np.arange(M), nodes)
    assert np.all(sig[outside] == 0.0)
    if precision == "f64":
        full, _ = dc_spectrum_fftcheb(c, *Vd, p, M)
        assert rel_err(sig[nodes], full[nodes]) < 1e-10
        every, _ = dc_spectrum_qe(c, *Vd, p, M)
        assert rel_err(every, full) < 1e-10


def test_qe_route_sandwich_and_errors(torch_cuda):
    """The sandwich form through the QE route equals the fftcheb route;
    a node outside the grid is refused."""
    torch = torch_cuda
    from rsatb_b200._capi import RsatbError
    from rsatb_b200.calc import Chebyshev, ISQRTMPreconditioner
    from rsatb_b200.transport import dc_spectrum_fftcheb, dc_spectrum_qe
    H, V = _tbg()
    emin, emax = _bounds(H)
    n = H.n_rows
    rng = np.random.default_rng(2)
    Zd = np.eye(n) + 0.01 * rng.standard_normal((n, n))
    mask = np.abs(H.to_dense()) > 0
    np.fill_diagonal(mask, True)
    Zd = np.where(mask, Zd, 0.0)
    from rsatb_b200.lattice import BsrArrays
    rows, cols = np.nonzero(Zd)
    rp = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=n))]).astype(np.int32)
    Z = BsrArrays(rp, cols.astype(np.int32), Zd[rows, cols].reshape(-1, 1, 1).copy(), 1)
    c = Chebyshev(_dev(H), emin - 1.0, emax + 1.0, preconditioner=ISQRTMPreconditioner(_dev(Z)))
    Vd = [_dev(v, imaginary=True) for v in V]
    p = torch.as_tensor(_phases(n, 2, seed=3)).cuda().contiguous()
    M = 48
    full, _ = dc_spectrum_fftcheb(c, *Vd, p, M)
    nodes = np.array([5, 17, 30, 47])
    sig, _ = dc_spectrum_qe(c, *Vd, p, M, nodes_ascending=nodes)
    assert rel_err(sig[nodes], full[nodes]) < 1e-10
    with pytest.raises(RsatbError, match="out of range"):
        dc_spectrum_qe(c, *Vd, p, M, nodes_ascending=[0, M])


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_fused_row_stage_at_2048_moments(torch_cuda, precision, monkeypatch):
    """M = 2048 takes the fused Greenwood row stage (extension, 4096-point
    DCT-III and contraction in one kernel): equal to the chunked cuFFT row
    stage on the same stores, over one section and three, and to the oracle.
    FP32 vectors take the FP32 transform (FP64 products and sums): within
    1e-6 of the FP64 transform of the same stores, which equals cuFFT's."""
    H, V = _tbg()
    emin, emax = _bounds(H)
    psi = _phases(H.n_rows, 2, seed=13)
    fused, en, st = _gpu(torch_cuda, H, V, psi, 2048, emin, emax, precision=precision)
    fused3, _, st3 = _gpu(torch_cuda, H, V, psi, 2048, emin, emax, precision=precision,
                          partition_sections=3)
    # gathered chunks of 100 sequence pairs: nine per axis
    monkeypatch.setenv("RSATB_FFTCHEB_CHUNK", "100")
    small, _, st_s = _gpu(torch_cuda, H, V, psi, 2048, emin, emax, precision=precision)
    monkeypatch.delenv("RSATB_FFTCHEB_CHUNK")
    monkeypatch.setenv("RSATB_FFTCHEB_FP64", "1")
    fused64, _, _ = _gpu(torch_cuda, H, V, psi, 2048, emin, emax, precision=precision)
    monkeypatch.setenv("RSATB_FFTCHEB_FUSED", "0")
    chunked, _, st_c = _gpu(torch_cuda, H, V, psi, 2048, emin, emax, precision=precision)
    # one gathered chunk per axis and section
    assert st["fft_chunks"] == 3 and st3["sections"] >= 3 and st_c["fft_chunks"] >= 1
    assert rel_err(fused64, chunked) < 1e-12
    assert rel_err(fused, chunked) < (1e-12 if precision == "f64" else 1e-6)
    assert rel_err(fused3, fused) < 1e-12
    assert st_s["fft_chunks"] == 27 and rel_err(small, fused) < 1e-12
    assert np.all(fused[:, [1, 2, 4]] == 0.0)
    if precision == "f64":
        sig_o, en_o = _oracle(H, V, psi, 2048, emin, emax)
        assert np.allclose(en, en_o, rtol=0, atol=1e-13)
        assert rel_err(fused, sig_o) < 1e-10
