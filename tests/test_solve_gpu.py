"""The Solve operator form S^-1 H: the batched CG (rsatb_cg_solve,
LinearSolver::solve for a multivector, rsatb/calc/solver.hpp:216-312), the
operator application (Chebyshev::apply_form's Solve branch,
rsatb/calc/cheby.hpp:569-590) and the plain KPM recurrence over it
(dos.hpp:172-187), against dense FP64 solves and the oracle's dense
recurrence."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from _util import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    torch.cuda.set_device(0)
    return torch


@pytest.fixture(scope="module")
def diamond():
    from rsatb_b200 import lattice
    H, S = lattice.diamond_lcao(L=2, seed=3)
    Hd, Sd = H.to_dense(), S.to_dense()
    assert np.linalg.eigvalsh(Sd)[0] > 0.05
    w = np.linalg.eigvals(np.linalg.solve(Sd, Hd)).real
    return H, S, Hd, Sd, w.min() - 0.5, w.max() + 0.5


def _dev(A, precision="f64"):
    from rsatb_b200.vbcsr import BlockSpMat
    M = BlockSpMat(A.row_ptr, A.col_ind, A.values, A.block_size)
    return M.astype("f32") if precision == "f32" else M


@pytest.mark.parametrize("cplx,precision", [(False, "f64"), (True, "f64"), (False, "f32")])
def test_cg_solve_matches_dense(torch_cuda, diamond, cplx, precision):
    torch = torch_cuda
    from rsatb_b200.calc import cg_solve
    H, S, Hd, Sd, _, _ = diamond
    rng = np.random.default_rng(5)
    n, R = Sd.shape[0], (3 if cplx else 5)
    B = rng.standard_normal((n, R))
    if cplx:
        B = B + 1j * rng.standard_normal((n, R))
    B[:, 1] = 0.0   # a zero right-hand side freezes at once (no 0/0)
    dt = {(False, "f64"): torch.float64, (True, "f64"): torch.complex128,
          (False, "f32"): torch.float32}[(cplx, precision)]
    Bd = torch.as_tensor(B).to(dt).cuda().contiguous()
    Xd = torch.zeros_like(Bd)
    tol = 1e-12 if precision == "f64" else 1e-4
    it, res = cg_solve(_dev(S, precision), Bd, Xd, tol=tol, max_iter=500)
    want = np.linalg.solve(Sd, B)
    got = Xd.cpu().numpy()
    assert res < tol and 0 < it < 500
    assert rel_err(got, want) < (1e-10 if precision == "f64" else 1e-4)
    assert np.all(got[:, 1] == 0)
    # started from the solution, the CG stops after one iteration
    it2, res2 = cg_solve(_dev(S, precision), Bd, Xd, tol=max(tol, 10 * res), max_iter=500)
    assert it2 == 1


def test_solve_form_apply_matches_dense(torch_cuda, diamond):
    torch = torch_cuda
    from rsatb_b200.calc import Chebyshev
    H, S, Hd, Sd, emin, emax = diamond
    c = Chebyshev(_dev(H), emin, emax, overlap=_dev(S), cg_tol=1e-12)
    rng = np.random.default_rng(2)
    X = rng.standard_normal((Hd.shape[0], 4)) + 1j * rng.standard_normal((Hd.shape[0], 4))
    Xd = torch.as_tensor(X).cuda().contiguous()
    Yd = torch.zeros_like(Xd)
    c.apply_op(Xd, Yd)
    cen, hw = (emax + emin) / 2, (emax - emin) / 2
    want = (np.linalg.solve(Sd, Hd @ X) - cen * X) / hw
    assert rel_err(Yd.cpu().numpy(), want) < 1e-10


@pytest.mark.parametrize("cg_tol,tol", [(1e-12, 1e-9), (1e-8, 1e-5)])
def test_solve_form_moments_match_oracle(torch_cuda, diamond, cg_tol, tol):
    """Plain moments of S^-1 H (op_is_hermitian() is false for this form)
    against the oracle's dense recurrence on S^-1 H."""
    torch = torch_cuda
    from rsatb_b200.calc import Chebyshev, kpm_dos_moments
    from rsatb_b200.vbcsr import set_random
    H, S, Hd, Sd, emin, emax = diamond
    c = Chebyshev(_dev(H), emin, emax, overlap=_dev(S), cg_tol=cg_tol)
    assert not c.op_is_hermitian()
    psi = torch.empty(Hd.shape[0], 4, dtype=torch.float64, device="cuda")
    set_random(psi, 9)
    mu = kpm_dos_moments(c, psi, 40)
    want = oracle.kpm_plain_moments_dense(np.linalg.solve(Sd, Hd), psi.cpu().numpy(),
                                          (emax + emin) / 2, (emax - emin) / 2, 40)
    assert np.abs(mu.real - want).max() < tol * abs(want[0])
    assert np.abs(mu.imag).max() == 0.0


def test_solve_form_refuses_doubling(torch_cuda, diamond):
    torch = torch_cuda
    from rsatb_b200._capi import RsatbError
    from rsatb_b200.calc import Chebyshev, _moments
    H, S, Hd, Sd, emin, emax = diamond
    c = Chebyshev(_dev(H), emin, emax, overlap=_dev(S))
    psi = torch.ones(Hd.shape[0], 2, dtype=torch.float64, device="cuda")
    with pytest.raises(RsatbError):
        _moments(c, psi, 8, doubled=True)


def _factor(S):
    from rsatb_b200.calc import ISQRTMPreconditioner
    from rsatb_b200.isqrt import graph_inverse_sqrt_host
    return ISQRTMPreconditioner(_dev(graph_inverse_sqrt_host(S)))


def test_preconditioned_cg_matches_dense(torch_cuda, diamond):
    """Symmetric preconditioning by the graph-local factor Z
    (solver.hpp:329-338): Z^H S Z Y = Z^H B from Y = 0, X = Z Y; the same
    solution as the dense solve in fewer iterations than the plain CG."""
    torch = torch_cuda
    from rsatb_b200.calc import cg_solve
    H, S, Hd, Sd, _, _ = diamond
    rng = np.random.default_rng(8)
    B = rng.standard_normal((Sd.shape[0], 6))
    Bd = torch.as_tensor(B).cuda().contiguous()
    X0 = torch.zeros_like(Bd)
    it0, _ = cg_solve(_dev(S), Bd, X0, tol=1e-12, max_iter=500)
    X1 = torch.full_like(Bd, 7.0)   # ignored: the preconditioned solve starts from Y = 0
    it1, res1 = cg_solve(_dev(S), Bd, X1, tol=1e-12, max_iter=500, preconditioner=_factor(S))
    want = np.linalg.solve(Sd, B)
    assert res1 < 1e-12 and it1 < it0
    assert rel_err(X1.cpu().numpy(), want) < 1e-10


def test_preconditioned_solve_form_moments(torch_cuda, diamond):
    torch = torch_cuda
    from rsatb_b200.calc import Chebyshev, kpm_dos_moments
    from rsatb_b200.vbcsr import set_random
    H, S, Hd, Sd, emin, emax = diamond
    c = Chebyshev(_dev(H), emin, emax, overlap=_dev(S), preconditioner=_factor(S), cg_tol=1e-12)
    assert c.form.name == "Solve"
    psi = torch.empty(Hd.shape[0], 3, dtype=torch.float64, device="cuda")
    set_random(psi, 12)
    mu = kpm_dos_moments(c, psi, 32)
    want = oracle.kpm_plain_moments_dense(np.linalg.solve(Sd, Hd), psi.cpu().numpy(),
                                          (emax + emin) / 2, (emax - emin) / 2, 32)
    assert np.abs(mu.real - want).max() < 1e-9 * abs(want[0])



@pytest.mark.parametrize("preconditioned", [False, True])
def test_solve_form_apply_dual_and_propagate(torch_cuda, diamond, preconditioned):
    """Chebyshev::apply_dual for the Solve form: scale S^-1 V X (NORMAL)
    and scale V S^-1 X (ADJOINT); propagate: sum_n c_n T_n(Op~) X with
    Op~ = (S^-1 H - c) / hw and complex coefficients, one CG per
    application; against dense FP64 solves, with the plain and the
    Z-preconditioned CG (CG tolerance 1e-12)."""
    torch = torch_cuda
    from rsatb_b200.calc import ChebyMode, Chebyshev, ISQRTMPreconditioner
    from rsatb_b200.isqrt import graph_inverse_sqrt
    from rsatb_b200.lattice import BsrArrays
    H, S, Hd, Sd, emin, emax = diamond
    rng = np.random.default_rng(6)
    v = rng.standard_normal(H.values.shape)
    Vd = BsrArrays(H.row_ptr, H.col_ind, v, 8).to_dense()
    Vd = 0.5 * (Vd + Vd.T)
    rows = np.repeat(np.arange(H.n_block_rows), np.diff(H.row_ptr))
    vv = np.stack([Vd[i * 8:(i + 1) * 8, j * 8:(j + 1) * 8] for i, j in zip(rows, H.col_ind)])
    V = _dev(BsrArrays(H.row_ptr, H.col_ind, vv, 8))
    pre = None
    if preconditioned:
        Z = graph_inverse_sqrt(S)
        pre = ISQRTMPreconditioner(_dev(Z))
    c = Chebyshev(_dev(H), emin, emax, preconditioner=pre, overlap=_dev(S), cg_tol=1e-12)
    X = rng.standard_normal((H.n_rows, 4))
    Xd = torch.as_tensor(X).cuda()
    Y = torch.zeros_like(Xd)
    c.apply_dual(V, Xd, Y, scale=0.7)
    assert rel_err(Y.cpu().numpy(), 0.7 * np.linalg.solve(Sd, Vd @ X)) < 1e-9
    Y.zero_()
    c.apply_dual(V, Xd, Y, mode=ChebyMode.ADJOINT, scale=0.7)
    assert rel_err(Y.cpu().numpy(), 0.7 * Vd @ np.linalg.solve(Sd, X)) < 1e-9
    coeffs = np.array([0.3 - 0.1j, -0.2 + 0.4j, 0.15, 0.05j, -0.07 + 0.02j])
    Xc = (X + 1j * rng.standard_normal(X.shape)).astype(np.complex128)
    Pc = torch.as_tensor(Xc).cuda()
    out = torch.zeros_like(Pc)
    c.propagate(Pc, out, coeffs)
    cen, hw = (emax + emin) / 2, (emax - emin) / 2
    At = (np.linalg.solve(Sd, Hd) - cen * np.eye(Hd.shape[0])) / hw
    t0, t1 = Xc, At @ Xc
    want = coeffs[0] * t0 + coeffs[1] * t1
    for n in range(2, coeffs.size):
        t0, t1 = t1, 2 * At @ t1 - t0
        want = want + coeffs[n] * t1
    assert rel_err(out.cpu().numpy(), want) < 1e-8
    with pytest.raises(NotImplementedError):
        c.propagate(Pc, out, coeffs, mode=ChebyMode.ADJOINT)
