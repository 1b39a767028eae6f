"""The step kernel's default dispatch over a grid of shapes: block sizes 1,
2, 3, 5, 8; real, complex and imaginary-unit matrices; real and complex
panels of 1 to 64 columns; FP64 and FP32.  Every case runs the SpMM
(rsatb_bsr_mult_dense) against the oracle's SpMM and the doubled KPM
recurrence (rsatb_kpm_dos_moments, whose step kernels carry the fused dots)
against the oracle's moments (Hermitian matrices).  The point is the launch
path itself: each shape reaches one kernel family and launch configuration
(mapping, shared memory opt-in, grid), and a shape no other test reaches
must still launch and agree."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from _util import random_hermitian_bsr, rel_err, to_oracle

pytestmark = pytest.mark.gpu

WIDTHS = [1, 2, 3, 4, 5, 7, 8, 12, 16, 24, 32, 40, 64]
KINDS = [("real", False, False, False), ("complex", True, False, True),
         ("imaginary", False, True, True), ("real_cplx_panel", False, False, True)]


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    torch.cuda.set_device(0)
    return torch


def _dtype(torch, precision, cv):
    return {("f64", True): torch.complex128, ("f64", False): torch.float64,
            ("f32", True): torch.complex64, ("f32", False): torch.float32}[(precision, cv)]


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("kind", KINDS, ids=[k[0] for k in KINDS])
@pytest.mark.parametrize("b", [1, 2, 3, 5, 8])
def test_default_dispatch_sweep(torch_cuda, b, kind, precision):
    torch = torch_cuda
    from rsatb_b200.calc import Chebyshev, kpm_dos_moments
    from rsatb_b200.vbcsr import BlockSpMat
    _, cm, imag, cv = kind
    n = 37
    A = random_hermitian_bsr(n, b, 4, seed=100 + b, complex_values=cm, scale=0.3)
    if imag:
        A = A.with_values(A.values.real.copy())
    Ao = to_oracle(A, imag=imag)
    Ad = BlockSpMat(A.row_ptr, A.col_ind, A.values, b, A.n_block_cols, imaginary=imag)
    if precision == "f32":
        Ad = Ad.astype("f32")
    # i W of a symmetric W is anti-Hermitian: it is swept through the SpMM
    # only (velocity matrices never enter the recurrence as the operator).
    bound = 1.0 if imag else np.abs(np.linalg.eigvalsh(A.to_dense())).max() + 0.5
    c = Chebyshev(Ad, -bound, bound)
    op = oracle.make_op(Ao, 0.0, bound)
    rng = np.random.default_rng(b * 17 + len(kind[0]))
    tol_mv = 1e-13 if precision == "f64" else 2e-5
    tol_mu = 1e-10 if precision == "f64" else 2e-5
    failures = []
    for R in WIDTHS:
        X = rng.standard_normal((n * b, R))
        if cv:
            X = X + 1j * rng.standard_normal((n * b, R))
        Xd = torch.as_tensor(X).cuda().to(_dtype(torch, precision, cv)).contiguous()
        Yd = torch.empty_like(Xd)
        Ad.mult_dense(Xd, Yd, alpha=0.5)
        err = rel_err(Yd.cpu().numpy(), oracle.spmm(Ao, X, alpha=0.5))
        if not err < tol_mv:
            failures.append(("spmm", R, err))
        if imag:
            continue
        Xq = Xd.to(torch.complex128 if cv else torch.float64).cpu().numpy()
        mu = kpm_dos_moments(c, Xd, 10)
        want = oracle.kpm_moments(op, Xq, 10)
        err = np.abs(mu - want).max() / abs(want[0])
        if not err < tol_mu:
            failures.append(("moments", R, err))
    assert not failures, failures


@pytest.mark.parametrize("cm", [False, True], ids=["real", "complex"])
@pytest.mark.parametrize("b", [1, 3, 8])
def test_cg_solve_sweep(torch_cuda, b, cm):
    """The batched CG (rsatb_cg_solve: the fused S P + <p|Sp>, the update with
    alpha and the new residual, the direction) over column counts that do
    and do not divide the 256 threads of its dot CTAs (1, 3, 8, 17, 64),
    real and complex Hermitian S, against the dense solve to 1e-9."""
    torch = torch_cuda
    from rsatb_b200.calc import cg_solve
    from rsatb_b200.vbcsr import BlockSpMat
    n = 29
    A = random_hermitian_bsr(n, b, 3, seed=7 + b, complex_values=cm, scale=0.2)
    w = np.linalg.eigvalsh(A.to_dense())
    shift = 1.0 - w[0]  # S = A + shift I, smallest eigenvalue 1
    vals = A.values.copy()
    for i in range(n):
        for k in range(A.row_ptr[i], A.row_ptr[i + 1]):
            if A.col_ind[k] == i:
                vals[k] += shift * np.eye(b)
    S = A.with_values(vals)
    Sd = BlockSpMat(S.row_ptr, S.col_ind, S.values, b)
    dense = S.to_dense()
    rng = np.random.default_rng(b)
    dt = torch.complex128 if cm else torch.float64
    for R in (1, 3, 8, 17, 64):
        Bh = rng.standard_normal((n * b, R))
        if cm:
            Bh = Bh + 1j * rng.standard_normal((n * b, R))
        B = torch.as_tensor(Bh).cuda().to(dt).contiguous()
        X = torch.zeros_like(B)
        it, res = cg_solve(Sd, B, X, tol=1e-12, max_iter=500)
        want = np.linalg.solve(dense, Bh)
        assert rel_err(X.cpu().numpy(), want) < 1e-9, (R, it, res)


def _antisymmetric(A):
    """Real W with W^T = -W on A's (symmetric) pattern: V = i W is Hermitian."""
    vals = np.zeros_like(A.values, dtype=np.float64)
    rows = np.repeat(np.arange(A.n_block_rows), np.diff(A.row_ptr))
    index = {(int(i), int(j)): k for k, (i, j) in enumerate(zip(rows, A.col_ind))}
    for (i, j), k in index.items():
        blk = A.values[k].real
        if i == j:
            vals[k] = 0.5 * (blk - blk.T)
        elif i < j:
            vals[k] = blk
            vals[index[(j, i)]] = -blk.T
    return A.with_values(vals)


@pytest.mark.parametrize("b", [1, 2, 5])
def test_fftcheb_sweep(torch_cuda, b):
    """rsatb_dc_spectrum_fftcheb (Greenwood and Bastin) for block sizes 1, 2,
    5 and sample counts 1, 2, 5 (left panels of 2R, right panels of 6R real
    values) against the oracle's dc_spectrum_fftcheb to 1e-10."""
    torch = torch_cuda
    from rsatb_b200.calc import Chebyshev
    from rsatb_b200.transport import dc_spectrum_fftcheb
    from rsatb_b200.vbcsr import BlockSpMat
    n = 23
    H = random_hermitian_bsr(n, b, 3, seed=31 + b, complex_values=False, scale=0.4)
    Ws = [_antisymmetric(random_hermitian_bsr(n, b, 3, seed=31 + b, complex_values=False,
                                              scale=0.2 + 0.1 * a)) for a in range(3)]
    w = np.linalg.eigvalsh(H.to_dense())
    emin, emax = w[0] - 0.3, w[-1] + 0.3
    c = Chebyshev(BlockSpMat(H.row_ptr, H.col_ind, H.values, b), emin, emax)
    Vd = [BlockSpMat(W.row_ptr, W.col_ind, W.values, b, imaginary=True) for W in Ws]
    op = oracle.make_op(to_oracle(H), (emax + emin) / 2, (emax - emin) / 2)
    Vo = [to_oracle(W, imag=True) for W in Ws]
    rng = np.random.default_rng(b)
    for R, M, form in ((1, 7, 0), (2, 16, 1), (5, 9, 0), (5, 12, 1)):
        psi = np.exp(2j * np.pi * rng.random((n * b, R))) / np.sqrt(n * b)
        p = torch.as_tensor(psi).cuda().contiguous()
        sig, en = dc_spectrum_fftcheb(c, *Vd, p, M, formulation=form)
        sig_o, en_o = oracle.fftcheb(op, Vo, psi, M, formulation=form, prefactor=1.0,
                                     sections=1)
        assert np.allclose(en, en_o, rtol=0, atol=1e-13)
        assert rel_err(sig, sig_o) < 1e-10, (R, M, form)


@pytest.mark.parametrize("b", [1, 2, 3, 4, 5, 8])
def test_vjp_sweep(torch_cuda, b):
    """rsatb_kpm_moments_vjp for every built block size and sample counts 1,
    3, 8 (the recurrence kernels and the SDDMM at each width) against the
    oracle's dense FP64 reference gradient to 1e-10."""
    torch = torch_cuda
    from rsatb_b200.adjoint import kpm_moments_vjp
    from rsatb_b200.calc import Chebyshev
    from rsatb_b200.vbcsr import BlockSpMat
    n = 19
    H = random_hermitian_bsr(n, b, 3, seed=51 + b, complex_values=False, scale=0.4)
    Hd = H.to_dense()
    w = np.linalg.eigvalsh(Hd)
    emin, emax = w[0] - 0.3, w[-1] + 0.3
    c = Chebyshev(BlockSpMat(H.row_ptr, H.col_ind, H.values, b), emin, emax)
    cc, hw = (emax + emin) / 2, (emax - emin) / 2
    rows = np.repeat(np.arange(n), np.diff(H.row_ptr))
    rng = np.random.default_rng(b)
    for R, M in ((1, 5), (3, 12), (8, 9)):
        psi = rng.choice([-1.0, 1.0], size=(n * b, R)) / np.sqrt(n * b)
        dmu = rng.standard_normal(M)
        grad, mu, _ = kpm_moments_vjp(c, torch.as_tensor(psi).cuda(), M, dmu, 0)
        G = oracle.kpm_moments_vjp_dense(Hd, psi, cc, hw, M, dmu)
        want = np.stack([G[i * b:(i + 1) * b, j * b:(j + 1) * b]
                         for i, j in zip(rows, H.col_ind)])
        assert np.abs(mu - oracle.kpm_plain_moments_dense(Hd, psi, cc, hw, M)).max() < 1e-12
        assert rel_err(grad.cpu().numpy().reshape(want.shape), want) < 1e-10, (R, M)


@pytest.mark.parametrize("b", [1, 2, 3, 5, 8])
def test_refine_sweep(torch_cuda, b):
    """The sparse Newton-Schulz refinement (rsatb_inverse_sqrt_refine: the
    block SpGEMM at every block size up to 8, the runtime-size numeric phase
    below 8) from the seed c I on S's pattern, against the oracle's dense
    restatement of the loop: same steps, factor to 1e-10."""
    from rsatb_b200.isqrt import InverseSqrtOptions, inverse_sqrt
    n = 26
    A = random_hermitian_bsr(n, b, 3, seed=71 + b, complex_values=False, scale=0.15)
    w = np.linalg.eigvalsh(A.to_dense())
    vals = A.values.copy()
    seed_vals = np.zeros_like(vals)
    s_max = w[-1] + (1.0 - w[0])
    for i in range(n):
        for k in range(A.row_ptr[i], A.row_ptr[i + 1]):
            if A.col_ind[k] == i:
                vals[k] += (1.0 - w[0]) * np.eye(b)  # spectrum in [1, s_max]
                seed_vals[k] = np.eye(b) / np.sqrt(s_max)
    S = A.with_values(vals)
    Z0 = A.with_values(seed_vals)
    Z, rep = inverse_sqrt(S, InverseSqrtOptions(tol=1e-11, sptol=0.0, maxit=30, route=1),
                          seed=Z0)
    Zd = Z.to_arrays().to_dense()
    Z_ref, r_ref = oracle.ns_refine_dense(S.to_dense(), Z0.to_dense(), b, tol=1e-11, maxit=30)
    assert rep.converged == r_ref["converged"] and rep.steps == r_ref["steps"], (rep, r_ref)
    assert np.abs(Zd - Z_ref).max() <= 1e-10 * np.abs(Z_ref).max()


@pytest.mark.parametrize("b", [1, 2, 5])
def test_qe_sweep(torch_cuda, b):
    """The quasi-eigenstate route (rsatb_dc_spectrum_qe) for block sizes 1,
    2, 5, sample counts 1 and 3, all nodes and a window of them, equal to the
    FFT-Chebyshev Greenwood spectrum on the same nodes to 1e-10."""
    torch = torch_cuda
    from rsatb_b200.calc import Chebyshev
    from rsatb_b200.transport import dc_spectrum_fftcheb, dc_spectrum_qe
    from rsatb_b200.vbcsr import BlockSpMat
    n = 21
    H = random_hermitian_bsr(n, b, 3, seed=91 + b, complex_values=False, scale=0.4)
    Ws = [_antisymmetric(random_hermitian_bsr(n, b, 3, seed=91 + b, complex_values=False,
                                              scale=0.3 + 0.1 * a)) for a in range(3)]
    w = np.linalg.eigvalsh(H.to_dense())
    c = Chebyshev(BlockSpMat(H.row_ptr, H.col_ind, H.values, b), w[0] - 0.3, w[-1] + 0.3)
    Vd = [BlockSpMat(W.row_ptr, W.col_ind, W.values, b, imaginary=True) for W in Ws]
    rng = np.random.default_rng(b)
    for R, M, nodes in ((1, 11, None), (3, 20, [2, 3, 7, 15, 19])):
        psi = np.exp(2j * np.pi * rng.random((n * b, R))) / np.sqrt(n * b)
        p = torch.as_tensor(psi).cuda().contiguous()
        sig_f, en_f = dc_spectrum_fftcheb(c, *Vd, p, M)
        sig_q, en_q = dc_spectrum_qe(c, *Vd, p, M, nodes_ascending=nodes)
        idx = np.arange(M) if nodes is None else np.array(nodes)
        assert np.allclose(en_q, en_f, rtol=0, atol=1e-13)
        assert rel_err(sig_q[idx], sig_f[idx]) < 1e-10, (R, M)
        if nodes is not None:
            rest = np.setdiff1d(np.arange(M), idx)
            assert np.all(sig_q[rest] == 0.0)
