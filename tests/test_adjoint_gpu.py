"""Adjoint KPM (rsatb_kpm_moments_vjp, KpmDosLoss) against the dense FP64
reference gradient of the oracle and against central finite differences
(h = 1e-6) of the loss, on a small silicon sp3s* operator (5x5 blocks to the
2nd neighbour shell)."""
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
def si():
    from rsatb_b200 import lattice
    H = lattice.silicon_sp3s(L=2, seed=5)          # 64 atoms, N = 320
    w = np.linalg.eigvalsh(H.to_dense())
    return H, w[0] - 0.5, w[-1] + 0.5


def _rademacher(n, R, seed=3):
    rng = np.random.default_rng(seed)
    return rng.choice([-1.0, 1.0], size=(n, R)) / np.sqrt(n)


def _pattern_grad(H, G):
    rows = np.repeat(np.arange(H.n_block_rows), np.diff(H.row_ptr))
    b = H.block_size
    out = np.zeros_like(H.values)
    for k, (i, j) in enumerate(zip(rows, H.col_ind)):
        out[k] = G[i * b:(i + 1) * b, j * b:(j + 1) * b]
    return out


def _cheby(H, emin, emax, precision="f64"):
    from rsatb_b200.calc import Chebyshev
    from rsatb_b200.vbcsr import BlockSpMat
    c = Chebyshev(BlockSpMat(H.row_ptr, H.col_ind, H.values, H.block_size), emin, emax)
    return c.astype("f32") if precision == "f32" else c


@pytest.mark.parametrize("M,stride", [(2, 0), (3, 1), (32, 0), (40, 7), (33, 33)])
def test_vjp_matches_dense_reference(torch_cuda, si, M, stride):
    from rsatb_b200.adjoint import kpm_moments_vjp
    H, emin, emax = si
    psi = _rademacher(H.n_rows, 4)
    dmu = np.random.default_rng(M).standard_normal(M)
    c = _cheby(H, emin, emax)
    grad, mu, st = kpm_moments_vjp(c, torch_cuda.as_tensor(psi).cuda(), M, dmu, stride)
    Hd = H.to_dense()
    cc, hw = (emax + emin) / 2, (emax - emin) / 2
    mu_ref = oracle.kpm_plain_moments_dense(Hd, psi, cc, hw, M)
    G = oracle.kpm_moments_vjp_dense(Hd, psi, cc, hw, M, dmu)
    assert np.abs(mu - mu_ref).max() < 1e-12
    assert rel_err(grad.cpu().numpy(), _pattern_grad(H, G)) < 1e-10
    if stride:
        assert st["checkpoint_stride"] == min(stride, M)


def test_checkpoint_stride_does_not_change_gradient(torch_cuda, si):
    from rsatb_b200.adjoint import kpm_moments_vjp
    H, emin, emax = si
    psi = torch_cuda.as_tensor(_rademacher(H.n_rows, 8)).cuda()
    dmu = np.random.default_rng(1).standard_normal(64)
    c = _cheby(H, emin, emax)
    g = [kpm_moments_vjp(c, psi, 64, dmu, s)[0] for s in (1, 8, 0, 64)]
    for x in g[1:]:
        assert rel_err(x.cpu().numpy(), g[0].cpu().numpy()) < 1e-13


def test_fp32_vjp_against_fp64(torch_cuda, si):
    from rsatb_b200.adjoint import kpm_moments_vjp
    H, emin, emax = si
    psi = _rademacher(H.n_rows, 8)
    dmu = np.random.default_rng(2).standard_normal(48)
    g64, _, _ = kpm_moments_vjp(_cheby(H, emin, emax), torch_cuda.as_tensor(psi).cuda(), 48,
                                dmu)
    g32, _, _ = kpm_moments_vjp(_cheby(H, emin, emax, "f32"),
                                torch_cuda.as_tensor(psi).float().cuda(), 48, dmu)
    assert rel_err(g32.cpu().numpy(), g64.cpu().numpy()) < 1e-4


def _loss_setup(torch, si, M=48):
    from rsatb_b200.vbcsr import BlockSpMat
    H, emin, emax = si
    Hd = BlockSpMat(H.row_ptr, H.col_ind, H.values, H.block_size)
    psi = torch.as_tensor(_rademacher(H.n_rows, 8, seed=9)).cuda()
    x = np.linspace(-0.95, 0.95, 81)
    target = np.random.default_rng(4).random(x.size) * 0.3
    return H, Hd, psi, emin, emax, M, x, target


def test_autograd_loss_matches_finite_differences(torch_cuda, si):
    """Central differences (h = 1e-6) on 12 sampled block values and along
    one random direction over all of them."""
    torch = torch_cuda
    from rsatb_b200.adjoint import KpmDosLoss
    H, Hd, psi, emin, emax, M, x, target = _loss_setup(torch, si)
    v0 = torch.as_tensor(H.values).cuda().clone()
    v = v0.clone().requires_grad_(True)
    loss = KpmDosLoss.apply(v, Hd, psi, emin, emax, M, x, target)
    loss.backward()
    g = v.grad.cpu().numpy()

    def L(vals):
        return float(KpmDosLoss.apply(vals, Hd, psi, emin, emax, M, x, target))

    h = 1e-6
    rng = np.random.default_rng(7)
    flat = v0.reshape(-1)
    for e in rng.choice(flat.numel(), size=12, replace=False):
        p = flat.clone()
        m = flat.clone()
        p[e] += h
        m[e] -= h
        fd = (L(p.view_as(v0)) - L(m.view_as(v0))) / (2 * h)
        assert abs(fd - g.reshape(-1)[e]) <= 1e-6 * max(1.0, abs(fd)), (e, fd, g.reshape(-1)[e])
    D = torch.as_tensor(rng.standard_normal(tuple(v0.shape))).cuda()
    fd = (L(v0 + h * D) - L(v0 - h * D)) / (2 * h)
    assert abs(fd - float((v.grad * D).sum())) <= 1e-6 * max(1.0, abs(fd))
    # the reference gradient of the same loss
    Hm = H.to_dense()
    cc, hw = (emax + emin) / 2, (emax - emin) / 2
    from rsatb_b200.adjoint import dos_basis
    Db = dos_basis(M, x)
    mu = oracle.kpm_plain_moments_dense(Hm, psi.cpu().numpy(), cc, hw, M)
    dmu = 2.0 * ((Db @ mu - target) @ Db)
    G = oracle.kpm_moments_vjp_dense(Hm, psi.cpu().numpy(), cc, hw, M, dmu)
    assert rel_err(g, _pattern_grad(H, G)) < 1e-10


def test_sandwich_and_complex_refused(torch_cuda, si):
    from rsatb_b200._capi import RsatbError
    from rsatb_b200.adjoint import kpm_moments_vjp
    H, emin, emax = si
    c = _cheby(H, emin, emax)
    psi = torch_cuda.as_tensor(_rademacher(H.n_rows, 2)).cuda()
    with pytest.raises(RsatbError):     # FP32 vectors on an FP64 operator
        kpm_moments_vjp(c, psi.float(), 8, np.ones(8))
    with pytest.raises(ValueError):
        kpm_moments_vjp(c, psi, 8, np.ones(5))


# ------------------------------------------------------ sandwich form and S

def _diamond_sandwich_case(torch, L=2, R=6, M=40):
    from rsatb_b200 import lattice
    from rsatb_b200.calc import Chebyshev, ISQRTMPreconditioner
    from rsatb_b200.isqrt import graph_inverse_sqrt
    from rsatb_b200.vbcsr import BlockSpMat
    H, S = lattice.diamond_lcao(L=L, seed=3)
    Z = graph_inverse_sqrt(S)
    Hd, Zd = H.to_dense(), Z.to_dense()
    w = np.linalg.eigvalsh(Zd.T @ Hd @ Zd)
    emin, emax = w[0] - 0.5, w[-1] + 0.5
    cheby = Chebyshev(BlockSpMat(H.row_ptr, H.col_ind, H.values, 8), emin, emax,
                      preconditioner=ISQRTMPreconditioner(BlockSpMat(Z.row_ptr, Z.col_ind,
                                                                     Z.values, 8)))
    psi = np.random.default_rng(9).choice([-1.0, 1.0], (H.n_rows, R)) / np.sqrt(H.n_rows)
    dmu = np.random.default_rng(10).standard_normal(M)
    return H, S, Z, cheby, psi, dmu, emin, emax


def _on_pattern(A, dense):
    b = A.block_size
    rows = np.repeat(np.arange(A.n_block_rows), np.diff(A.row_ptr))
    return np.stack([dense[i * b:(i + 1) * b, j * b:(j + 1) * b]
                     for i, j in zip(rows, A.col_ind)])


def test_sandwich_vjp_matches_dense_reference(torch_cuda):
    """grad_h = Z G Z^T and grad_z = H Z (G + G^T) (G = dL/d(Z^T H Z), the
    dense FP64 reverse-mode gradient of the oracle) on the stored patterns,
    1e-10 of the largest entry; FP32 panels within 1e-5."""
    torch = torch_cuda
    from rsatb_b200.adjoint import kpm_moments_vjp_sandwich
    H, S, Z, cheby, psi, dmu, emin, emax = _diamond_sandwich_case(torch)
    M = dmu.size
    Hd, Zd = H.to_dense(), Z.to_dense()
    c, hw = (emax + emin) / 2, (emax - emin) / 2
    Gs = oracle.kpm_moments_vjp_dense(Zd.T @ Hd @ Zd, psi, c, hw, M, dmu)
    want_h = _on_pattern(H, Zd @ Gs @ Zd.T)
    want_z = _on_pattern(Z, Hd @ Zd @ (Gs + Gs.T))
    p = torch.as_tensor(psi).cuda()
    gh, gz, mu, _ = kpm_moments_vjp_sandwich(cheby, p, M, dmu, checkpoint_stride=7)
    mu_ref = oracle.kpm_plain_moments_dense(Zd.T @ Hd @ Zd, psi, c, hw, M)
    assert np.abs(mu - mu_ref).max() < 1e-12
    assert rel_err(gh.cpu().numpy(), want_h) < 1e-10
    assert rel_err(gz.cpu().numpy(), want_z) < 1e-10
    gh32, gz32, _, _ = kpm_moments_vjp_sandwich(cheby.astype("f32"), p.float(), M, dmu)
    assert rel_err(gh32.cpu().numpy(), want_h) < 1e-5
    assert rel_err(gz32.cpu().numpy(), want_z) < 1e-5


def test_grad_s_matches_dense_frechet_adjoint(torch_cuda):
    """grad_s_from_grad_z (device, batched eigh) against the oracle's
    row-by-row dense Frechet adjoint of the graph-local factor."""
    torch = torch_cuda
    from rsatb_b200.adjoint import grad_s_from_grad_z
    from rsatb_b200 import lattice
    _, S = lattice.diamond_lcao(L=2, seed=3)
    dZ = np.random.default_rng(12).standard_normal((S.nnz_blocks, 8, 8))
    gs = grad_s_from_grad_z(S, torch.as_tensor(dZ).cuda()).cpu().numpy()
    Zpat = lattice.BsrArrays(S.row_ptr, S.col_ind, dZ, 8)
    want = oracle.graph_seed_grad_s(S.to_dense(), np.asarray(S.row_ptr),
                                    np.asarray(S.col_ind), 8, Zpat.to_dense())
    assert rel_err(gs, _on_pattern(S, want)) < 1e-9


def test_dos_loss_gradient_in_h_and_s_against_finite_differences(torch_cuda):
    """d(L)/d(H, S block values) of the Jackson-DOS L2 loss of Z^T H Z:
    the directional derivative along a random symmetric perturbation of H
    and of S (both copies of each off-diagonal block moved together)
    against central finite differences with h = 1e-6."""
    torch = torch_cuda
    from rsatb_b200.adjoint import KpmDosLossSandwich
    from rsatb_b200 import lattice
    H, S, _, cheby, psi, _, emin, emax = _diamond_sandwich_case(torch, M=48)
    M = 48
    x = np.linspace(-0.95, 0.95, 41)
    target = np.random.default_rng(3).uniform(0.0, 0.3, x.size)
    p = torch.as_tensor(psi).cuda()

    def sym_dir(A, seed):
        d = np.random.default_rng(seed).standard_normal(A.values.shape)
        T = lattice.BsrArrays(A.row_ptr, A.col_ind, d, A.block_size)
        Dd = T.to_dense()
        return _on_pattern(A, 0.5 * (Dd + Dd.T))

    dH, dS = sym_dir(H, 21), 0.05 * sym_dir(S, 22)
    hv = torch.as_tensor(H.values).cuda().requires_grad_(True)
    sv = torch.as_tensor(S.values).cuda().requires_grad_(True)
    loss = KpmDosLossSandwich.apply(hv, sv, H, S, p, emin, emax, M, x, target)
    loss.backward()
    analytic = float((hv.grad.cpu().numpy() * dH).sum() + (sv.grad.cpu().numpy() * dS).sum())
    h = 1e-6

    def L(eps):
        with torch.no_grad():
            return float(KpmDosLossSandwich.apply(
                torch.as_tensor(H.values + eps * dH).cuda(),
                torch.as_tensor(S.values + eps * dS).cuda(), H, S, p, emin, emax, M, x, target))

    fd = (L(h) - L(-h)) / (2 * h)
    assert abs(fd - analytic) <= 1e-5 * max(abs(fd), 1e-12), (fd, analytic)
