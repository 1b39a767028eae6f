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
