"""GPU parity of the KPM path against the CPU oracle.

Tolerances: bit-exact for the seeded sample vectors; 1e-13 relative for
single FP64 SpMM / operator applications; 1e-10 of mu_0 for FP64 moments
(the bar of test_dos.cpp:131 and of the FP64 mode); FP32 (mixed) kernels
against the FP64 oracle at 1e-5 relative per application and a DOS error
<= 1e-5 of the FP64 DOS peak.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import oracle
from _util import adjoint_arrays, random_hermitian_bsr, rel_err, to_oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    return torch


def dev_bsr(A, precision="f64", imaginary=False):
    from rsatb_b200.vbcsr import BlockSpMat
    M = BlockSpMat(A.row_ptr, A.col_ind, A.values, A.block_size, A.n_block_cols,
                   imaginary=imaginary)
    return M.astype("f32") if precision == "f32" else M


def to_dev(torch, X, dtype=None):
    t = torch.as_tensor(np.ascontiguousarray(X)).cuda()
    return t.to(dtype) if dtype is not None else t


# ----------------------------------------------------------- sample vectors

@pytest.mark.parametrize("kind,cplx", [(0, True), (1, False), (1, True), (2, True), (2, False)])
def test_set_random_bit_exact(torch_cuda, kind, cplx):
    torch = torch_cuda
    from rsatb_b200.vbcsr import set_random
    ids = (np.arange(300) * 7 + 11).astype(np.int64)
    orbs, R, seed = 3, 5, 20240917
    want = oracle.set_random(seed, kind, True, ids, orbs, 900, R, cplx)
    out = torch.empty(900, R, dtype=torch.complex128 if cplx else torch.float64, device="cuda")
    set_random(out, seed, normalize=True, atom_index=ids, orbitals_per_atom=orbs, kind=kind)
    got = out.cpu().numpy()
    assert np.array_equal(got.view(np.float64), want.view(np.float64))
    # FP32 output is the FP64 value rounded once
    out32 = torch.empty(900, R, dtype=torch.complex64 if cplx else torch.float32, device="cuda")
    set_random(out32, seed, normalize=True, atom_index=ids, orbitals_per_atom=orbs, kind=kind)
    assert np.array_equal(out32.cpu().numpy(), want.astype(np.complex64 if cplx else np.float32))


# --------------------------------------------------------------- SpMM

CASES = [
    # (n_blocks, b, degree, complex matrix, imaginary flag, R, complex vectors)
    (300, 1, 3, False, False, 8, True),
    (300, 1, 3, False, False, 3, False),
    (120, 5, 6, False, False, 32, False),
    (64, 8, 10, False, False, 128, False),
    (64, 8, 10, False, False, 16, True),
    (90, 2, 4, True, False, 4, True),
    (70, 3, 5, False, False, 6, False),
    (70, 3, 5, True, False, 3, True),
    (200, 1, 8, False, True, 48, True),
    (50, 5, 4, True, False, 2, True),
    (40, 8, 5, True, False, 8, True),
    # imaginary-unit 8x8 blocks on complex panels: W = 16 and 32 (the
    # tensor-core and bulk-copy kernels), W = 256 (paired tensor-core loads)
    (40, 8, 5, False, True, 8, True),
    (40, 8, 5, False, True, 16, True),
    (33, 8, 4, False, True, 128, True),
]


def _panel(rng, n, R, cplx):
    X = rng.standard_normal((n, R))
    if cplx:
        X = X + 1j * rng.standard_normal((n, R))
    return X


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_mult_dense_matches_oracle(torch_cuda, case, precision):
    torch = torch_cuda
    n, b, deg, cm, imag, R, cv = case
    A = random_hermitian_bsr(n, b, deg, seed=n + b, complex_values=cm)
    if imag:
        A = A.with_values(A.values.real.copy())
    rng = np.random.default_rng(3)
    X = _panel(rng, n * b, R, cv)
    want = oracle.spmm(to_oracle(A, imag=imag), X, alpha=0.75)
    Ad = dev_bsr(A, precision, imaginary=imag)
    dt = {("f64", True): torch.complex128, ("f64", False): torch.float64,
          ("f32", True): torch.complex64, ("f32", False): torch.float32}[(precision, cv)]
    Xd = to_dev(torch, X, dt)
    Yd = torch.empty_like(Xd)
    Ad.mult_dense(Xd, Yd, alpha=0.75)
    got = Yd.cpu().numpy()
    tol = 1e-13 if precision == "f64" else 2e-5
    assert rel_err(got, want) < tol


def test_adjoint_matches_host_adjoint(torch_cuda):
    torch = torch_cuda
    A = random_hermitian_bsr(80, 3, 4, seed=5, complex_values=True)
    # make it non-Hermitian so the adjoint matters
    A = A.with_values(A.values * (1.0 + 0.3j))
    AH = adjoint_arrays(A)
    X = _panel(np.random.default_rng(1), 240, 4, True)
    want = oracle.spmm(to_oracle(AH), X)
    Ad = dev_bsr(A).adjoint()
    Xd = to_dev(torch, X)
    Yd = torch.empty_like(Xd)
    Ad.mult_dense(Xd, Yd)
    assert rel_err(Yd.cpu().numpy(), want) < 1e-13
    # imaginary-unit matrix: (i W)^H = -i W^T
    W = random_hermitian_bsr(60, 1, 3, seed=9, complex_values=False)
    W = W.with_values(np.random.default_rng(2).standard_normal(W.values.shape))
    WH = adjoint_arrays(W)
    want = oracle.spmm(to_oracle(WH, imag=True), X[:60], alpha=-1.0)
    Wd = dev_bsr(W, imaginary=True).adjoint()
    Xd = to_dev(torch, X[:60].copy())
    Yd = torch.empty_like(Xd)
    Wd.mult_dense(Xd, Yd)
    assert rel_err(Yd.cpu().numpy(), want) < 1e-13


# ------------------------------------------------------ operators and moments

def graphene_case(n1=12, n2=12):
    from rsatb_b200 import lattice
    H, _, _ = lattice.graphene(n1, n2)
    return H


def diamond_case(L=2):
    from rsatb_b200 import lattice
    from rsatb_b200.isqrt import graph_inverse_sqrt_host
    H, S = lattice.diamond_lcao(L=L, seed=3)
    Z = graph_inverse_sqrt_host(S)
    return H, S, Z


def build_cheby(H, emin, emax, Z=None, precision="f64"):
    from rsatb_b200.calc import Chebyshev, ISQRTMPreconditioner
    pre = ISQRTMPreconditioner(dev_bsr(Z)) if Z is not None else None
    c = Chebyshev(dev_bsr(H), emin, emax, preconditioner=pre)
    return c.astype("f32") if precision == "f32" else c


def oracle_op(H, emin, emax, Z=None):
    c, hw = (emax + emin) / 2, (emax - emin) / 2
    if Z is None:
        return oracle.make_op(to_oracle(H), c, hw)
    return oracle.make_op(to_oracle(H), c, hw, to_oracle(Z), to_oracle(adjoint_arrays(Z)))


def test_apply_op_orthogonal_and_sandwich(torch_cuda):
    torch = torch_cuda
    H = graphene_case()
    X = _panel(np.random.default_rng(4), H.n_rows, 8, True)
    c = build_cheby(H, -8.7, 8.9)
    Y = torch.empty(H.n_rows, 8, dtype=torch.complex128, device="cuda")
    c.apply_op(to_dev(torch, X), Y)
    assert rel_err(Y.cpu().numpy(), oracle.apply_op(oracle_op(H, -8.7, 8.9), X)) < 1e-13
    Hd, S, Z = diamond_case()
    X = _panel(np.random.default_rng(5), Hd.n_rows, 16, False)
    c = build_cheby(Hd, -12.0, 11.0, Z)
    Y = torch.empty(Hd.n_rows, 16, dtype=torch.float64, device="cuda")
    c.apply_op(to_dev(torch, X), Y)
    assert rel_err(Y.cpu().numpy(), oracle.apply_op(oracle_op(Hd, -12.0, 11.0, Z), X)) < 1e-13


def _moment_err(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("doubled", [True, False])
def test_kpm_moments_graphene_fp64(torch_cuda, doubled):
    torch = torch_cuda
    from rsatb_b200.calc import _moments
    from rsatb_b200.vbcsr import set_random
    H = graphene_case()
    emin, emax = -8.6, 8.6
    R, n_moments = 8, 128
    psi = torch.empty(H.n_rows, R, dtype=torch.complex128, device="cuda")
    set_random(psi, 20240917)
    want_mu, want_col = oracle.kpm_moments(oracle_op(H, emin, emax), psi.cpu().numpy(),
                                           n_moments, doubled=doubled, per_column=True)
    mu, col = _moments(build_cheby(H, emin, emax), psi, n_moments, doubled, per_column=True)
    assert _moment_err(mu, want_mu) < 1e-10
    assert _moment_err(col, want_col) < 1e-10


def test_kpm_moments_doubled_equals_plain(torch_cuda):
    torch = torch_cuda
    from rsatb_b200.calc import kpm_dos_moments, kpm_dos_moments_plain
    from rsatb_b200.vbcsr import set_random
    H = graphene_case(8, 8)
    c = build_cheby(H, -8.6, 8.6)
    psi = torch.empty(H.n_rows, 4, dtype=torch.complex128, device="cuda")
    set_random(psi, 1)
    a = kpm_dos_moments(c, psi, 64)
    b = kpm_dos_moments_plain(c, psi, 64)
    assert np.abs(a - b).max() < 1e-10


def test_kpm_moments_diamond_sandwich_fp64(torch_cuda):
    torch = torch_cuda
    from rsatb_b200.calc import kpm_dos_moments
    from rsatb_b200.vbcsr import set_random
    H, S, Z = diamond_case()
    emin, emax = -14.0, 14.0
    psi = torch.empty(H.n_rows, 16, dtype=torch.float64, device="cuda")
    set_random(psi, 7, orbitals_per_atom=8)
    want = oracle.kpm_moments(oracle_op(H, emin, emax, Z), psi.cpu().numpy(), 256)
    got = kpm_dos_moments(build_cheby(H, emin, emax, Z), psi, 256)
    assert _moment_err(got, want) < 1e-10
    assert np.abs(got).max() <= 1.0 + 1e-9  # spectrum inside the window


@pytest.mark.parametrize("n_moments", [1, 2, 3, 4, 5, 33])
def test_kpm_moments_complex_matrix_edge_counts(torch_cuda, n_moments):
    torch = torch_cuda
    from rsatb_b200.calc import _moments
    A = random_hermitian_bsr(40, 2, 3, seed=21, complex_values=True, scale=0.3)
    psi = _panel(np.random.default_rng(8), 80, 3, True)
    bound = np.abs(np.linalg.eigvalsh(A.to_dense())).max() + 0.5
    for doubled in (True, False):
        want = oracle.kpm_moments(oracle_op(A, -bound, bound), psi, n_moments, doubled=doubled)
        got, _ = _moments(build_cheby(A, -bound, bound), to_dev(torch, psi), n_moments, doubled)
        assert got.shape == (n_moments,)
        assert _moment_err(got, want) < 1e-10


def dos_error(mu, mu_ref, nt=200):
    from rsatb_b200.calc import evaluate_kpm_density
    i = np.arange(nt)
    x = np.concatenate([(i - nt) / nt, i / nt])
    rho = 2 * evaluate_kpm_density(mu, x, 0.5 / nt)
    ref = 2 * evaluate_kpm_density(mu_ref, x, 0.5 / nt)
    return float(np.abs(rho - ref).max() / np.abs(ref).max())


def test_mixed_precision_dos_error(torch_cuda):
    """FP32 matrices/vectors with FP64 rescale and dots: DOS within 1e-5 of the
    FP64 path (peak-normalised), on graphene (orthogonal) and diamond
    (sandwich)."""
    torch = torch_cuda
    from rsatb_b200.calc import kpm_dos_moments
    from rsatb_b200.vbcsr import set_random
    H = graphene_case(30, 30)
    c64 = build_cheby(H, -8.6, 8.6)
    psi = torch.empty(H.n_rows, 8, dtype=torch.complex128, device="cuda")
    set_random(psi, 20240917)
    mu64 = kpm_dos_moments(c64, psi, 512)
    mu32 = kpm_dos_moments(c64.astype("f32"), psi.to(torch.complex64), 512)
    assert dos_error(mu32, mu64) < 1e-5
    Hd, S, Z = diamond_case()
    c64 = build_cheby(Hd, -14.0, 14.0, Z)
    psi = torch.empty(Hd.n_rows, 32, dtype=torch.float64, device="cuda")
    set_random(psi, 4, orbitals_per_atom=8)
    mu64 = kpm_dos_moments(c64, psi, 1024)
    mu32 = kpm_dos_moments(c64.astype("f32"), psi.to(torch.float32), 1024)
    assert dos_error(mu32, mu64) < 1e-5


def test_density_matches_oracle(torch_cuda):
    from rsatb_b200.calc import KpmKernel, evaluate_kpm_density
    rng = np.random.default_rng(0)
    mu = rng.standard_normal(300) * np.exp(-np.arange(300) / 60) + 0j
    mu[0] = 1.0
    x = np.linspace(-1, 1, 2001)
    for k in (KpmKernel.Jackson, KpmKernel.None_, KpmKernel.CosTaper, KpmKernel.VpTaper):
        got = evaluate_kpm_density(mu, x, 1e-3, k)
        want = oracle.density(mu, x, 1e-3, int(k))
        assert rel_err(got, want) < 1e-12


def test_lanczos_bounds_contain_spectrum(torch_cuda):
    from rsatb_b200.bounds import estimate_spectral_bounds
    from rsatb_b200.calc import Chebyshev
    H = graphene_case(20, 20)
    emin, emax = estimate_spectral_bounds(Chebyshev(dev_bsr(H), -1, 1))
    assert emin < -8.1 and emax > 8.1 and emax < 10.5


@pytest.mark.parametrize("kind", ["real", "complex", "f32", "solve"])
def test_native_lanczos_matches_oracle(torch_cuda, kind):
    """rsatb_lanczos_extremes (device FP64 basis, host implicit QL) against
    the oracle's host Lanczos from the same seeded start vector: the padded
    20-step window to 1e-9 for a real, a complex and an FP32 operator (its
    matvecs in FP32: 1e-5); for the Solve form S^-1 H the converged window
    contains the dense generalised eigenvalues and its Ritz values match
    them to 1e-6."""
    from rsatb_b200.bounds import estimate_spectral_bounds, lanczos_extremes
    from rsatb_b200.calc import Chebyshev
    if kind == "solve":
        from rsatb_b200 import lattice
        from rsatb_b200.vbcsr import BlockSpMat
        Hd, S = lattice.diamond_lcao(L=2, seed=3)
        dev = lambda A: BlockSpMat(A.row_ptr, A.col_ind, A.values, A.block_size)
        c = Chebyshev(dev(Hd), -1, 1, overlap=dev(S), cg_tol=1e-12)
        info = {}
        tmin, tmax, rmin, rmax = lanczos_extremes(c, tol=1e-8, info=info)
        w = np.linalg.eigvals(np.linalg.solve(S.to_dense(), Hd.to_dense())).real
        assert info["converged"]
        assert abs(tmin - w.min()) < 1e-6 * np.abs(w).max()
        assert abs(tmax - w.max()) < 1e-6 * np.abs(w).max()
        return
    if kind == "complex":
        A = random_hermitian_bsr(60, 4, 5, seed=9, complex_values=True, scale=0.5)
    else:
        A = graphene_case(12, 12)
    Ad = A.to_dense()
    c = Chebyshev(dev_bsr(A, "f32" if kind == "f32" else "f64"), -1, 1)
    got = estimate_spectral_bounds(c, steps=20)
    want = oracle.lanczos_bounds(lambda x: Ad @ x, Ad.shape[0], steps=20,
                                 complex_values=(kind == "complex"))
    tol = 1e-5 if kind == "f32" else 1e-9
    assert abs(got[0] - want[0]) < tol * abs(want[0]) and abs(got[1] - want[1]) < tol * abs(want[1])


NARROW = [(96, 8, 6, False, False, 8, False), (96, 8, 6, False, False, 4, True),
          (96, 8, 6, False, False, 16, False), (80, 5, 5, False, False, 4, False),
          (80, 5, 5, False, False, 8, True), (80, 5, 5, False, False, 4, True),
          # bulk-copy kernel widths W = 64 and 256 and ragged group counts
          # (97 block rows: not a multiple of the 2..32 block rows per warp)
          (97, 8, 7, False, False, 64, False), (97, 8, 7, False, False, 128, True),
          (97, 8, 7, False, False, 256, False), (97, 8, 7, False, False, 2, True),
          # narrow tensor-core widths W = 32 and complex W = 16, 32
          (97, 8, 7, False, False, 32, False), (97, 8, 7, False, False, 8, True),
          (97, 8, 7, False, False, 16, True),
          # complex H of 1x1 blocks, 3 complex columns: the staged kernel's
          # 48 KB of dynamic shared memory plus its static dot-finish arrays
          (60, 1, 5, True, False, 3, True)]


@pytest.mark.parametrize("kernel", ["staged", "rowsplit", "bulk", "bulk_smem", "narrow", "dmma",
                                    "tf32"])
@pytest.mark.parametrize("case", [c for c in CASES if c[1] in (1, 5, 8)] + NARROW)
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_kernel_variants_match_register_kernel(torch_cuda, case, precision, kernel, monkeypatch):
    """The cp.async-staged, the row-split, the bulk-copy, the lock-step
    narrow-panel and the FP64 tensor-core step kernels against the register
    kernel, including the fused epilogue and
    dots (the row-split kernel sums in another order, hence a relative
    tolerance; the bulk-copy kernel keeps the register kernel's order per
    output and differs only in the FP64 dot reduction order)."""
    torch = torch_cuda
    from rsatb_b200.calc import Chebyshev, _moments
    n, b, deg, cm, imag, R, cv = case
    if imag:
        return
    A = random_hermitian_bsr(n, b, deg, seed=n + 7 * b, complex_values=cm, scale=0.2)
    bound = np.abs(np.linalg.eigvalsh(A.to_dense())).max() + 0.5
    c = build_cheby(A, -bound, bound, precision=precision)
    X = _panel(np.random.default_rng(11), n * b, R, cv)
    dt = {("f64", True): torch.complex128, ("f64", False): torch.float64,
          ("f32", True): torch.complex64, ("f32", False): torch.float32}[(precision, cv)]
    Xd = to_dev(torch, X, dt)
    monkeypatch.setenv("RSATB_STEP_KERNEL", kernel.split("_")[0])
    if kernel == "bulk_smem":
        monkeypatch.setenv("RSATB_BULK_X", "smem")  # X rows through the copy ring too
    Y1 = torch.empty_like(Xd)
    c.H.mult_dense(Xd, Y1)
    mu1, col1 = _moments(c, Xd, 24, True, per_column=True)
    monkeypatch.setenv("RSATB_STEP_KERNEL", "v1")
    Y2 = torch.empty_like(Xd)
    c.H.mult_dense(Xd, Y2)
    mu2, col2 = _moments(c, Xd, 24, True, per_column=True)
    tol = (1e-13 if precision == "f64" else 1e-6) * (50 if kernel == "rowsplit" else 1)
    if kernel == "tf32" and precision == "f32":
        tol = 5e-6  # split TF32: the lo x lo term is dropped, the tensor core sums a block
    assert rel_err(Y1.cpu().numpy(), Y2.cpu().numpy()) < tol
    assert np.abs(col1 - col2).max() <= tol * np.abs(col2).max() * 10


def test_recurrence_graph_replay_matches_direct_run(torch_cuda, monkeypatch):
    """The second identical call captures the recurrence as a CUDA graph and
    later ones replay it: same moments bit for bit, same launch count."""
    torch = torch_cuda
    monkeypatch.setenv("RSATB_NO_PERSIST", "1")  # the small-operator path is one launch
    from rsatb_b200.calc import kpm_dos_moments
    from rsatb_b200.vbcsr import set_random
    H = graphene_case(16, 16)
    c = build_cheby(H, -9.0, 9.0)
    psi = torch.empty(H.n_rows, 4, dtype=torch.complex128, device="cuda")
    set_random(psi, 7)
    ctx = c.H.ctx
    mus, counts = [], []
    for _ in range(4):
        l0 = ctx.launch_count()
        mus.append(kpm_dos_moments(c, psi, 96))
        counts.append(ctx.launch_count() - l0)
    monkeypatch.setenv("RSATB_NO_GRAPH", "1")
    direct = kpm_dos_moments(c, psi, 96)
    for m in mus:
        assert np.array_equal(m, direct)
    assert len(set(counts)) == 1 and counts[0] == 1 + 48


def test_bulk_kernel_bounded_wait_reports_fault(torch_cuda, monkeypatch):
    """A bounded mbarrier wait that runs out (armed for bytes no copy
    delivers) sets the context's fault word; rsatb_kpm_dos_moments then
    fails with RSATB_CUDA_ERROR instead of hanging, and the context stays
    usable: the next call returns the oracle's moments."""
    torch = torch_cuda
    from rsatb_b200._capi import RsatbError
    from rsatb_b200.calc import kpm_dos_moments
    A = random_hermitian_bsr(40, 8, 5, seed=3, complex_values=False, scale=0.2)
    bound = np.abs(np.linalg.eigvalsh(A.to_dense())).max() + 0.5
    c = build_cheby(A, -bound, bound, precision="f32")
    X = np.random.default_rng(5).standard_normal((40 * 8, 16))
    Xd = to_dev(torch, X, torch.float32)
    monkeypatch.setenv("RSATB_STEP_KERNEL", "bulk")
    monkeypatch.setenv("RSATB_TEST_BULK_WAIT", "1")
    with pytest.raises(RsatbError, match="bounded wait"):
        kpm_dos_moments(c, Xd, 8)
    monkeypatch.delenv("RSATB_TEST_BULK_WAIT")
    mu = kpm_dos_moments(c, Xd, 8)
    monkeypatch.setenv("RSATB_STEP_KERNEL", "v1")
    ref = kpm_dos_moments(c, Xd, 8)
    assert np.all(np.isfinite(mu))
    assert np.abs(mu - ref).max() <= 1e-6 * np.abs(ref).max()


def test_async_entry_points_report_a_bounded_wait_at_the_next_synchronisation(torch_cuda,
                                                                             monkeypatch):
    """rsatb_bsr_mult_dense, rsatb_cheb_apply_op, rsatb_cheb_apply_dual and
    rsatb_cheb_propagate return as soon as their launches are queued, so a
    bounded wait that gives up inside them is reported by the next
    synchronising call on the context: rsatb_ctx_synchronize here.  The
    synchronisation after that, and the moments of the next call, are clean."""
    torch = torch_cuda
    from rsatb_b200._capi import RsatbError
    from rsatb_b200.calc import kpm_dos_moments
    A = random_hermitian_bsr(40, 8, 5, seed=3, complex_values=False, scale=0.2)
    bound = np.abs(np.linalg.eigvalsh(A.to_dense())).max() + 0.5
    c = build_cheby(A, -bound, bound, precision="f32")
    X = to_dev(torch, np.random.default_rng(5).standard_normal((40 * 8, 16)), torch.float32)
    Y = torch.empty_like(X)
    ctx = c.H.ctx
    calls = {"mult_dense": lambda: c.H.mult_dense(X, Y),
             "apply_op": lambda: c.apply_op(X, Y),
             "apply_dual": lambda: c.apply_dual(c.H, X, Y),
             "propagate": lambda: c.propagate(X, Y, np.array([0.5, 0.25, 0.125]))}
    for name, call in calls.items():
        monkeypatch.setenv("RSATB_STEP_KERNEL", "bulk")
        monkeypatch.setenv("RSATB_TEST_BULK_WAIT", "1")
        call()  # queued: no error yet
        with pytest.raises(RsatbError, match="bounded wait"):
            ctx.synchronize()
        monkeypatch.delenv("RSATB_TEST_BULK_WAIT")
        ctx.synchronize()  # the word was cleared by the report
    mu = kpm_dos_moments(c, X, 8)
    monkeypatch.setenv("RSATB_STEP_KERNEL", "v1")
    ref = kpm_dos_moments(c, X, 8)
    assert np.abs(mu - ref).max() <= 1e-6 * np.abs(ref).max()


@pytest.mark.parametrize("precision,doubled,R", [("f64", True, 8), ("f64", False, 8),
                                                 ("f32", True, 8), ("f64", True, 3),
                                                 ("f64", True, 5), ("f32", True, 6),
                                                 ("f64", False, 1)])
def test_persistent_recurrence_matches_graph_path(torch_cuda, monkeypatch, precision, doubled, R):
    """Small scalar-block operators run the whole recurrence as one
    cooperative launch (grid barriers between steps); its moments match the
    per-step path to rounding (only the order of the FP64 dot sums differs)
    and the oracle, in two launches per call.  R = 3, 5, 6 give rows of 3, 5
    and 3 lanes, which do not divide 256 threads."""
    torch = torch_cuda
    from rsatb_b200.calc import kpm_dos_moments, kpm_dos_moments_plain
    from rsatb_b200.vbcsr import set_random
    H = graphene_case(12, 10)
    c = build_cheby(H, -9.0, 9.0, precision=precision)
    dt = torch.complex128 if precision == "f64" else torch.complex64
    psi = torch.empty(H.n_rows, R, dtype=dt, device="cuda")
    set_random(psi, 11)
    run = kpm_dos_moments if doubled else kpm_dos_moments_plain
    ctx = c.H.ctx
    l0 = ctx.launch_count()
    mu_p = run(c, psi, 64)
    assert ctx.launch_count() - l0 == 2
    monkeypatch.setenv("RSATB_NO_PERSIST", "1")
    mu_g = run(c, psi, 64)
    tol = 1e-12 if precision == "f64" else 1e-6
    assert np.abs(mu_p - mu_g).max() <= tol * np.abs(mu_g).max()
    if precision == "f64":
        want = oracle.kpm_moments(oracle_op(H, -9.0, 9.0), psi.cpu().numpy(), 64,
                                  doubled=doubled)
        assert _moment_err(mu_p, want) < 1e-10


def _dense_op(H, emin, emax, Z=None):
    c, hw = (emax + emin) / 2, (emax - emin) / 2
    Hd = H.to_dense()
    if Z is not None:
        Zd = Z.to_dense()
        Hd = Zd.conj().T @ Hd @ Zd
    return (Hd - c * np.eye(Hd.shape[0])) / hw


def _propagate_ref(Op, X, coeffs):
    """sum_n c_n T_n(Op) X by the three-term recurrence (cheby.hpp:399-441)."""
    t0, out = X.copy(), coeffs[0] * X
    if len(coeffs) > 1:
        t1 = Op @ X
        out = out + coeffs[1] * t1
        for c in coeffs[2:]:
            t0, t1 = t1, 2 * (Op @ t1) - t0
            out = out + c * t1
    return out


@pytest.mark.parametrize("case", ["graphene_c128", "diamond_sandwich_f64", "bsr8_f32"])
def test_propagate_matches_dense(torch_cuda, case):
    """Chebyshev::propagate: V_out = sum c_n T_n(Op~) V_in with complex
    coefficients (a real panel takes their real parts)."""
    torch = torch_cuda
    rng = np.random.default_rng(8)
    coeffs = rng.standard_normal(13) + 1j * rng.standard_normal(13)
    if case == "graphene_c128":
        H, Z, emin, emax, prec, cv, R = graphene_case(8, 8), None, -8.7, 8.9, "f64", True, 4
    elif case == "diamond_sandwich_f64":
        H, S, Z = diamond_case()
        emin, emax, prec, cv, R = -15.0, 15.0, "f64", False, 16
    else:
        H = random_hermitian_bsr(30, 8, 5, seed=4, complex_values=False, scale=0.2)
        Z, prec, cv, R = None, "f32", True, 8
        b = np.abs(np.linalg.eigvalsh(H.to_dense())).max() + 0.5
        emin, emax = -b, b
    X = _panel(rng, H.n_rows, R, cv)
    dt = {("f64", True): torch.complex128, ("f64", False): torch.float64,
          ("f32", True): torch.complex64, ("f32", False): torch.float32}[(prec, cv)]
    c = build_cheby(H, emin, emax, Z, precision=prec)
    Xd = to_dev(torch, X, dt)
    Yd = torch.empty_like(Xd)
    c.propagate(Xd, Yd, coeffs)
    want = _propagate_ref(_dense_op(H, emin, emax, Z), X, coeffs if cv else coeffs.real)
    tol = 1e-12 if prec == "f64" else 2e-5
    assert rel_err(Yd.cpu().numpy(), want) < tol
    # no coefficients: the output is left as it was
    Yd.fill_(3.0)
    c.propagate(Xd, Yd, [])
    assert (Yd.cpu().numpy() == 3.0).all()


def test_apply_dual_orthogonal_and_sandwich(torch_cuda):
    """Chebyshev::apply_dual: scale * V X (orthogonal) and scale * Z^H V Z X
    (sandwich) with an imaginary-unit velocity matrix."""
    torch = torch_cuda
    rng = np.random.default_rng(12)
    H, S, Z = diamond_case()
    W = random_hermitian_bsr(H.n_block_rows, 8, 4, seed=21, complex_values=False)
    Vd = dev_bsr(W, imaginary=True)
    X = _panel(rng, H.n_rows, 6, True)
    Xd = to_dev(torch, X)
    Yd = torch.empty_like(Xd)
    Vdense = 1j * W.to_dense()
    c = build_cheby(H, -15.0, 15.0)
    c.apply_dual(Vd, Xd, Yd, scale=-0.25)
    assert rel_err(Yd.cpu().numpy(), -0.25 * (Vdense @ X)) < 1e-13
    cs = build_cheby(H, -15.0, 15.0, Z)
    cs.apply_dual(Vd, Xd, Yd, scale=0.5)
    Zd = Z.to_dense()
    assert rel_err(Yd.cpu().numpy(), 0.5 * (Zd.conj().T @ Vdense @ Zd @ X)) < 1e-12


def test_vbcsr_subset(torch_cuda):
    """The vbcsr pieces the calc layer calls (DistMultiVector algebra,
    BlockSpMat mult / mult_dense_adjoint / duplicate) against numpy."""
    torch = torch_cuda
    from rsatb_b200.vbcsr import DistMultiVector
    rng = np.random.default_rng(31)
    A = random_hermitian_bsr(20, 5, 4, seed=6, complex_values=True)
    Ad = dev_bsr(A)
    n = A.n_rows
    X = _panel(rng, n, 3, True)
    Y = torch.empty(n, 3, dtype=torch.complex128, device="cuda")
    Ad.mult_dense_adjoint(to_dev(torch, X), Y, alpha=0.5)
    assert rel_err(Y.cpu().numpy(), 0.5 * A.to_dense().conj().T @ X) < 1e-13
    x = to_dev(torch, X[:, 0].copy())
    y = torch.empty(n, dtype=torch.complex128, device="cuda")
    Ad.mult(x, y)
    assert rel_err(y.cpu().numpy(), A.to_dense() @ X[:, 0]) < 1e-13
    D = Ad.duplicate()
    D.mult_dense(to_dev(torch, X), Y)
    assert rel_err(Y.cpu().numpy(), A.to_dense() @ X) < 1e-13
    assert Ad.get_block_density() == A.nnz_blocks / (20 * 20)
    a = DistMultiVector(n, 3, data=to_dev(torch, X))
    b = DistMultiVector(n, 3, data=to_dev(torch, _panel(rng, n, 3, True)))
    Bh = b.data.cpu().numpy()
    assert np.allclose(a.bdot(b), (X * Bh).sum(0)) and np.allclose(a.dot(b), (X.conj() * Bh).sum(0))
    a.axpy(2.0, b)
    assert np.allclose(a.data.cpu().numpy(), X + 2.0 * Bh)
    a.swap(b)
    assert np.allclose(a.data.cpu().numpy(), Bh)
    b.set_constant(1.5)
    assert (b.data.cpu().numpy() == 1.5).all()
    a.set_col(1, b.get_col(0))
    assert np.allclose(a.data[:, 1].cpu().numpy(), 1.5) and a(0, 1) == 1.5


# ------------------------------------------------ time propagation, corr DOS

@pytest.mark.parametrize("t", [np.pi, 5 * np.pi, 70 * np.pi, 700 * np.pi, 2000 * np.pi])
def test_timeprop_coeff_matches_oracle(torch_cuda, t):
    """timeprop_coeff (cheby.hpp:85-106): the same truncation length as the
    ascending Bessel evaluation of bessel.hpp, coefficients to 1e-12."""
    from rsatb_b200.calc import timeprop_coeff
    got = timeprop_coeff(t)
    want = oracle.timeprop_coeff(t)
    assert got.size == want.size
    assert np.abs(got - want).max() < 1e-12
    back = timeprop_coeff(t, forward=False)
    assert np.abs(back - np.conj(want)).max() < 1e-12


def test_timeprop_coeff_length_at_production_time(torch_cuda):
    """test_dos.cpp:235-248: at t = 2000 pi the expansion is finite and has
    between 6283 and 7000 terms."""
    from rsatb_b200.calc import timeprop_coeff
    c = timeprop_coeff(2000 * np.pi)
    assert np.all(np.isfinite(c)) and 6283 < c.size < 7000


def test_corr_series_analytic(torch_cuda):
    """test_dos.cpp:150-170: with mu_n = cos(n pi / 3) for even n and 0 for
    odd n, the correlation series is C(t) = cos(t / 2) exactly."""
    from rsatb_b200.calc import corr_dos, corr_moment_count
    nt = 40
    N = corr_moment_count(nt)
    n = np.arange(N)
    mu = np.where(n % 2 == 0, np.cos(n * np.pi / 3), 0.0).astype(np.complex128)
    dos, cdos = corr_dos(mu, nt)
    assert np.abs(cdos - np.cos(0.5 * np.pi * np.arange(nt + 1))).max() < 1e-10
    want, want_c = oracle.corr_dos(mu, nt)
    assert np.abs(cdos - want_c).max() < 1e-12
    assert np.abs(dos - want).max() < 1e-10 * np.abs(want).max()
    with pytest.raises(Exception):
        corr_dos(mu, 0)


def test_corr_series_matches_stepwise_propagation(torch_cuda):
    """test_dos.cpp:171-232: the moment route equals stepwise propagation
    psi_j = e^{-i Op pi} psi_{j-1} (Chebyshev::propagate) with overlaps
    <psi_0|psi_j>, to expansion truncation."""
    torch = torch_cuda
    from rsatb_b200.calc import corr_dos, corr_moment_count, kpm_dos_moments, timeprop_coeff
    from rsatb_b200.vbcsr import set_random
    H = graphene_case(6, 6)
    c = build_cheby(H, -8.7, 8.9)
    R, nt = 3, 24
    psi = torch.empty(H.n_rows, R, dtype=torch.complex128, device="cuda")
    set_random(psi, 31)
    mu = kpm_dos_moments(c, psi, corr_moment_count(nt))
    _, cdos = corr_dos(mu, nt)
    step = timeprop_coeff(np.pi)
    cur = psi.clone()
    nxt = torch.empty_like(psi)
    stepwise = [complex((psi.conj() * psi).sum().item()) / R]
    for _ in range(nt):
        c.propagate(cur, nxt, step)
        cur, nxt = nxt, cur
        stepwise.append(complex((psi.conj() * cur).sum().item()) / R)
    assert np.abs(cdos - np.array(stepwise)).max() < 1e-12
