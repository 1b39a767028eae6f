"""Pins the CPU oracle to the reference's own golden vectors and checks.

Each test restates an assertion of the reference's tests (file:line in
the docstring) or compares against a fixture generated from the reference
(tests/golden/make_golden.py).  CPU only.
"""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest

import oracle

GOLDEN = Path(__file__).resolve().parent / "golden"


def diag_model(N=100):
    """rsatb/calc/test/test_dos.cpp:69-100: H = diag(+-0.5), deterministic
    +-1/sqrt(N) sample."""
    h = np.array([0.5 if g % 2 == 0 else -0.5 for g in range(N)])
    H = oracle.Bsr(N, N, 1, np.arange(N + 1), np.arange(N), h.reshape(N, 1, 1))
    psi = np.array([1.0 if (g * 7 + 3) % 5 < 2 else -1.0 for g in range(N)]) / math.sqrt(N)
    return H, psi


@pytest.mark.parametrize("complex_sample", [True, False])
def test_dos_diagonal_model_analytic(complex_sample):
    """test_dos.cpp:102-138: mu_n = cos(n pi/3) (n even), 0 (n odd) to 1e-10;
    doubled == plain to 1e-10; Jackson density integral ~1, peak at 0.5."""
    H, psi = diag_model()
    p = psi.astype(complex if complex_sample else float).reshape(-1, 1)
    op = oracle.make_op(H, 0.0, 1.0)
    n_moments = 64
    mu = oracle.kpm_moments(op, p, n_moments, doubled=True)
    mu_plain = oracle.kpm_moments(op, p, n_moments, doubled=False)
    exact = np.array([math.cos(n * math.pi / 3) if n % 2 == 0 else 0.0 for n in range(n_moments)])
    assert np.abs(mu - exact).max() < 1e-10
    assert np.abs(mu - mu_plain).max() < 1e-10
    n_grid = 400
    x = -1.0 + 2.0 * (np.arange(n_grid) + 0.5) / n_grid
    rho = oracle.density(mu, x, 1.0 / n_grid)
    integral = (rho * 2.0 / n_grid).sum()
    pos = x > 0
    peak = x[pos][np.argmax(rho[pos])]
    assert abs(integral - 1.0) < 0.02
    assert abs(peak - 0.5) < 0.05


def test_jackson_matches_kpm_ref():
    """jackson_kernel (kpm.hpp:18-26) against kpm_ref.jackson."""
    z = np.load(GOLDEN / "kpm_ref_density.npz")
    for m in (1, 2, 7, 64, 513):
        g = oracle.kernel_weights(1, m)
        np.testing.assert_allclose(g, z[f"jackson_{m}"], rtol=0, atol=1e-15)


def test_density_matches_kpm_ref_fixture():
    """Exact-trace KPM density of a seeded spectrum against the reference's
    kpm_ref.kpm_curves (same moment count, inset 0.5/nt, 2*rho)."""
    z = np.load(GOLDEN / "kpm_ref_density.npz")
    eps = z["eps"]
    n = eps.size
    emin, emax, de = float(z["emin"]), float(z["emax"]), float(z["de"])
    center, hw = (emax + emin) / 2, (emax - emin) / 2
    H = oracle.Bsr(n, n, 1, np.arange(n + 1), np.arange(n), eps.reshape(n, 1, 1))
    op = oracle.make_op(H, center, hw)
    psi = np.eye(n)  # R = N unit columns: the column average is the exact trace / N
    n_moments = int(z["n_moments"])
    mu = oracle.kpm_moments(op, psi, n_moments)
    nt = math.ceil((emax - emin) / de)
    i = np.arange(nt)
    x = np.concatenate([(i - nt) / nt, i / nt])
    rho2 = 2.0 * oracle.density(mu, x, 0.5 / nt)
    curve = z["curve"]
    assert np.abs(rho2 - curve).max() <= 1e-10 * np.abs(curve).max()


def test_dct3_fft_route_matches_cosine_sum():
    """test_fftcheb_transport.cpp:511-528: dct_type3_batch == explicit sum to 1e-12."""
    n, batch = 8, 2
    m = np.arange(n)
    x = np.stack([0.1 * (1 + b) * (m + 1) - 0.05j * (2 + b) * (m + 1) for b in range(batch)])
    a = oracle.dct3(x, "fft")
    e = oracle.dct3(x, "direct")
    assert np.abs(a - e).max() < 1e-12


def test_philox_known_answers():
    """Philox-4x32-10 known-answer vectors of the Random123 distribution."""
    cases = [
        ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
        ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
        ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
         [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
    ]
    for ctr, key, want in cases:
        assert list(oracle.philox4x32_10(ctr, key)) == want


def test_sample_vectors_properties():
    """Unit modulus 1/sqrt(N) phases; values keyed by atom id, not row order."""
    ids = np.arange(50) * 3 + 7
    v = oracle.set_random(20240917, 0, True, ids, 2, 100, 4, True)
    np.testing.assert_allclose(np.abs(v) ** 2 * 100, 1.0, rtol=1e-14)
    perm = np.random.default_rng(0).permutation(50)
    w = oracle.set_random(20240917, 0, True, ids[perm], 2, 100, 4, True)
    np.testing.assert_array_equal(w.reshape(50, 2, 4), v.reshape(50, 2, 4)[perm])
    r = oracle.set_random(5, 1, True, ids, 2, 100, 3, False)
    assert set(np.unique(r * 10)) <= {-1.0, 1.0}
    u = oracle.set_random(5, 2, False, ids, 2, 100, 3, True)
    assert np.all(np.abs(u.real) <= 1) and np.all(np.abs(u.imag) <= 1)
    # phases are spread over the circle
    ang = np.angle(v.ravel())
    assert np.histogram(ang, bins=4, range=(-np.pi, np.pi))[0].min() > 40


# ---------------------------------------------------------------- transport

def _toy(name):
    d = json.loads((GOLDEN / "fftcheb_toys.json").read_text())[name]

    def mat(k):
        a = np.array(d[k])
        return a[..., 0] + 1j * a[..., 1]
    return {k: mat(k) for k in d}


def moment_reference(H, V, sample, M, formulation, center=0.0, hw=1.0):
    """Independent O(M^2) moment-sum reference, restating
    test_fftcheb_transport.cpp:157-360 (build_reference_sequences and
    reference_spectrum) with dense numpy matrices (orthogonal form)."""
    Hs = (H - center * np.eye(H.shape[0])) / hw
    vs = 1.0 / (2.0 * hw)
    right = [[None] * M for _ in range(3)]
    left = [[None] * M for _ in range(3)]
    r_prev = [-vs * V[a] @ sample for a in range(3)]
    lb_prev = sample.copy()
    for a in range(3):
        right[a][0] = r_prev[a]
        left[a][0] = -vs * V[a] @ lb_prev
    if M > 1:
        r_curr = [Hs @ r_prev[a] for a in range(3)]
        lb_curr = Hs @ lb_prev
        for a in range(3):
            right[a][1] = r_curr[a]
            left[a][1] = -vs * V[a] @ lb_curr
    for m in range(2, M):
        r_next = [2 * Hs @ r_curr[a] - r_prev[a] for a in range(3)]
        lb_next = 2 * Hs @ lb_curr - lb_prev
        for a in range(3):
            right[a][m] = r_next[a]
            left[a][m] = -vs * V[a] @ lb_next
        r_prev, r_curr = r_curr, r_next
        lb_prev, lb_curr = lb_curr, lb_next
    g = oracle.kernel_weights(1, M)
    gm = 2.0 * g / (np.pi * (1.0 + (np.arange(M) == 0)))
    k = np.arange(M)
    eps_native = np.cos(np.pi * (k + 0.5) / M)
    comp = {(0, 0): 0, (0, 1): 1, (0, 2): 2, (1, 1): 3, (1, 2): 4, (2, 2): 5}
    result = np.zeros((M, 6))
    if formulation == 0:
        kern = np.zeros((M, 6))
        for a in range(3):
            D = np.array([[np.vdot(left[a][m], right[a][n]).real for n in range(M)]
                          for m in range(M)])
            for kk in range(M):
                e = eps_native[kk]
                T = np.cos(np.arange(M) * np.arccos(e))
                w = gm * T
                kern[kk, comp[(a, a)]] = (w @ D @ w) / max(1e-14, 1 - e * e)
        result = kern[::-1].copy()
        return result
    kern = np.zeros((M, 6), dtype=complex)
    for kk in range(M):
        theta = np.pi * (kk + 0.5) / M
        eps, root = np.cos(theta), np.sin(theta)
        m = np.arange(M)
        w1 = gm * np.exp(1j * m * theta)
        w2 = m * w1
        w3 = gm * np.cos(m * theta)
        phi = {}
        for a in range(3):
            L = np.array(left[a])
            R = np.array(right[a])
            phi[("l", 1, a)], phi[("l", 2, a)], phi[("l", 3, a)] = w1 @ L, w2 @ L, w3 @ L
            phi[("r", 1, a)], phi[("r", 2, a)], phi[("r", 3, a)] = w1 @ R, w2 @ R, w3 @ R
        for a in range(3):
            for b in range(a, 3):
                val = eps * (np.vdot(phi[("l", 3, a)], phi[("r", 1, b)]) +
                             np.vdot(phi[("l", 1, a)], phi[("r", 3, b)])) + \
                    1j * root * (np.vdot(phi[("l", 2, a)], phi[("r", 3, b)]) -
                                 np.vdot(phi[("l", 3, a)], phi[("r", 2, b)]))
                kern[kk, comp[(a, b)]] = val
    eps_sorted = eps_native[::-1]
    running = np.zeros(6)
    prev = np.zeros(6)
    for kk in range(M):
        integrand = (1j * kern[M - 1 - kk]).real
        if kk > 0:
            running = running + 0.5 * (prev + integrand) * (eps_sorted[kk] - eps_sorted[kk - 1])
        result[kk] = running
        prev = integrand
    return result


def _toy_op(t):
    H = oracle.Bsr.from_dense(t["H"])
    V = [oracle.Bsr.from_dense(t[k]) for k in ("Vx", "Vy", "Vz")]
    return H, V


@pytest.mark.parametrize("name,form,M", [("greenwood", 0, 12), ("bastin", 1, 12)])
def test_fftcheb_matches_moment_reference(name, form, M):
    """test_fftcheb_transport.cpp:530-560: fftcheb == O(M^2) reference to 1e-8
    (orthogonal form, window [-1, 1], sample_a)."""
    t = _toy(name)
    H, V = _toy_op(t)
    op = oracle.make_op(H, 0.0, 1.0)
    s = t["sample_a"].reshape(-1, 1)
    sigma, energy = oracle.fftcheb(op, V, s, M, formulation=form, prefactor=1.0)
    ref = moment_reference(t["H"], [t["Vx"], t["Vy"], t["Vz"]], s[:, 0], M, form)
    assert np.abs(sigma - ref).max() < 1e-8
    assert np.all(np.diff(energy) > 0)


def test_fftcheb_partition_and_sample_average():
    """test_fftcheb_transport.cpp:572-600: partitioned == unpartitioned, and a
    two-sample block == the average of single-sample runs."""
    t = _toy("bastin")
    H, V = _toy_op(t)
    op = oracle.make_op(H, 0.0, 1.0)
    a = t["sample_a"].reshape(-1, 1)
    b = t["sample_b"].reshape(-1, 1)
    for form in (0, 1):
        s1, _ = oracle.fftcheb(op, V, a, 10, formulation=form, sections=1)
        s2, _ = oracle.fftcheb(op, V, a, 10, formulation=form, sections=2)
        assert np.abs(s1 - s2).max() < 1e-12
        sb, _ = oracle.fftcheb(op, V, b, 10, formulation=form)
        sab, _ = oracle.fftcheb(op, V, np.hstack([a, b]), 10, formulation=form)
        assert np.abs(sab - 0.5 * (s1 + sb)).max() < 1e-12


def test_sandwich_equals_orthogonal_on_transformed_operator():
    """Sandwich Z^H H Z with Z = S^-1/2 against the orthogonal form on the
    explicitly transformed matrices (moments and transport)."""
    t = _toy("greenwood")
    w, U = np.linalg.eigh(t["S"])
    Z = U @ np.diag(w ** -0.5) @ U.conj().T
    Hp = Z.conj().T @ t["H"] @ Z
    Vp = [Z.conj().T @ t[k] @ Z for k in ("Vx", "Vy", "Vz")]
    Hb, Zb, ZHb = (oracle.Bsr.from_dense(m) for m in (t["H"], Z, Z.conj().T))
    op_s = oracle.make_op(Hb, 0.1, 1.5, Zb, ZHb)
    op_o = oracle.make_op(oracle.Bsr.from_dense(Hp), 0.1, 1.5)
    s = np.stack([t["sample_a"], t["sample_b"]], 1)
    mu_s = oracle.kpm_moments(op_s, s, 20)
    mu_o = oracle.kpm_moments(op_o, s, 20)
    assert np.abs(mu_s - mu_o).max() < 1e-12
    Vb = [oracle.Bsr.from_dense(t[k]) for k in ("Vx", "Vy", "Vz")]
    sig_s, _ = oracle.fftcheb(op_s, Vb, s, 10)
    sig_o, _ = oracle.fftcheb(op_o, [oracle.Bsr.from_dense(v) for v in Vp], s, 10)
    assert np.abs(sig_s - sig_o).max() < 1e-10


def test_dense_ns_chain_cases():
    """rsatb/calc/test/test_isqrtm.cpp:132-186 on the dense restatement: the
    0.6 chain is indefinite and diverges, 0.49 converges, a 1-step cap is
    neither converged nor diverged."""
    n = 24

    def chain(off):
        return np.eye(n) + off * (np.eye(n, k=1) + np.eye(n, k=-1))

    _, r = oracle.ns_inverse_sqrt_dense(chain(0.60), 1e-10, 20)
    assert r["diverged"] and not r["converged"]
    Z, r = oracle.ns_inverse_sqrt_dense(chain(0.49), 1e-10, 20)
    assert r["converged"] and not r["diverged"]
    assert np.abs(Z @ chain(0.49) @ Z.T - np.eye(n)).max() < 1e-9
    _, r = oracle.ns_inverse_sqrt_dense(chain(0.49), 1e-16, 1)
    assert r["hit_maxiter"] and not r["converged"] and not r["diverged"]


def test_dense_ns_and_eigen_route_agree_on_exact_construction():
    """Q diag(lambda) Q^T problems (benchmark_isqrt_action.cpp:53-140): the
    NS restatement and the clamped eigen action both reproduce the exact
    Q diag(lambda^-1/2) Q^T."""
    rng = np.random.default_rng(4)
    for n, kappa in ((40, 1e2), (90, 1e5)):
        lam = np.logspace(-np.log10(kappa), 0.0, n)
        Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
        A = (Q * lam) @ Q.T
        A = 0.5 * (A + A.T)
        exact = (Q / np.sqrt(lam)) @ Q.T
        ref = np.linalg.norm(exact)
        assert np.linalg.norm(oracle.isqrt_columns_eigen(A) - exact) / ref < 1e-10
        Z, r = oracle.ns_inverse_sqrt_dense(A)
        assert r["converged"]
        assert np.linalg.norm(Z - exact) / ref < 1e-10


def test_oracle_corr_series_analytic():
    """test_dos.cpp:150-170 pins the correlation route: mu_n = cos(n pi / 3)
    (even n), 0 (odd n) gives C(t) = cos(t / 2) at t = j pi."""
    nt = 30
    N = oracle.timeprop_coeff(nt * np.pi).size
    n = np.arange(N)
    mu = np.where(n % 2 == 0, np.cos(n * np.pi / 3), 0.0)
    cd = oracle.corr_from_moments(mu, nt)
    assert np.abs(cd - np.cos(0.5 * np.pi * np.arange(nt + 1))).max() < 1e-10


def test_oracle_timeprop_length():
    """test_dos.cpp:235-248: 6283 < terms(2000 pi) < 7000, all finite; the
    forward and backward expansions are conjugate."""
    c = oracle.timeprop_coeff(2000 * np.pi)
    assert 6283 < c.size < 7000 and np.all(np.isfinite(c))
    b = oracle.timeprop_coeff(3.0, forward=False)
    assert np.allclose(b, np.conj(oracle.timeprop_coeff(3.0)), rtol=0, atol=1e-16)


def test_oracle_integrate_dc_linear_spectrum():
    """integrate_dc_spectrum is exact for a piecewise-linear spectrum: a
    linear sigma(E) = a + b E gives a + b mu at any T once the grid covers
    the -df/dE window; T = 0 interpolates."""
    e = np.linspace(-12.0, 12.0, 961)   # -df/dE below 1e-16 at the ends up to 3000 K
    a = np.arange(1.0, 7.0)
    b = np.linspace(-0.5, 0.5, 6)
    s = a[None, :] + e[:, None] * b[None, :]
    for T in (0.0, 30.0, 300.0, 3000.0):
        got = oracle.integrate_dc_spectrum(s, e, 0.37, T)
        assert np.abs(got - (a + 0.37 * b)).max() < 1e-10


# ------------------------------------------------- exact diagonalisation (ED)

def test_kubo_greenwood_ed_matches_the_reference_ed_sum():
    """oracle.kubo_greenwood_ed against the reference's own exact-
    diagonalisation Kubo-Greenwood sum (make_ref_curves.py delta_matrix on
    the Chebyshev-node grid, committed by tests/golden/make_golden.py):
    4N K(E_k) = sum_nm |V_nm|^2 dJ dJ to 1e-12 relative, on the grid whose
    window the reference's window_from_cheb_grid recovers exactly."""
    z = np.load(GOLDEN / "ed_greenwood.npz")
    H, V = z["H"], z["V"]
    c, hw, M = float(z["center"]), float(z["half_width"]), int(z["n_moments"])
    E, K = oracle.kubo_greenwood_ed(H, V, c, hw, M)
    assert np.allclose(z["window"], [c, hw], rtol=0, atol=1e-12)
    assert np.abs(E - z["energy"]).max() < 1e-13
    assert np.array_equal(oracle.kernel_weights(1, M), z["jackson"]) or \
        np.abs(oracle.kernel_weights(1, M) - z["jackson"]).max() < 1e-15
    ref = z["kg_sum"]
    assert np.abs(4 * H.shape[0] * K - ref).max() <= 1e-12 * np.abs(ref).max()


def test_kpm_moments_ed_equals_the_recurrence():
    """The ED moments (eigen-decomposition, T_n at the eigenvalues) against
    the oracle's Chebyshev recurrence (doubled and plain) on a small
    complex-Hermitian BSR operator with complex sample columns."""
    rng = np.random.default_rng(4)
    n = 60
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    A = 0.1 * (A + A.conj().T)
    A[np.abs(A) < 0.12] = 0.0
    bound = float(np.abs(np.linalg.eigvalsh(A)).max()) + 0.3
    psi = rng.standard_normal((n, 5)) + 1j * rng.standard_normal((n, 5))
    rows, cols = np.nonzero(A)
    row_ptr = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=n))]).astype(np.int32)
    Hb = oracle.Bsr(n, n, 1, row_ptr, cols.astype(np.int32),
                    A[rows, cols].reshape(-1, 1, 1))
    op = oracle.make_op(Hb, 0.05, bound)
    want = oracle.kpm_moments_ed(A, psi, 0.05, bound, 64)
    for doubled in (True, False):
        got = oracle.kpm_moments(op, psi, 64, doubled=doubled)
        assert np.abs(got - want).max() <= 1e-11 * np.abs(want[0])


# ------------------------------------------- sparse Newton-Schulz refinement

def test_ns_refine_dense_keeps_test_isqrtm_chain_semantics():
    """The dense restatement of inverse_sqrt's loop from the graph-local seed
    on test_isqrtm.cpp's 24-site chains: off-diagonal 0.6 (indefinite) is
    reported DIVERGED, 0.49 converges to tol 1e-10, and one step towards an
    unreachable tol is capped (neither converged nor diverged)."""
    def run(off, maxit, tol):
        S, rp, ci = oracle.chain_overlap(24, 1.0, off)
        Z0 = oracle.graph_seed_dense(S, rp, ci, 1)
        return oracle.ns_refine_dense(S, Z0, 1, tol=tol, maxit=maxit)

    _, r = run(0.60, 20, 1e-10)
    assert not r["converged"] and r["diverged"]
    Z, r = run(0.49, 20, 1e-10)
    assert r["converged"] and not r["diverged"]
    S, _, _ = oracle.chain_overlap(24, 1.0, 0.49)
    assert np.abs(Z.T @ S @ Z - np.eye(24)).max() < 1e-9
    _, r = run(0.49, 1, 1e-16)
    assert not r["converged"] and not r["diverged"] and r["hit_maxiter"]


def test_qe_restatement_equals_fftcheb_greenwood():
    """oracle.qe_dense (accumulate_qe_block restated) against the oracle's
    fftcheb Greenwood route, itself pinned to test_fftcheb_transport.cpp's
    toys: the same bilinear form, equal to rounding on every node and on a
    window (zero outside it)."""
    rng = np.random.default_rng(14)
    n, R, M = 24, 3, 40
    H = rng.standard_normal((n, n)) * 0.3
    H = H + H.T
    W = [rng.standard_normal((n, n)) * 0.2 for _ in range(3)]
    W = [w - w.T for w in W]                  # V_a = i W_a, imaginary Hermitian
    psi = np.exp(2j * np.pi * rng.random((n, R))) / np.sqrt(n)
    bound = float(np.abs(np.linalg.eigvalsh(H)).max()) + 0.5
    op = oracle.make_op(oracle.Bsr.from_dense(H), 0.0, bound)
    Vb = [oracle.Bsr.from_dense(w, imag=True) for w in W]
    want, en = oracle.fftcheb(op, Vb, psi, M)
    got, en2 = oracle.qe_dense(H, [1j * w for w in W], psi, 0.0, bound, M)
    assert np.abs(en - en2).max() < 1e-13
    assert np.abs(got - want).max() <= 1e-11 * np.abs(want).max()
    nodes = np.array([3, 11, 12, 30])
    win, _ = oracle.qe_dense(H, [1j * w for w in W], psi, 0.0, bound, M, nodes)
    assert np.abs(win[nodes] - want[nodes]).max() <= 1e-11 * np.abs(want).max()
    assert np.all(np.delete(win, nodes, axis=0) == 0.0)
