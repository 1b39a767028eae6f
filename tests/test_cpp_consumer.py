"""Compiled C++ consumers of the C ABI.

tests/cpp/kpm_consumer.cpp is written against RSATB's calc-layer shapes
(BlockSpMat<T>, DistMultiVector<T>, ISQRTMPreconditioner<T>, Chebyshev<T>
with its Orthogonal and Sandwich constructors, kpm_dos_moments(Chebyshev&,
psi, n)) as provided by include/rsatb_b200.hpp over include/rsatb_b200.h.
It is compiled with g++ here (no GPU needed) and, on a GPU, its moments must
equal the oracle's restatement of kpm_dos_moments to 1e-10 of mu_0.

tests/cpp/calc_consumer.cpp drives the rest of the C++ layer:
Chebyshev<double>::propagate, apply_dual and compute_moments, the spectral-
bounds Lanczos and the sparse inverse_sqrt refinement; its results are
checked against dense numpy references of the same operators.
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
SRC = ROOT / "tests" / "cpp" / "kpm_consumer.cpp"
EXE = ROOT / "_build" / "kpm_consumer"
CALC_SRC = ROOT / "tests" / "cpp" / "calc_consumer.cpp"
CALC_EXE = ROOT / "_build" / "calc_consumer"
LIBDIR = ROOT / "rsatb_b200" / "_lib"


def build_consumer(src: Path = SRC, exe: Path = EXE) -> Path:
    exe.parent.mkdir(parents=True, exist_ok=True)
    if not (LIBDIR / "librsatb_b200.so").exists():
        from rsatb_b200 import build
        build.build()
    cmd = [shutil.which("g++") or "g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror",
           "-I", str(ROOT / "include"), str(src), "-o", str(exe), "-L", str(LIBDIR),
           "-lrsatb_b200", f"-Wl,-rpath,{LIBDIR}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def write_input(path: Path, H, Z, emin, emax, R, n_moments, orbitals, seed):
    with open(path, "wb") as f:
        np.array([H.n_block_rows, H.block_size, H.nnz_blocks, Z is not None, R, n_moments,
                  orbitals], dtype=np.int32).tofile(f)
        np.array([emin, emax], dtype=np.float64).tofile(f)
        np.array([seed], dtype=np.uint64).tofile(f)
        np.asarray(H.row_ptr, dtype=np.int32).tofile(f)
        np.asarray(H.col_ind, dtype=np.int32).tofile(f)
        np.ascontiguousarray(H.values, dtype=np.float64).tofile(f)
        if Z is not None:
            np.ascontiguousarray(Z.values, dtype=np.float64).tofile(f)


def test_consumer_compiles_against_the_headers():
    exe = build_consumer()
    assert exe.exists()
    # Without an input it prints its usage and exits 2; it loads the library.
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 2 and "usage" in out.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("sandwich", [False, True])
def test_consumer_moments_match_the_oracle(tmp_path, sandwich):
    import oracle
    from rsatb_b200 import lattice
    exe = build_consumer()
    H, S = lattice.diamond_lcao(L=2, seed=3)
    Z = None
    if sandwich:
        Z = lattice.BsrArrays(S.row_ptr, S.col_ind,
                              oracle.graph_inverse_sqrt_eigen(S.row_ptr, S.col_ind, S.values, 8,
                                                              workers=1), 8)
    emin, emax, R, M, seed = -14.0, 14.0, 12, 96, 20240917
    write_input(tmp_path / "in.bin", H, Z, emin, emax, R, M, 8, seed)
    out = subprocess.run([str(exe), str(tmp_path / "in.bin")], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    d = json.loads(out.stdout)
    got = np.array(d["moments_re"]) + 1j * np.array(d["moments_im"])
    Hb = oracle.Bsr(H.n_block_rows, H.n_block_rows, 8, H.row_ptr, H.col_ind, H.values)
    c, hw = (emax + emin) / 2, (emax - emin) / 2
    if sandwich:
        Zb = oracle.Bsr(Z.n_block_rows, Z.n_block_rows, 8, Z.row_ptr, Z.col_ind, Z.values)
        op = oracle.make_op(Hb, c, hw, Zb, oracle.bsr_adjoint(Zb))
    else:
        op = oracle.make_op(Hb, c, hw)
    psi = oracle.set_random(seed, 1, True, np.arange(H.n_block_rows), 8, H.n_rows, R, False)
    want = oracle.kpm_moments(op, psi, M)
    assert np.abs(got - want).max() <= 1e-10 * abs(want[0])


def test_calc_consumer_compiles_against_the_headers():
    exe = build_consumer(CALC_SRC, CALC_EXE)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 2 and "usage" in out.stderr


def _cheb_series(Ht, X, coeffs):
    """sum_n Re(c_n) T_n(Ht) X (a real panel takes Re(c_n))."""
    t0, t1 = X, Ht @ X
    Y = coeffs[0].real * t0 + (coeffs[1].real * t1 if len(coeffs) > 1 else 0)
    for c in coeffs[2:]:
        t0, t1 = t1, 2 * Ht @ t1 - t0
        Y = Y + c.real * t1
    return Y


@pytest.mark.gpu
def test_calc_consumer_matches_dense_references(tmp_path):
    """propagate and apply_dual to 1e-10 of the dense results, the plain
    moments to 1e-10 of mu_0, the Lanczos extremes to 1e-6 of the spectral
    radius, and the refined Z with ||Z^T S Z psi - psi|| / ||psi|| <= 1e-8."""
    import oracle
    from rsatb_b200 import lattice
    exe = build_consumer(CALC_SRC, CALC_EXE)
    H, S = lattice.diamond_lcao(L=2, seed=3)
    V, _ = lattice.diamond_lcao(L=2, seed=4)
    for A in (S, V):
        assert np.array_equal(A.row_ptr, H.row_ptr) and np.array_equal(A.col_ind, H.col_ind)
    Z0 = oracle.graph_inverse_sqrt_eigen(S.row_ptr, S.col_ind, S.values, 8, workers=1)
    emin, emax, scale, R, M, seed = -14.0, 14.0, -0.37, 4, 24, 7
    coeffs = np.array([0.5, 0.25 - 0.1j, -0.3, 0.125j, 0.2, -0.05 + 0.02j])
    with open(tmp_path / "in.bin", "wb") as f:
        np.array([H.n_block_rows, 8, H.nnz_blocks, R, coeffs.size, M], dtype=np.int32).tofile(f)
        np.array([emin, emax, scale], dtype=np.float64).tofile(f)
        np.array([seed], dtype=np.uint64).tofile(f)
        np.asarray(H.row_ptr, dtype=np.int32).tofile(f)
        np.asarray(H.col_ind, dtype=np.int32).tofile(f)
        for vals in (H.values, V.values, S.values, Z0):
            np.ascontiguousarray(vals, dtype=np.float64).tofile(f)
        np.stack([coeffs.real, coeffs.imag], axis=1).astype(np.float64).tofile(f)
    out = subprocess.run([str(exe), str(tmp_path / "in.bin")], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    d = json.loads(out.stdout)
    Hd, Vd = H.to_dense(), V.to_dense()
    n = Hd.shape[0]
    psi = oracle.set_random(seed, 1, True, np.arange(H.n_block_rows), 8, n, R, False)
    c, hw = (emax + emin) / 2, (emax - emin) / 2
    Ht = (Hd - c * np.eye(n)) / hw
    want = _cheb_series(Ht, psi, coeffs)
    got = np.array(d["propagate"]).reshape(n, R)
    assert np.abs(got - want).max() <= 1e-10 * np.abs(want).max()
    got = np.array(d["apply_dual"]).reshape(n, R)
    want = scale * Vd @ psi
    assert np.abs(got - want).max() <= 1e-10 * np.abs(want).max()
    mu = np.array(d["moments"])
    t0, t1 = psi, Ht @ psi
    ref = [np.mean(np.sum(psi * t0, 0)), np.mean(np.sum(psi * t1, 0))]
    for _ in range(M - 2):
        t0, t1 = t1, 2 * Ht @ t1 - t0
        ref.append(np.mean(np.sum(psi * t1, 0)))
    assert np.abs(mu - np.array(ref)).max() <= 1e-10 * abs(ref[0])
    w = np.linalg.eigvalsh(Hd)
    tmin, tmax, _, _, _, conv = d["lanczos"]
    radius = np.abs(w).max()
    assert conv == 1.0
    assert abs(tmin - w[0]) <= 1e-6 * radius and abs(tmax - w[-1]) <= 1e-6 * radius
    steps, converged, residual, nnz, nnz_pattern, check = d["refine"]
    assert converged == 1.0 and residual <= 1e-10 and nnz == nnz_pattern and nnz > 0
    assert check <= 1e-8


TRANSPORT_SRC = ROOT / "tests" / "cpp" / "transport_consumer.cpp"
TRANSPORT_EXE = ROOT / "_build" / "transport_consumer"


def test_transport_consumer_compiles_against_the_headers():
    exe = build_consumer(TRANSPORT_SRC, TRANSPORT_EXE)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 2 and "usage" in out.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("formulation", [0, 1])
def test_transport_consumer_matches_the_oracle(tmp_path, formulation):
    """calc::dc_spectrum_fftcheb from C++ (complex H and V_a = i W_a) against
    the oracle's restatement of dc_spectrum_fftcheb with the real H and the
    imaginary-unit velocities, Greenwood and Bastin, to 1e-10."""
    import oracle
    from _util import to_oracle
    from rsatb_b200 import lattice
    exe = build_consumer(TRANSPORT_SRC, TRANSPORT_EXE)
    H, pos, cell, disp = lattice.twisted_bilayer_graphene(m=1, tiles=(4, 4))
    V = lattice.commutator_velocity(H, disp)
    w = np.linalg.eigvalsh(H.to_dense())
    emin, emax, R, M = w[0] - 0.5, w[-1] + 0.5, 3, 33
    rng = np.random.default_rng(5)
    psi = np.exp(2j * np.pi * rng.random((H.n_rows, R))) / np.sqrt(H.n_rows)
    with open(tmp_path / "in.bin", "wb") as f:
        np.array([H.n_block_rows, H.block_size, H.nnz_blocks, R, M, formulation],
                 dtype=np.int32).tofile(f)
        np.array([emin, emax], dtype=np.float64).tofile(f)
        np.asarray(H.row_ptr, dtype=np.int32).tofile(f)
        np.asarray(H.col_ind, dtype=np.int32).tofile(f)
        for A in (H, *V):
            np.ascontiguousarray(A.values, dtype=np.float64).tofile(f)
        np.ascontiguousarray(psi, dtype=np.complex128).view(np.float64).tofile(f)
    out = subprocess.run([str(exe), str(tmp_path / "in.bin")], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    d = json.loads(out.stdout)
    sig = np.array(d["sigma"]).reshape(M, 6)
    c, hw = (emax + emin) / 2, (emax - emin) / 2
    op = oracle.make_op(to_oracle(H), c, hw)
    sig_o, en_o = oracle.fftcheb(op, [to_oracle(v, imag=True) for v in V], psi, M,
                                 formulation=formulation, prefactor=1.0, sections=1)
    assert np.allclose(np.array(d["energy"]), en_o, rtol=0, atol=1e-13)
    assert np.linalg.norm(sig - sig_o) <= 1e-10 * np.linalg.norm(sig_o)
