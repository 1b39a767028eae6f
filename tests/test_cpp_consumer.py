"""A compiled C++ consumer of the C ABI.

tests/cpp/kpm_consumer.cpp is written against RSATB's calc-layer shapes
(BlockSpMat<T>, DistMultiVector<T>, ISQRTMPreconditioner<T>, Chebyshev<T>
with its Orthogonal and Sandwich constructors, kpm_dos_moments(Chebyshev&,
psi, n)) as provided by include/rsatb_b200.hpp over include/rsatb_b200.h.
It is compiled with g++ here (no GPU needed) and, on a GPU, its moments must
equal the oracle's restatement of kpm_dos_moments to 1e-10 of mu_0.
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
LIBDIR = ROOT / "rsatb_b200" / "_lib"


def build_consumer() -> Path:
    EXE.parent.mkdir(parents=True, exist_ok=True)
    if not (LIBDIR / "librsatb_b200.so").exists():
        from rsatb_b200 import build
        build.build()
    cmd = [shutil.which("g++") or "g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror",
           "-I", str(ROOT / "include"), str(SRC), "-o", str(EXE), "-L", str(LIBDIR),
           "-lrsatb_b200", f"-Wl,-rpath,{LIBDIR}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return EXE


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
