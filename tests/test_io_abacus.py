"""ABACUS H(R) files (rsatb/io/abacus_csr.hpp) through rsatb_b200.io_abacus.

Synthetic files are written in the three layouts the reference reads (text,
binary, and binary with the older all-zero offsets after an empty R) from
known CSR matrices; they must read back identically, and the images must
carry rsatb's orbital order, sign and units (abacus_convention.hpp: rsatb's
p shell (y, z, x) is (-ABACUS[2], ABACUS[0], -ABACUS[1]) of ABACUS's
(z, -x, -y); Ry -> eV by 13.605698).  On a GPU the images give H(k) through
the device Bloch sum.
"""
from __future__ import annotations

import numpy as np
import pytest

from rsatb_b200 import io_abacus

SHELLS = [[0, 1], [0, 1]]  # two atoms, s + p: 4 orbitals each, n = 8


def _records(complex_values=False, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for shift, density in (((0, 0, 0), 0.6), ((1, 0, 0), 0.3), ((0, 1, 0), 0.0)):
        A = rng.standard_normal((8, 8)) * (rng.random((8, 8)) < density)
        if complex_values:
            A = A + 1j * rng.standard_normal((8, 8)) * (A != 0)
        out.append((shift, A))
    return out


def _csr(A):
    rows, cols = np.nonzero(A)
    rp = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=A.shape[0]))])
    return rp.astype(np.int32), cols.astype(np.int32), A[rows, cols]


def _write_text(path, recs, complex_values=False, step=True):
    lines = ["STEP: 0"] if step else []
    lines += ["Matrix Dimension of H(R): 8", f"Matrix number of H(R): {len(recs)}"]
    for shift, A in recs:
        rp, ci, v = _csr(A)
        lines.append(f"{shift[0]} {shift[1]} {shift[2]} {v.size}")
        if v.size:
            if complex_values:
                lines.append(" ".join(f"({float(x.real)!r},{float(x.imag)!r})" for x in v))
            else:
                lines.append(" ".join(repr(float(x)) for x in v))
            lines.append(" ".join(str(c) for c in ci))
            lines.append(" ".join(str(r) for r in rp))
    path.write_text("\n".join(lines) + "\n")


def _write_binary(path, recs, complex_values=False, old=False):
    parts = [np.array([0, 8, len(recs)], np.int32).tobytes()]
    for shift, A in recs:
        rp, ci, v = _csr(A)
        parts.append(np.array([*shift, v.size], np.int32).tobytes())
        if v.size:
            parts.append(v.astype(np.complex128 if complex_values else np.float64).tobytes())
            parts.append(ci.tobytes())
            parts.append(rp.tobytes())
        elif old:
            parts.append(np.zeros(9, np.int32).tobytes())
    path.write_bytes(b"".join(parts))


def _dense(rec, n=8):
    A = np.zeros((n, n), dtype=rec.values.dtype)
    rows = np.repeat(np.arange(n), np.diff(rec.row_ptr))
    A[rows, rec.col_ind] = rec.values
    return A


@pytest.mark.parametrize("layout", ["text", "text_nostep", "binary", "binary_old"])
def test_layouts_read_back(tmp_path, layout):
    recs = _records()
    path = tmp_path / "data-HR-sparse_SPIN0.csr"
    if layout.startswith("text"):
        _write_text(path, recs, step=layout == "text")
    else:
        _write_binary(path, recs, old=layout == "binary_old")
    n, got = io_abacus.read_hr(path)
    assert n == 8 and len(got) == 3
    for (shift, A), rec in zip(recs, got):
        assert rec.shift == shift
        assert np.array_equal(_dense(rec), A)


def test_complex_values_and_mode_errors(tmp_path):
    recs = _records(complex_values=True, seed=3)
    t, bfile = tmp_path / "c.csr", tmp_path / "c.bin"
    _write_text(t, recs, complex_values=True)
    _write_binary(bfile, recs, complex_values=True)
    for p in (t, bfile):
        n, got = io_abacus.read_hr(p, complex_values=True)
        for (shift, A), rec in zip(recs, got):
            assert np.array_equal(_dense(rec), A)
    with pytest.raises(io_abacus.AbacusFormatError, match="nspin=4"):
        io_abacus.read_hr(t)
    _write_text(t, _records())
    with pytest.raises(io_abacus.AbacusFormatError, match="spin-degenerate"):
        io_abacus.read_hr(t, complex_values=True)
    t.write_text(t.read_text() + "STEP: 1\n")
    with pytest.raises(io_abacus.AbacusFormatError, match="more than one STEP"):
        io_abacus.read_hr(t)


def test_orbital_order_and_images():
    src, sign = io_abacus.abacus_orbital_order([0, 1])
    assert src.tolist() == [0, 3, 1, 2] and sign.tolist() == [1.0, -1.0, 1.0, -1.0]
    src2, sign2 = io_abacus.abacus_orbital_order([1], spin_components=2)
    assert src2.tolist() == [4, 5, 0, 1, 2, 3] and sign2.tolist() == [-1, -1, 1, 1, -1, -1]
    recs = _records()
    hr = [io_abacus.HrRecord(s, *_csr(A)) for s, A in recs]
    pos = np.array([[0.0, 0.0, 0.0], [0.9, 0.9, 0.9]])
    cell = np.eye(3) * 3.5
    rows, cols, shifts, blocks, vecs, n_atoms, b = io_abacus.hr_to_images(8, hr, SHELLS, pos,
                                                                          cell)
    assert n_atoms == 2 and b == 4
    P = np.zeros((8, 8))  # rsatb orbital k of atom a <- sign * ABACUS orbital src
    for a in range(2):
        for k in range(4):
            P[4 * a + k, 4 * a + src[k]] = sign[k]
    for e in range(rows.size):
        A = dict(recs)[tuple(int(x) for x in shifts[e])]
        want = io_abacus.EV_PER_RYDBERG * (P @ A @ P.T)
        i, j = rows[e], cols[e]
        assert np.allclose(blocks[e], want[4 * i:4 * i + 4, 4 * j:4 * j + 4], rtol=0, atol=1e-14)
        assert np.allclose(vecs[e], shifts[e] @ cell + pos[j] - pos[i])
    # every nonzero block of every R is present once
    n_blocks = sum(int(np.count_nonzero(np.abs(A.reshape(2, 4, 2, 4)).sum(axis=(1, 3))))
                   for _, A in recs)
    assert rows.size == n_blocks
    with pytest.raises(ValueError, match="orbitals"):
        io_abacus.hr_to_images(8, hr, [[0, 1], [0]])


@pytest.mark.gpu
def test_images_give_h_of_k_on_the_device():
    import torch
    from rsatb_b200.bloch import ImageOperator
    torch.cuda.set_device(0)
    recs = _records(seed=5)
    # Hermitian H(R): H(-R) = H(R)^T
    full = []
    for s, A in recs:
        full.append((s, A))
        if any(s):
            full.append((tuple(-x for x in s), A.T.copy()))
        else:
            full[-1] = (s, 0.5 * (A + A.T))
    hr = [io_abacus.HrRecord(s, *_csr(A)) for s, A in full]
    rows, cols, shifts, blocks, _, n_atoms, b = io_abacus.hr_to_images(8, hr, SHELLS)
    op = ImageOperator(rows, cols, shifts, blocks, b, n_atoms)
    k = np.array([0.13, 0.27, 0.0])
    Hk = op.at_k(k).to_arrays().to_dense()
    src, sign = io_abacus.abacus_orbital_order([0, 1])
    P = np.zeros((8, 8))
    for a in range(2):
        for kk in range(4):
            P[4 * a + kk, 4 * a + src[kk]] = sign[kk]
    want = sum(np.exp(-2j * np.pi * np.dot(k, s)) * (P @ A @ P.T) for s, A in full)
    assert np.abs(Hk - io_abacus.EV_PER_RYDBERG * want).max() < 1e-12
