"""ABACUS sparse H(R) / S(R) files (``out_mat_hs2 1``) as real-space images.

The reader of rsatb/io/abacus_csr.hpp, restated for the host side of this
package: it parses the file (text or binary) into one n x n CSR matrix per
lattice vector R, and ``hr_to_images`` cuts those into atom blocks, puts each
block into rsatb's orbital order and units (abacus_convention.hpp), and
returns the bond list that ``bloch.ImageOperator`` sums into H(k) on the
device.

File layout (abacus_csr.hpp:4-30):

* text: an optional ``STEP: s`` line (ABACUS >= 3.0), ``Matrix Dimension of
  H(R): n``, ``Matrix number of H(R): nR``, then per R the line
  ``Rx Ry Rz nnz`` and, when nnz > 0, nnz values, nnz column indices and n + 1
  row offsets; a value is ``x`` (spin-degenerate run) or ``(re,im)`` (nspin =
  4, spin interleaved inside each orbital);
* binary: int32 step, n, nR; per R int32 Rx, Ry, Rz, nnz and, when nnz > 0,
  nnz values (float64, or two float64 per complex value), nnz int32 columns,
  n + 1 int32 row offsets.  An R with nnz = 0 is followed by nothing, or (in
  older ABACUS versions) by an all-zero offset array; both are accepted.

Rows and columns run over the whole basis, atom by atom in structure order.
Energies are in Rydberg and are converted with ABACUS's own factor.  Inside
a shell ABACUS orders m as 0, +1, -1, +2, -2, ... and its real harmonics
carry the Condon-Shortley phase, so rsatb's orbital m of a shell is (-1)^m
times ABACUS's orbital at position (0 for m = 0, 2m - 1 for m > 0, 2|m| for
m < 0) of the same shell (abacus_convention.hpp:41-75).
"""
from __future__ import annotations

import dataclasses
import re
from pathlib import Path

import numpy as np

EV_PER_RYDBERG = 13.605698  # ABACUS's Ry -> eV factor (abacus_convention.hpp:39)


@dataclasses.dataclass
class HrRecord:
    """One lattice vector's n x n CSR matrix."""
    shift: tuple
    row_ptr: np.ndarray
    col_ind: np.ndarray
    values: np.ndarray


class AbacusFormatError(ValueError):
    pass


def _looks_binary(raw: bytes) -> bool:
    head = raw[:64]
    return not head.lstrip()[:4] in (b"STEP", b"Matr")


def _parse_value(tok: str, complex_values: bool):
    if tok.startswith("("):
        if not complex_values:
            raise AbacusFormatError("the file holds complex '(re,im)' values, as an nspin=4 run "
                                    "writes; read it with complex_values=True")
        m = re.fullmatch(r"\(([^,]+),([^)]+)\)", tok)
        if not m:
            raise AbacusFormatError(f"malformed complex value {tok!r}")
        return complex(float(m.group(1)), float(m.group(2)))
    if complex_values:
        raise AbacusFormatError(f"read as spinor (nspin=4) but holds {tok!r}: it is from a "
                                "spin-degenerate run")
    return float(tok)


def _read_text(text: str, complex_values: bool):
    toks = text.split()
    pos = 0

    def nxt(what):
        nonlocal pos
        if pos >= len(toks):
            raise AbacusFormatError(f"the file ends before {what}")
        pos += 1
        return toks[pos - 1]

    def integer_after(word):
        seen = False
        while True:
            t = nxt("the header")
            if t == word:
                seen = True
                continue
            if re.fullmatch(r"-?\d+", t):
                if not seen:
                    raise AbacusFormatError(f"expected the '{word}' header line")
                return int(t)

    if toks and toks[0].startswith("STEP"):
        nxt("the header")
        if toks[0] == "STEP:" or toks[0] == "STEP":
            nxt("the step number")
    n = integer_after("Dimension")
    n_rec = integer_after("number")
    if n <= 0 or n_rec < 0:
        raise AbacusFormatError("bad dimension or R count")
    records = []
    for _ in range(n_rec):
        shift = tuple(int(nxt("an R vector")) for _ in range(3))
        nnz = int(nxt("a nonzero count"))
        if nnz > 0:
            vals = np.array([_parse_value(nxt("the values"), complex_values) for _ in range(nnz)])
            cols = np.array([int(nxt("the columns")) for _ in range(nnz)], dtype=np.int32)
            rp = np.array([int(nxt("the row offsets")) for _ in range(n + 1)], dtype=np.int32)
        else:
            vals = np.zeros(0, np.complex128 if complex_values else np.float64)
            cols = np.zeros(0, np.int32)
            rp = np.zeros(n + 1, np.int32)
        records.append(HrRecord(shift, rp, cols, vals))
    if pos < len(toks):
        extra = toks[pos]
        raise AbacusFormatError("the file holds more than one STEP (an MD run); split it"
                                if extra.startswith("STEP") else f"trailing data {extra!r}")
    return n, records


def _read_binary(raw: bytes, complex_values: bool):
    at = 0

    def ints(k):
        nonlocal at
        if at + 4 * k > len(raw):
            raise AbacusFormatError("the file ends inside a record")
        out = np.frombuffer(raw, dtype=np.int32, count=k, offset=at)
        at += 4 * k
        return out

    _step, n, n_rec = (int(x) for x in ints(3))
    if n <= 0 or n_rec < 0:
        raise AbacusFormatError("bad dimension or R count")
    vsize = 16 if complex_values else 8
    records = []
    for r in range(n_rec):
        rx, ry, rz, nnz = (int(x) for x in ints(4))
        if nnz > 0:
            if at + vsize * nnz > len(raw):
                raise AbacusFormatError("the file ends inside a record")
            vals = np.frombuffer(raw, dtype=np.complex128 if complex_values else np.float64,
                                 count=nnz, offset=at).copy()
            at += vsize * nnz
            cols = ints(nnz).copy()
            rp = ints(n + 1).copy()
        else:
            # Older ABACUS wrote an all-zero offset array after an empty R.
            if at + 4 * (n + 1) <= len(raw) and r < n_rec - 1:
                peek = np.frombuffer(raw, dtype=np.int32, count=n + 1, offset=at)
                if not peek.any():
                    at += 4 * (n + 1)
            elif at + 4 * (n + 1) == len(raw):
                at += 4 * (n + 1)
            vals = np.zeros(0, np.complex128 if complex_values else np.float64)
            cols = np.zeros(0, np.int32)
            rp = np.zeros(n + 1, np.int32)
        records.append(HrRecord((rx, ry, rz), rp, cols, vals))
    if at != len(raw):
        raise AbacusFormatError("trailing data after the last R record")
    return n, records


def read_hr(path, binary: bool | None = None, complex_values: bool = False):
    """(n, [HrRecord]) of an ABACUS H(R) or S(R) file; binary is detected
    from the first bytes when not given."""
    raw = Path(path).read_bytes()
    if binary is None:
        binary = _looks_binary(raw)
    n, recs = (_read_binary(raw, complex_values) if binary
               else _read_text(raw.decode(), complex_values))
    for rec in recs:
        if rec.row_ptr[-1] != rec.values.size or np.any(np.diff(rec.row_ptr) < 0):
            raise AbacusFormatError(f"R {rec.shift}: row offsets do not match nnz")
        if rec.col_ind.size and (rec.col_ind.min() < 0 or rec.col_ind.max() >= n):
            raise AbacusFormatError(f"R {rec.shift}: column index out of range")
    return n, recs


def abacus_orbital_order(shells, spin_components: int = 1):
    """(source, sign) of MakeAbacusOrbitalOrder (abacus_convention.hpp:
    51-75): rsatb orbital k of one atom is sign[k] times ABACUS orbital
    source[k]; shells are the atom's angular momenta in block order."""
    source, sign = [], []
    offset = 0
    for l in shells:
        if l < 0:
            raise ValueError("negative angular momentum in a basis shell")
        for m in range(-l, l + 1):
            pos = 0 if m == 0 else (2 * m - 1 if m > 0 else 2 * (-m))
            for s in range(spin_components):
                source.append(spin_components * (offset + pos) + s)
                sign.append(1.0 if abs(m) % 2 == 0 else -1.0)
        offset += 2 * l + 1
    return np.array(source, dtype=np.int64), np.array(sign)


def hr_to_images(n: int, records, atom_shells, positions=None, cell=None,
                 spin_components: int = 1, energy_factor: float = EV_PER_RYDBERG):
    """Atom blocks of the records as images for bloch.ImageOperator.

    atom_shells: per atom, its shells' angular momenta (every atom must have
    the same orbital count: the device operators use one block size).
    positions (n_atoms x 3) and cell (3 x 3, rows the lattice vectors), both
    Cartesian, give the bond vectors R + r_j - r_i the velocities need.
    energy_factor: EV_PER_RYDBERG for H(R), 1 for S(R).  Returns
    (rows, cols, shifts[n, 3], blocks[n, b, b], bond_vectors or None,
    n_atoms, block_size)."""
    orders = [abacus_orbital_order(s, spin_components) for s in atom_shells]
    sizes = np.array([o[0].size for o in orders])
    if sizes.sum() != n:
        raise ValueError(f"the shells give {sizes.sum()} orbitals, the file {n}")
    if not np.all(sizes == sizes[0]):
        raise NotImplementedError("atoms with different orbital counts: the device operators "
                                  "take one block size")
    b = int(sizes[0])
    n_atoms = len(atom_shells)
    offs = np.concatenate([[0], np.cumsum(sizes)])
    rows, cols, shifts, blocks = [], [], [], []
    for rec in records:
        if rec.values.size == 0:
            continue
        dense_rows = np.repeat(np.arange(n), np.diff(rec.row_ptr))
        ai = dense_rows // b
        aj = rec.col_ind // b
        key = ai * n_atoms + aj
        for k in np.unique(key):
            i, j = divmod(int(k), n_atoms)
            sel = key == k
            blk = np.zeros((b, b), dtype=rec.values.dtype)
            blk[dense_rows[sel] - offs[i], rec.col_ind[sel] - offs[j]] = rec.values[sel]
            si, gi = orders[i]
            sj, gj = orders[j]
            rows.append(i)
            cols.append(j)
            shifts.append(rec.shift)
            blocks.append(energy_factor * gi[:, None] * gj[None, :] * blk[np.ix_(si, sj)])
    shifts = np.asarray(shifts, dtype=np.float64).reshape(-1, 3)
    vecs = None
    if positions is not None and cell is not None:
        pos = np.asarray(positions, dtype=np.float64)
        vecs = shifts @ np.asarray(cell, dtype=np.float64) + pos[cols] - pos[rows]
    return (np.asarray(rows, np.int64), np.asarray(cols, np.int64), shifts,
            np.asarray(blocks), vecs, n_atoms, b)
