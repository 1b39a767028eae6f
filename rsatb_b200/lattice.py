"""Seeded synthetic operators for the benchmark workloads.

The reference builds H and S from model files through vbcsr's AtomicData
(out of scope here); these generators produce the same kinds of operators
directly as uniform-block BSR arrays on the host, with atoms ordered as
generated (cell-major) and neighbour lists from explicit lattice
enumeration.  Every random draw comes from ``numpy.random.default_rng``
with an explicit seed, so the GPU path and the oracle see the same input.

A ``BsrArrays`` holds (row_ptr, col_ind, values[nnzb, b, b], b).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class BsrArrays:
    row_ptr: np.ndarray
    col_ind: np.ndarray
    values: np.ndarray
    block_size: int
    n_block_cols: int | None = None

    @property
    def n_block_rows(self) -> int:
        return self.row_ptr.size - 1

    @property
    def n_rows(self) -> int:
        return self.n_block_rows * self.block_size

    @property
    def nnz_blocks(self) -> int:
        return self.col_ind.size

    def to_dense(self) -> np.ndarray:
        b = self.block_size
        nbc = self.n_block_cols or self.n_block_rows
        A = np.zeros((self.n_block_rows * b, nbc * b), dtype=self.values.dtype)
        rows = np.repeat(np.arange(self.n_block_rows), np.diff(self.row_ptr))
        for k in range(self.nnz_blocks):
            i, j = rows[k], self.col_ind[k]
            A[i * b:(i + 1) * b, j * b:(j + 1) * b] += self.values[k]
        return A

    def with_values(self, values: np.ndarray) -> "BsrArrays":
        return BsrArrays(self.row_ptr, self.col_ind, values, self.block_size, self.n_block_cols)

    def block_index(self) -> dict:
        rows = np.repeat(np.arange(self.n_block_rows), np.diff(self.row_ptr))
        return {(int(i), int(j)): k for k, (i, j) in enumerate(zip(rows, self.col_ind))}


def csr_from_pairs(n: int, rows: np.ndarray, cols: np.ndarray):
    """Sorted, de-duplicated CSR pattern from (row, col) pairs; returns
    (row_ptr, col_ind, order) with order mapping pattern slots to pairs."""
    key = rows.astype(np.int64) * n + cols.astype(np.int64)
    order = np.argsort(key, kind="stable")
    key_sorted = key[order]
    if key_sorted.size and np.any(np.diff(key_sorted) == 0):
        raise ValueError("duplicate (row, col) pairs")
    r = rows[order]
    row_ptr = np.zeros(n + 1, dtype=np.int32)
    np.add.at(row_ptr, r + 1, 1)
    row_ptr = np.cumsum(row_ptr).astype(np.int32)
    return row_ptr, cols[order].astype(np.int32), order


# ------------------------------------------------------------------ graphene

def graphene(n1: int = 60, n2: int = 60, t: float = -2.7, a_cc: float = 1.42):
    """pz graphene n1 x n2 honeycomb supercell, periodic, nearest-neighbour t,
    onsite 0 (S = I).  Atom 2*(i + n1*j) + s, s = 0 (A) / 1 (B).
    Returns (H BsrArrays with b = 1, positions[n, 3], cell[3, 3])."""
    a = math.sqrt(3.0) * a_cc
    a1 = np.array([a, 0.0, 0.0])
    a2 = np.array([a / 2, a * math.sqrt(3.0) / 2, 0.0])
    delta = (a1 + a2) / 3.0
    n = 2 * n1 * n2
    i, j = np.meshgrid(np.arange(n1), np.arange(n2), indexing="ij")
    i = i.ravel(order="F")
    j = j.ravel(order="F")
    cell_id = i + n1 * j
    A = 2 * cell_id
    B = A + 1
    pos = np.zeros((n, 3))
    pos[A] = i[:, None] * a1 + j[:, None] * a2
    pos[B] = pos[A] + delta

    def bidx(ii, jj):
        return 2 * ((ii % n1) + n1 * (jj % n2)) + 1

    rows = np.concatenate([A, A, A])
    cols = np.concatenate([bidx(i, j), bidx(i - 1, j), bidx(i, j - 1)])
    rows, cols = np.concatenate([rows, cols]), np.concatenate([cols, rows])
    row_ptr, col_ind, _ = csr_from_pairs(n, rows, cols)
    vals = np.full((col_ind.size, 1, 1), t)
    cell = np.array([n1 * a1, n2 * a2, [0.0, 0.0, 20.0]])
    return BsrArrays(row_ptr, col_ind, vals, 1), pos, cell


def graphene_images(n1: int = 60, n2: int = 60, t: float = -2.7, a_cc: float = 1.42):
    """The bonds of graphene()'s n1 x n2 supercell as real-space images: for
    every A atom the three bonds to B at cells (i, j), (i - 1, j), (i, j - 1),
    and their reverses, each with its supercell image shift R (integer, in
    units of the supercell vectors) and bond vector r_j + R - r_i.  Any
    n1, n2 >= 1 (a 1 x 1 cell has three images of the one A-B pair).
    Returns (rows, cols, shifts[n, 3], blocks[n, 1, 1], bond_vectors[n, 3],
    n_atoms, cell[3, 3])."""
    a = math.sqrt(3.0) * a_cc
    a1 = np.array([a, 0.0, 0.0])
    a2 = np.array([a / 2, a * math.sqrt(3.0) / 2, 0.0])
    delta = (a1 + a2) / 3.0
    i, j = np.meshgrid(np.arange(n1), np.arange(n2), indexing="ij")
    i = i.ravel(order="F")
    j = j.ravel(order="F")
    A = 2 * (i + n1 * j)
    rows, cols, shifts, vecs = [], [], [], []
    for di, dj in ((0, 0), (-1, 0), (0, -1)):
        ii, jj = i + di, j + dj
        B = 2 * ((ii % n1) + n1 * (jj % n2)) + 1
        R = np.stack([np.floor_divide(ii, n1), np.floor_divide(jj, n2), np.zeros_like(ii)], 1)
        d = delta + di * a1 + dj * a2
        rows += [A, B]
        cols += [B, A]
        shifts += [R, -R]
        vecs += [np.tile(d, (A.size, 1)), np.tile(-d, (A.size, 1))]
    rows = np.concatenate(rows)
    cols = np.concatenate(cols)
    shifts = np.concatenate(shifts).astype(np.float64)
    vecs = np.concatenate(vecs)
    blocks = np.full((rows.size, 1, 1), float(t))
    cell = np.array([n1 * a1, n2 * a2, [0.0, 0.0, 20.0]])
    return rows, cols, shifts, blocks, vecs, 2 * n1 * n2, cell


# ------------------------------------------------------------------- diamond

_DIAMOND_BASIS4 = np.array([[0, 0, 0], [0, 2, 2], [2, 0, 2], [2, 2, 0],
                            [1, 1, 1], [1, 3, 3], [3, 1, 3], [3, 3, 1]])


def diamond_pattern(L: int, max_shell_sq: int = 11):
    """Neighbour pattern of an L^3 conventional-cell diamond supercell to the
    shell with |d|^2 <= max_shell_sq in units of (a/4)^2 (3: 1st, 8: 2nd,
    11: 3rd shell).  Atom 8*(cx + L*(cy + L*cz)) + basis.  Returns
    (row_ptr, col_ind, dist2 per pattern slot, int positions[n, 3])."""
    G = 4 * L
    grid = -np.ones((G, G, G), dtype=np.int64)
    cx, cy, cz = np.meshgrid(np.arange(L), np.arange(L), np.arange(L), indexing="ij")
    cells = np.stack([cx.ravel(order="F"), cy.ravel(order="F"), cz.ravel(order="F")], 1)
    n = 8 * L ** 3
    ipos = (4 * cells[:, None, :] + _DIAMOND_BASIS4[None, :, :]).reshape(n, 3)
    grid[ipos[:, 0], ipos[:, 1], ipos[:, 2]] = np.arange(n)
    r = int(math.isqrt(max_shell_sq))
    d = np.array([(x, y, z) for x in range(-r, r + 1) for y in range(-r, r + 1)
                  for z in range(-r, r + 1) if x * x + y * y + z * z <= max_shell_sq])
    rows, cols, dist2 = [], [], []
    for dv in d:
        q = (ipos + dv) % G
        nb = grid[q[:, 0], q[:, 1], q[:, 2]]
        ok = nb >= 0
        rows.append(np.nonzero(ok)[0])
        cols.append(nb[ok])
        dist2.append(np.full(ok.sum(), int(dv @ dv)))
    rows = np.concatenate(rows)
    cols = np.concatenate(cols)
    dist2 = np.concatenate(dist2)
    row_ptr, col_ind, order = csr_from_pairs(n, rows, cols)
    return row_ptr, col_ind, dist2[order], ipos


def _symmetric_blocks(row_ptr, col_ind, gen_block, b):
    """Values for a symmetric pattern with V[j,i] = V[i,j]^T: blocks are drawn
    for i < j (and i == j) in pattern order, then mirrored."""
    n = row_ptr.size - 1
    rows = np.repeat(np.arange(n), np.diff(row_ptr))
    nnz = col_ind.size
    key = rows.astype(np.int64) * n + col_ind
    tkey = col_ind.astype(np.int64) * n + rows
    mirror = np.searchsorted(key, tkey)
    upper = rows <= col_ind
    vals = np.zeros((nnz, b, b))
    idx_upper = np.nonzero(upper)[0]
    vals[idx_upper] = gen_block(idx_upper, rows[idx_upper], col_ind[idx_upper])
    lower = np.nonzero(~upper)[0]
    vals[lower] = np.transpose(vals[mirror[lower]], (0, 2, 1))
    diag = np.nonzero(rows == col_ind)[0]
    vals[diag] = 0.5 * (vals[diag] + np.transpose(vals[diag], (0, 2, 1)))
    return vals


def diamond_lcao(L: int = 16, seed: int = 7, a: float = 3.567, orbitals: int = 8,
                 s_amplitude: float = 0.15, s_scale: float = 1.0):
    """Non-orthogonal LCAO diamond: H blocks N(0,1)*exp(-r/1.5), S = I on the
    diagonal and U(0, s_amplitude)*s_scale*exp(-r/1.2) off it, both
    symmetric, 8x8 blocks to the 3rd shell (29 blocks per row).  Returns
    (H, S) BsrArrays."""
    row_ptr, col_ind, dist2, _ = diamond_pattern(L, 11)
    r = np.sqrt(dist2) * a / 4.0
    b = orbitals
    rng_h = np.random.default_rng(seed)
    rng_s = np.random.default_rng(seed + 1)

    def gen_h(idx, _r, _c):
        blk = rng_h.standard_normal((idx.size, b, b))
        return blk * np.exp(-r[idx] / 1.5)[:, None, None]

    def gen_s(idx, rr, cc):
        blk = rng_s.uniform(0.0, s_amplitude, (idx.size, b, b)) * s_scale
        blk *= np.exp(-r[idx] / 1.2)[:, None, None]
        blk[rr == cc] = np.eye(b)
        return blk

    H = BsrArrays(row_ptr, col_ind, _symmetric_blocks(row_ptr, col_ind, gen_h, b), b)
    S = BsrArrays(row_ptr, col_ind, _symmetric_blocks(row_ptr, col_ind, gen_s, b), b)
    return H, S


def subgraph_problems(P: BsrArrays):
    """The graph-local problems of graph_inverse_sqrt (isqrtm.hpp:149-232):
    for block row i the dense sub-matrix of P on {i} + neighbours(i).
    Returns (members[n, k] sorted atom lists, slot[n] position of i,
    gather[n, k, k] block index into P.values or -1).  Rows must have equal
    neighbour counts (uniform lattices)."""
    n = P.n_block_rows
    deg = np.diff(P.row_ptr)
    if not np.all(deg == deg[0]):
        raise ValueError("subgraph_problems needs a uniform neighbour count")
    k = int(deg[0])
    members = P.col_ind.reshape(n, k).astype(np.int64)
    slot = np.argmax(members == np.arange(n)[:, None], axis=1)
    rows = np.repeat(np.arange(n), k)
    key = rows.astype(np.int64) * n + P.col_ind
    q = members[:, :, None] * n + members[:, None, :]
    pos = np.searchsorted(key, q)
    pos = np.minimum(pos, key.size - 1)
    gather = np.where(key[pos] == q, pos, -1).astype(np.int64)
    return members, slot, gather


# ----------------------------------------------------- twisted bilayer graphene

def _rot(theta: float) -> np.ndarray:
    c, s = math.cos(theta), math.sin(theta)
    return np.array([[c, -s], [s, c]])


def _layer_atoms(t1: np.ndarray, t2: np.ndarray, b1: np.ndarray, b2: np.ndarray,
                 delta: np.ndarray, span: int) -> np.ndarray:
    """Honeycomb sites (lattice b1, b2, basis {0, delta}) inside the cell
    spanned by t1, t2, as 2-D positions wrapped into the cell."""
    Tinv = np.linalg.inv(np.stack([t1, t2], axis=1))
    n = np.arange(-span, span + 1)
    n1, n2 = np.meshgrid(n, n, indexing="ij")
    base = n1.reshape(-1, 1) * b1 + n2.reshape(-1, 1) * b2
    out = []
    for off in (np.zeros(2), delta):
        p = base + off
        f = p @ Tinv.T
        keep = np.all((f > -1e-9) & (f < 1.0 - 1e-9), axis=1)
        out.append(p[keep])
    return np.concatenate(out)


def twisted_bilayer_graphene(m: int = 31, tiles=(4, 4), t: float = -2.7, a_cc: float = 1.42,
                             d0: float = 3.35, v0: float = 0.48, decay: float = 0.45,
                             cutoff: float = 6.0):
    """Commensurate twisted bilayer graphene (pz), periodic in-plane.

    Moire cell of index m: cos(theta) = (3m^2 + 3m + 1/2) / (3m^2 + 3m + 1),
    4 (3m^2 + 3m + 1) atoms (m = 31: theta = 1.0501 deg, 11,908 atoms),
    tiled tiles[0] x tiles[1].  Intralayer nearest neighbours hop t;
    interlayer pairs within `cutoff` hop v0 exp(-(d - d0) / decay).  Atoms
    are ordered layer-major inside each moire cell, cells in tile order.
    Returns (H BsrArrays with b = 1, positions[n, 3], cell[3, 3],
    displacements[nnz, 3]): displacements are the minimum-image bond vectors
    r_j + R - r_i of the stored pattern, for commutator velocities."""
    from scipy.spatial import cKDTree

    a = math.sqrt(3.0) * a_cc
    a1 = np.array([a, 0.0])
    a2 = np.array([a / 2.0, a * math.sqrt(3.0) / 2.0])
    delta = (a1 + a2) / 3.0
    theta = math.acos((3 * m * m + 3 * m + 0.5) / (3 * m * m + 3 * m + 1.0))
    t1 = m * a1 + (m + 1) * a2
    t2 = -(m + 1) * a1 + (2 * m + 1) * a2
    per_layer = 2 * (3 * m * m + 3 * m + 1)
    span = 3 * m + 4
    L1 = _layer_atoms(t1, t2, a1, a2, delta, span)
    # Layer 2 is layer 1 rotated by theta; the moire vectors are lattice
    # vectors of both layers (checked), so its sites tile the same cell.
    Rm = _rot(theta)
    b1, b2 = Rm @ a1, Rm @ a2
    B = np.stack([b1, b2], axis=1)
    for tv in (t1, t2):
        c = np.linalg.solve(B, tv)
        if not np.allclose(c, np.round(c), atol=1e-6):
            raise AssertionError("moire vector is not a lattice vector of the rotated layer")
    L2 = _layer_atoms(t1, t2, b1, b2, Rm @ delta, 4 * span)
    if L1.shape[0] != per_layer or L2.shape[0] != per_layer:
        raise AssertionError(f"site count {L1.shape[0]}, {L2.shape[0]} != {per_layer}")
    cell_pos = np.concatenate([np.c_[L1, np.zeros(per_layer)], np.c_[L2, np.full(per_layer, d0)]])
    layer_cell = np.r_[np.zeros(per_layer, np.int8), np.ones(per_layer, np.int8)]
    T1 = np.r_[t1, 0.0]
    T2 = np.r_[t2, 0.0]
    n_cell = cell_pos.shape[0]
    pos = []
    for q in range(tiles[1]):
        for p in range(tiles[0]):
            pos.append(cell_pos + p * T1 + q * T2)
    pos = np.concatenate(pos)
    layer = np.tile(layer_cell, tiles[0] * tiles[1])
    n = pos.shape[0]
    S1, S2 = tiles[0] * T1, tiles[1] * T2
    # Periodic neighbour search over the 3 x 3 images of the supercell.
    shifts = [(u, v) for u in (-1, 0, 1) for v in (-1, 0, 1)]
    img = np.concatenate([pos + u * S1 + v * S2 for u, v in shifts])
    tree = cKDTree(img)
    pairs = tree.query_ball_point(pos, cutoff + 1e-9, return_sorted=True)
    rows = np.repeat(np.arange(n), [len(p) for p in pairs])
    cols_img = np.concatenate([np.asarray(p, dtype=np.int64) for p in pairs])
    cols = cols_img % n
    disp = img[cols_img] - pos[rows]
    dist = np.linalg.norm(disp, axis=1)
    same = layer[rows] == layer[cols]
    keep = (dist > 1e-6) & ((~same) | (dist < 0.5 * (a_cc + a)))
    rows, cols, disp, dist, same = rows[keep], cols[keep], disp[keep], dist[keep], same[keep]
    vals = np.where(same, t, v0 * np.exp(-(dist - d0) / decay))
    row_ptr, col_ind, order = csr_from_pairs(n, rows, cols)
    H = BsrArrays(row_ptr, col_ind, vals[order].reshape(-1, 1, 1), 1)
    cell = np.array([S1, S2, [0.0, 0.0, 20.0]])
    return H, pos, cell, disp[order]


def commutator_velocity(H: BsrArrays, displacements: np.ndarray):
    """Real parts W_a of the velocities V_a = i W_a at the Gamma point:
    W_a,ij = (r_j + R - r_i)_a H_ij, the bond moment of
    rsatb/operator/commutator_velocity.hpp:100-255 (BuildCommutatorVelocity,
    factor i, kDisplacement weights) for b = 1 and a single image per bond.
    Returns three BsrArrays sharing H's pattern, to be stored with the
    imaginary-unit flag."""
    if H.block_size != 1:
        raise ValueError("commutator_velocity: pz (b = 1) operators only")
    out = []
    for axis in range(3):
        w = H.values[:, 0, 0] * displacements[:, axis]
        out.append(BsrArrays(H.row_ptr, H.col_ind, w.reshape(-1, 1, 1), 1))
    return out


def graphene_displacements(H: BsrArrays, pos: np.ndarray, cell: np.ndarray) -> np.ndarray:
    """Minimum-image bond vectors r_j + R - r_i of graphene()'s pattern."""
    rows = np.repeat(np.arange(H.n_block_rows), np.diff(H.row_ptr))
    d = pos[H.col_ind] - pos[rows]
    C = cell[:2, :2]
    f = d[:, :2] @ np.linalg.inv(C)
    f -= np.round(f)
    d[:, :2] = f @ C
    return d


# ----------------------------------------------------------- silicon sp3s*

# Fixed SK-like mean blocks of an sp3s* basis (s, px, py, pz, s*), eV: the
# onsite energies and one nearest- and one second-neighbour block.  The
# means set the spectrum's shape; every element is then perturbed by
# N(0, sigma) per bond.
_SI_ONSITE = np.diag([-4.20, 1.715, 1.715, 1.715, 6.685])
_SI_NN = np.array([[-2.08, 1.43, 1.43, 1.43, 0.00],
                   [-1.43, 0.43, 1.13, 1.13, -1.36],
                   [-1.43, 1.13, 0.43, 1.13, -1.36],
                   [-1.43, 1.13, 1.13, 0.43, -1.36],
                   [0.00, 1.36, 1.36, 1.36, 0.00]])
_SI_NNN = 0.1 * _SI_NN


def silicon_sp3s(L: int = 8, seed: int = 11, sigma: float = 0.1):
    """Silicon L^3 conventional cells (8 L^3 atoms, a = 5.431 A), sp3s*
    (5 orbitals), 5x5 blocks to the 2nd neighbour shell (1 + 4 + 12 = 17 per
    row); blocks are the fixed means above plus N(0, sigma) eV, symmetric
    (H_ji = H_ij^T).  Returns H BsrArrays."""
    row_ptr, col_ind, dist2, _ = diamond_pattern(L, 8)
    rng = np.random.default_rng(seed)
    means = {0: _SI_ONSITE, 3: _SI_NN, 8: _SI_NNN}

    def gen(idx, _r, _c):
        base = np.stack([means[int(d)] for d in dist2[idx]])
        return base + sigma * rng.standard_normal((idx.size, 5, 5))

    return BsrArrays(row_ptr, col_ind, _symmetric_blocks(row_ptr, col_ind, gen, 5), 5)
