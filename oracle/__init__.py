"""TEST INFRASTRUCTURE: the CPU oracle for the rsatb_b200 hot path.

``kpm_oracle.c`` restates the reference algorithms in plain C (FP64,
OpenMP); this module builds it with gcc into ``oracle/_build`` and wraps it
with ctypes, and adds the numpy exact-diagonalisation references.  Only the
tests, ``__graft_entry__.smoke()`` and the CPU baseline legs of ``bench.py``
use it, as the checker; the product (``rsatb_b200``) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build"
LIB = BUILD / "libkpm_oracle.so"
SRC = HERE / "kpm_oracle.c"

_lib = None


def build(force: bool = False) -> Path:
    """Compiles kpm_oracle.c (gcc -O2 -fopenmp, no FP contraction)."""
    BUILD.mkdir(exist_ok=True)
    if force or not LIB.exists() or LIB.stat().st_mtime < SRC.stat().st_mtime:
        cmd = ["gcc", "-O2", "-march=x86-64-v2", "-fopenmp", "-ffp-contract=off", "-fPIC",
               "-shared", "-o", str(LIB), str(SRC), "-lm"]
        subprocess.run(cmd, check=True)
    return LIB


class OrcBsr(C.Structure):
    _fields_ = [("n_block_rows", C.c_int), ("n_block_cols", C.c_int), ("b", C.c_int),
                ("row_ptr", C.c_void_p), ("col_ind", C.c_void_p), ("vals", C.c_void_p),
                ("cplx", C.c_int), ("imag", C.c_int)]


class OrcOp(C.Structure):
    _fields_ = [("sandwich", C.c_int), ("H", C.POINTER(OrcBsr)), ("Z", C.POINTER(OrcBsr)),
                ("ZH", C.POINTER(OrcBsr)), ("center", C.c_double), ("half_width", C.c_double)]


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        vp, i, d, u64, i64 = C.c_void_p, C.c_int, C.c_double, C.c_uint64, C.c_int64
        L.orc_set_random.argtypes = [u64, i, i, vp, i, i, i64, i, i64, i, vp]
        L.orc_spmm.argtypes = [C.POINTER(OrcBsr), vp, vp, i, i, d]
        L.orc_spmm.restype = None
        L.orc_apply_op.argtypes = [C.POINTER(OrcOp), vp, vp, i, i, vp]
        L.orc_apply_op.restype = None
        L.orc_kpm_moments.argtypes = [C.POINTER(OrcOp), vp, i, i, i, i, vp, vp]
        L.orc_kernel_weights.argtypes = [i, i, vp]
        L.orc_kernel_weights.restype = None
        L.orc_density.argtypes = [vp, i, vp, i, d, i, vp]
        L.orc_density.restype = None
        L.orc_dct3_direct.argtypes = [vp, i, i, vp]
        L.orc_dct3_direct.restype = None
        L.orc_dct3_fftroute.argtypes = [vp, i, i, vp]
        L.orc_dct3_fftroute.restype = None
        L.orc_fftcheb.argtypes = [C.POINTER(OrcOp), C.POINTER(OrcBsr), C.POINTER(OrcBsr),
                                  C.POINTER(OrcBsr), vp, i, i, i, d, i, i, vp, vp]
        L.orc_philox4x32_10.argtypes = [vp, vp, vp]
        L.orc_philox4x32_10.restype = None
        L.orc_num_threads.restype = i
        L.orc_set_threads.argtypes = [i]
        L.orc_set_threads.restype = None
        _lib = L
    return _lib


def num_threads() -> int:
    return lib().orc_num_threads()


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class Bsr:
    """Host BSR in the library's layout (row-major blocks, complex interleaved)."""

    def __init__(self, n_block_rows, n_block_cols, b, row_ptr, col_ind, values, imag=False):
        self.row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
        self.col_ind = np.ascontiguousarray(col_ind, dtype=np.int32)
        vals = np.asarray(values)
        self.cplx = np.iscomplexobj(vals)
        self.vals = np.ascontiguousarray(vals, dtype=np.complex128 if self.cplx else np.float64)
        self.n_block_rows, self.n_block_cols, self.b = int(n_block_rows), int(n_block_cols), int(b)
        self.imag = bool(imag)
        self.c = OrcBsr(self.n_block_rows, self.n_block_cols, self.b, _ptr(self.row_ptr),
                        _ptr(self.col_ind), _ptr(self.vals), int(self.cplx), int(self.imag))

    @classmethod
    def from_dense(cls, A: np.ndarray, b: int = 1, imag: bool = False, tol: float = 0.0):
        n = A.shape[0] // b
        m = A.shape[1] // b
        ptr, ind, vals = [0], [], []
        for i in range(n):
            for j in range(m):
                blk = A[i * b:(i + 1) * b, j * b:(j + 1) * b]
                if np.abs(blk).max() > tol:
                    ind.append(j)
                    vals.append(blk)
            ptr.append(len(ind))
        vals = np.array(vals).reshape(len(ind), b, b) if ind else np.zeros((0, b, b), A.dtype)
        return cls(n, m, b, ptr, ind, vals, imag=imag)

    def to_dense(self) -> np.ndarray:
        b = self.b
        dt = np.complex128 if (self.cplx or self.imag) else np.float64
        A = np.zeros((self.n_block_rows * b, self.n_block_cols * b), dtype=dt)
        v = self.vals.reshape(-1, b, b)
        for i in range(self.n_block_rows):
            for k in range(self.row_ptr[i], self.row_ptr[i + 1]):
                j = self.col_ind[k]
                A[i * b:(i + 1) * b, j * b:(j + 1) * b] = v[k] * (1j if self.imag else 1.0)
        return A


def bsr_adjoint(A: Bsr) -> Bsr:
    """A^H in the same layout (host counting sort by column)."""
    n = A.n_block_rows
    rows = np.repeat(np.arange(n), np.diff(A.row_ptr))
    order = np.lexsort((rows, A.col_ind))
    t_rows = A.col_ind[order]
    ptr = np.zeros(A.n_block_cols + 1, dtype=np.int64)
    np.add.at(ptr, t_rows + 1, 1)
    vals = np.conj(np.transpose(A.vals.reshape(-1, A.b, A.b)[order], (0, 2, 1)))
    if A.imag:
        vals = -vals
    return Bsr(A.n_block_cols, n, A.b, np.cumsum(ptr), rows[order], np.ascontiguousarray(vals),
               imag=A.imag)


def _as_panel(X: np.ndarray):
    """(N, R) real or complex -> contiguous float64 view and (W, cv)."""
    if np.iscomplexobj(X):
        Xc = np.ascontiguousarray(X, dtype=np.complex128)
        return Xc, 2 * X.shape[1], 1
    Xr = np.ascontiguousarray(X, dtype=np.float64)
    return Xr, X.shape[1], 0


def spmm(A: Bsr, X: np.ndarray, alpha: float = 1.0) -> np.ndarray:
    Xc, W, cv = _as_panel(X)
    cplx_out = cv or A.cplx or A.imag
    if cplx_out and not cv:
        Xc, W, cv = _as_panel(X.astype(np.complex128))
    Y = np.zeros_like(Xc)
    lib().orc_spmm(C.byref(A.c), _ptr(Xc), _ptr(Y), W, cv, float(alpha))
    return Y


def make_op(H: Bsr, center: float, half_width: float, Z: Bsr | None = None,
            ZH: Bsr | None = None) -> OrcOp:
    op = OrcOp(1 if Z is not None else 0, C.pointer(H.c),
               C.pointer(Z.c) if Z is not None else None,
               C.pointer(ZH.c) if ZH is not None else None, float(center), float(half_width))
    op._keep = (H, Z, ZH)
    return op


def apply_op(op: OrcOp, X: np.ndarray) -> np.ndarray:
    Xc, W, cv = _as_panel(X)
    Y = np.zeros_like(Xc)
    T = np.zeros_like(Xc)
    lib().orc_apply_op(C.byref(op), _ptr(Xc), _ptr(Y), W, cv, _ptr(T))
    return Y


def kpm_moments(op: OrcOp, psi: np.ndarray, n_moments: int, doubled: bool = True,
                per_column: bool = False):
    """dos.hpp:125 kpm_dos_moments; returns complex moments (and per-column)."""
    Xc, W, cv = _as_panel(psi)
    R = psi.shape[1]
    mu = np.zeros(2 * n_moments)
    col = np.zeros(2 * n_moments * R) if per_column else None
    st = lib().orc_kpm_moments(C.byref(op), _ptr(Xc), R, cv, int(n_moments), int(doubled),
                               _ptr(mu), _ptr(col) if per_column else None)
    if st != 0:
        raise RuntimeError(f"orc_kpm_moments failed ({st})")
    m = mu.view(np.complex128)
    if per_column:
        return m, col.view(np.complex128).reshape(n_moments, R)
    return m


def set_random(seed: int, kind: int, normalize: bool, atom_index: np.ndarray, orbitals: int,
               n_rows_global: int, n_vectors: int, complex_out: bool,
               first_column: int = 0) -> np.ndarray:
    ids = np.ascontiguousarray(atom_index, dtype=np.int64)
    n_rows = ids.size * orbitals
    out = np.zeros((n_rows, n_vectors), dtype=np.complex128 if complex_out else np.float64)
    st = lib().orc_set_random(C.c_uint64(seed), kind, int(normalize), _ptr(ids), ids.size,
                              orbitals, n_rows_global, n_vectors, int(first_column),
                              int(complex_out), _ptr(out))
    if st != 0:
        raise ValueError("orc_set_random: invalid arguments")
    return out


def philox4x32_10(ctr, key) -> np.ndarray:
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    lib().orc_philox4x32_10(_ptr(c), _ptr(k), _ptr(out))
    return out


def kernel_weights(kernel: int, n: int) -> np.ndarray:
    g = np.zeros(n)
    lib().orc_kernel_weights(kernel, n, _ptr(g))
    return g


def density(mu: np.ndarray, x: np.ndarray, edge_inset: float, kernel: int = 1) -> np.ndarray:
    m = np.ascontiguousarray(mu, dtype=np.complex128)
    xx = np.ascontiguousarray(x, dtype=np.float64)
    rho = np.zeros_like(xx)
    lib().orc_density(_ptr(m), m.size, _ptr(xx), xx.size, float(edge_inset), kernel, _ptr(rho))
    return rho


def dct3(x: np.ndarray, route: str = "direct") -> np.ndarray:
    """Batched DCT-III along the last axis of a complex (batch, n) array."""
    xx = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.zeros_like(xx)
    f = lib().orc_dct3_direct if route == "direct" else lib().orc_dct3_fftroute
    f(_ptr(xx), xx.shape[-1], int(np.prod(xx.shape[:-1])), _ptr(out))
    return out


def fftcheb(op: OrcOp, V, psi: np.ndarray, n_moments: int, formulation: int = 0,
            prefactor: float = 1.0, sections: int = 1, kernel: int = 1):
    """dc_spectrum_fftcheb; returns (sigma[n_moments, 6], energy[n_moments])."""
    p = np.ascontiguousarray(psi, dtype=np.complex128)
    sigma = np.zeros(n_moments * 6)
    energy = np.zeros(n_moments)
    st = lib().orc_fftcheb(C.byref(op), C.byref(V[0].c), C.byref(V[1].c), C.byref(V[2].c),
                           _ptr(p), p.shape[1], int(n_moments), int(formulation),
                           float(prefactor), int(sections), int(kernel), _ptr(sigma),
                           _ptr(energy))
    if st != 0:
        raise RuntimeError(f"orc_fftcheb failed ({st})")
    return sigma.reshape(n_moments, 6), energy


# ------------------------------------------------------------ Bloch sums

def bloch_dense(rows, cols, shifts, blocks, n_block_rows: int, k, weights=None,
                imag_unit: bool = False, n_block_cols: int | None = None) -> np.ndarray:
    """Dense H(k) = sum_e w_e (i) exp(-2 pi i k . R_e) H_e at blocks
    (rows[e], cols[e]) (BlochPhase and AddLocalBlock,
    rsatb/operator/block_assembly.hpp:31-100)."""
    blocks = np.asarray(blocks)
    b = blocks.shape[1]
    nbc = n_block_cols or n_block_rows
    out = np.zeros((n_block_rows * b, nbc * b), dtype=np.complex128)
    ph = np.exp(-2j * np.pi * (np.asarray(shifts, dtype=np.float64) @ np.asarray(k, dtype=np.float64)))
    if weights is not None:
        ph = ph * np.asarray(weights)
    if imag_unit:
        ph = 1j * ph
    for e in range(len(rows)):
        i, j = int(rows[e]), int(cols[e])
        out[i * b:(i + 1) * b, j * b:(j + 1) * b] += ph[e] * blocks[e]
    return out


# ------------------------------------------------- finite-temperature sigma

def qe_dense(H: np.ndarray, V, psi: np.ndarray, center: float, half_width: float,
             n_moments: int, nodes_ascending=None, kernel: int = 1, prefactor: float = 1.0):
    """dc_spectrum_qe / accumulate_qe_block (rsatb/calc/fftcheb_transport.hpp:
    662-884) restated densely for an orthogonal operator (TEST
    INFRASTRUCTURE): the right chains R_m = T_m(A) J_b psi summed into the
    node vectors q_j with w_m(j) = (2 - [m = 0]) g_m / pi T_m(e_j), then the
    left chain's J_a^H T_m(A) psi contracted against them with the same
    weights over 1 - e_j^2 (at least 1e-14), the sample average, and sigma =
    prefactor Re(kernel) at the window's nodes (zero elsewhere).
    H, V[a]: dense (complex); psi: N x R.  Returns (sigma[M, 6], energy)."""
    M = n_moments
    N = H.shape[0]
    R = psi.shape[1]
    nodes = np.arange(M) if nodes_ascending is None else np.unique(np.asarray(nodes_ascending))
    src = M - 1 - nodes
    A = (np.asarray(H) - center * np.eye(N)) / half_width
    g = kernel_weights(kernel, M)
    th = np.pi * (src + 0.5) / M
    eps = np.cos(th)
    denom = np.maximum(1e-14, 1.0 - eps * eps)
    vs = 1.0 / (2.0 * half_width)
    J = [-vs * (np.asarray(V[a]) @ psi) for a in range(3)]
    w = np.array([[(1.0 if m == 0 else 2.0) * g[m] / np.pi * np.cos(m * t) for t in th]
                  for m in range(M)])                                   # (M, NE)
    q = np.zeros((3, nodes.size, N, R), dtype=np.complex128)
    r_prev = [x.copy() for x in J]
    r_curr = None
    for m in range(M):
        if m == 1:
            r_curr = [A @ x for x in r_prev]
        elif m >= 2:
            r_next = [2.0 * A @ r_curr[a] - r_prev[a] for a in range(3)]
            r_prev, r_curr = r_curr, r_next
        rm = r_prev if m == 0 else r_curr
        for a in range(3):
            q[a] += w[m][:, None, None] * rm[a][None]
    K = np.zeros((M, 6), dtype=np.complex128)
    l_prev, l_curr = psi.astype(np.complex128), None
    for m in range(M):
        if m == 1:
            l_curr = A.conj().T @ l_prev
        elif m >= 2:
            l_next = 2.0 * A.conj().T @ l_curr - l_prev
            l_prev, l_curr = l_curr, l_next
        lm = l_prev if m == 0 else l_curr
        for a in range(3):
            la = -vs * (np.asarray(V[a]).conj().T @ lm)
            comp = (0, 3, 5)[a]
            part = np.einsum("nr,jnr->j", la.conj(), q[a])
            K[src, comp] += w[m] * part / denom
    K /= R
    energy = center + half_width * np.cos(np.pi * (M - 1 - np.arange(M) + 0.5) / M)
    sigma = np.zeros((M, 6))
    sigma[nodes] = prefactor * K[src].real
    return sigma, energy


def integrate_dc_spectrum(sigma: np.ndarray, energy: np.ndarray, mu: float,
                          temp: float) -> np.ndarray:
    """rsatb/calc/fftcheb_transport.hpp:950-1040 (with fermi_dirac_energy
    :67-82): interpolation at T <= 0, the exact integral of the
    piecewise-linear spectrum against -df/dE at T > 0."""
    import math
    s = np.asarray(sigma, dtype=np.float64).reshape(-1, 6)
    e = np.asarray(energy, dtype=np.float64)
    out = np.zeros(6)
    if e.size == 0:
        return out
    if temp <= 0.0:
        for c in range(6):
            out[c] = np.interp(mu, e, s[:, c])
        return out
    kb = 8.617333262e-5
    kt = kb * temp

    def f(x):
        beta = 1.0 / kt
        if x >= mu:
            t = math.exp(beta * (mu - x))
            return t / (1.0 + t)
        t = math.exp(beta * (x - mu))
        return 1.0 / (1.0 + t)

    def F(x):
        y = (x - mu) / kt
        return x - kt * (max(y, 0.0) + math.log1p(math.exp(-abs(y))))

    for i in range(1, e.size):
        e0, e1 = e[i - 1], e[i]
        de = e1 - e0
        w = f(e0) - f(e1)
        m = F(e1) - F(e0) - f(e1) * de
        out += s[i - 1] * w + (s[i] - s[i - 1]) / de * m
    return out


# ------------------------------------------------------ correlation-series DOS

def timeprop_coeff(time_step: float, precision: float = 1e-14, forward: bool = True) -> np.ndarray:
    """rsatb/calc/cheby.hpp:85-106 with build_bessel_vector
    (rsatb/calc/bessel.hpp:9-52): J_n(t) for ascending n from scipy's Bessel
    function (the reference uses the bessel-library's cyl_j), kept while
    |J_n| > eps or |J_{n+1}| > eps; c_n = (2 - delta_n0) (-+i)^n J_n."""
    from scipy.special import jv
    n_max = 65536
    chunk = int(time_step + 64 * max(1.0, time_step) ** (1.0 / 3.0) + 64)
    vals = jv(np.arange(min(chunk + 1, n_max + 1)), time_step)
    n_terms = None
    for n in range(vals.size - 1):
        if abs(vals[n]) <= precision and abs(vals[n + 1]) <= precision:
            n_terms = n
            break
    if n_terms is None:
        raise RuntimeError("bessel: series not converged")
    J = vals[:n_terms]
    phase = (-1j if forward else 1j) ** np.arange(n_terms)
    c = 2.0 * phase * J
    c[0] *= 0.5
    return c


def corr_from_moments(mu: np.ndarray, nt: int, precision: float = 1e-14) -> np.ndarray:
    """rsatb/calc/dos.hpp:30-46: C(j pi) = sum_n c_n(j pi) mu_n, C(0) = mu_0."""
    mu = np.asarray(mu, dtype=np.complex128)
    out = np.zeros(nt + 1, dtype=np.complex128)
    out[0] = mu[0]
    for j in range(1, nt + 1):
        c = timeprop_coeff(j * np.pi, precision, True)
        m = min(c.size, mu.size)
        out[j] = np.sum(c[:m] * mu[:m])
    return out


def corr_dos(mu: np.ndarray, nt: int, precision: float = 1e-14) -> np.ndarray:
    """ComputeDos "corr" (rsatb/calc/observables.hpp:393-428): Hann window,
    mirrored series, unnormalised inverse FFT of 2 nt points, reordered."""
    cd = corr_from_moments(mu, nt, precision)
    full = np.zeros(2 * nt + 1, dtype=np.complex128)
    full[0] = cd[0]
    for i in range(1, nt + 1):
        f = 0.5 * (1 + np.cos(np.pi * (i - 1) / nt))
        full[i] = cd[i] * f
        full[2 * nt - i] = np.conj(cd[i]) * f
    F = np.fft.ifft(full[:2 * nt]) * (2 * nt)   # FFTW_BACKWARD is unnormalised
    return np.concatenate([F[nt:].real, F[:nt].real]), cd


# ----------------------------------------------------- dense inverse square root

EIGEN_CLAMP = 1.0e-12


def isqrt_columns_eigen(A: np.ndarray, col_start: int = 0, k: int | None = None,
                        clamp: float = EIGEN_CLAMP) -> np.ndarray:
    """Columns [col_start, col_start + k) of the clamped A^{-1/2}: the eigen
    route of isqrt::eigen_action (rsatb/calc/isqrt_action.hpp:766-795),
    X = V f(w) V^T E with f(x) = x^-1/2 for x > clamp else 0, FP64 LAPACK
    (numpy eigh) on the upper triangle."""
    n = A.shape[0]
    k = n if k is None or k <= 0 else k
    w, V = np.linalg.eigh(A, UPLO="U")
    f = np.where(w > clamp, 1.0 / np.sqrt(np.maximum(w, clamp)), 0.0)
    return (V * f) @ V[col_start:col_start + k].T


def _graph_isqrt_chunk(args):
    """Worker of graph_inverse_sqrt_eigen: Z blocks of one chunk of block
    rows (one batched LAPACK eigh per chunk).  `values` is the block array or
    the path of a .npy file holding it (read memory-mapped)."""
    values, members_rows, slot_rows, gather_rows, b = args
    if isinstance(values, str):
        values = np.load(values, mmap_mode="r")
    n, k = members_rows.shape
    padded = np.concatenate([np.asarray(values), np.zeros((1, b, b))])
    g = np.where(gather_rows >= 0, gather_rows, values.shape[0])
    M = padded[g]                                   # (n, k, k, b, b)
    M = M.transpose(0, 1, 3, 2, 4).reshape(n, k * b, k * b)
    w, V = np.linalg.eigh(M, UPLO="U")
    f = np.where(w > EIGEN_CLAMP, 1.0 / np.sqrt(np.maximum(w, EIGEN_CLAMP)), 0.0)
    idx = slot_rows[:, None] * b + np.arange(b)[None, :]
    Vs = np.take_along_axis(V, idx[:, :, None], axis=1)       # (n, b, kb)
    X = np.einsum("nij,nj,nlj->nil", Vs, f, V)                 # rows of M^-1/2
    return X.reshape(n, b, k, b).transpose(0, 2, 1, 3).reshape(n * k, b, b)


def graph_inverse_sqrt_eigen(row_ptr: np.ndarray, col_ind: np.ndarray, values: np.ndarray,
                             block_size: int, workers: int | None = None,
                             chunk: int = 256) -> np.ndarray:
    """The graph-local S^-1/2 factor on the host, FP64: for block row i the
    dense sub-matrix of S on {i} + its neighbours (rsatb/calc/isqrtm.hpp:
    149-232, graph_inverse_sqrt) and the block row of its clamped inverse
    square root at i's position, by the eigen route of
    isqrt::inverse_sqrt_columns_inplace for n <= 256 (rsatb/calc/
    isqrt_action.hpp:766-795).  Needs a uniform neighbour count and sorted
    column indices per row; returns the factor's block values on S's pattern
    (nnz_blocks, b, b).  The rows are split in chunks over `workers` spawned
    processes (all host cores by default)."""
    from concurrent.futures import ProcessPoolExecutor
    import multiprocessing as mp
    import tempfile
    row_ptr = np.asarray(row_ptr, dtype=np.int64)
    col_ind = np.asarray(col_ind, dtype=np.int64)
    n = row_ptr.size - 1
    deg = np.diff(row_ptr)
    if not np.all(deg == deg[0]):
        raise ValueError("graph_inverse_sqrt_eigen needs a uniform neighbour count")
    k = int(deg[0])
    members = col_ind.reshape(n, k)
    slot = np.argmax(members == np.arange(n)[:, None], axis=1)
    key = np.repeat(np.arange(n), k) * n + col_ind
    b = int(block_size)
    vals = np.ascontiguousarray(values, dtype=np.float64).reshape(-1, b, b)
    workers = workers or os.cpu_count() or 1
    n_chunks = (n + chunk - 1) // chunk
    parallel = workers > 1 and n_chunks > 1

    def jobs(src):
        for r0 in range(0, n, chunk):
            r1 = min(n, r0 + chunk)
            q = members[r0:r1, :, None] * n + members[r0:r1, None, :]
            pos = np.minimum(np.searchsorted(key, q), key.size - 1)
            gather = np.where(key[pos] == q, pos, -1)
            yield (src, members[r0:r1], slot[r0:r1], gather, b)

    if not parallel:
        return np.concatenate([_graph_isqrt_chunk(j) for j in jobs(vals)])
    # Workers read the block values from one memory-mapped file and run
    # single-threaded LAPACK, one chunk each at a time.
    saved = {v: os.environ.get(v) for v in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS",
                                             "MKL_NUM_THREADS")}
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "values.npy")
        np.save(path, vals)
        try:
            for v in saved:
                os.environ[v] = "1"
            with ProcessPoolExecutor(max_workers=min(workers, n_chunks),
                                     mp_context=mp.get_context("spawn")) as pool:
                parts = list(pool.map(_graph_isqrt_chunk, jobs(path)))
        finally:
            for v, old in saved.items():
                if old is None:
                    os.environ.pop(v, None)
                else:
                    os.environ[v] = old
    return np.concatenate(parts)


def lanczos_bounds(op_apply, n: int, steps: int = 20, seed: int = 2, padding: float = 0.5,
                   complex_values: bool = False):
    """Host restatement of the library's spectral-window estimate (a fixed
    number of Lanczos steps with full reorthogonalisation in FP64, the
    extreme Ritz values widened by their residual norms and by the
    reference's 0.5 eV padding, rsatb/setup/spectral_bounds.hpp:67-76,
    445-490), on the unscaled operator x -> op_apply(x) (N x 1 panels), from
    the same seeded start vector: Rademacher (complex random phase for a
    complex operator) of set_random(seed), normalised."""
    v = set_random(seed, 0 if complex_values else 1, True, np.arange(n), 1, n, 1,
                   complex_values)[:, 0]
    dt = np.complex128 if complex_values else np.float64
    v = (v / np.sqrt(np.vdot(v, v).real)).astype(dt)
    m = min(steps, n)
    Q = np.zeros((n, m), dtype=dt)
    alpha = np.zeros(m)
    beta = np.zeros(m)
    q = v
    for j in range(m):
        Q[:, j] = q
        w = op_apply(q[:, None])[:, 0].astype(dt)
        a = np.vdot(Q[:, j], w).real
        alpha[j] = a
        for _ in range(2):
            w = w - Q[:, :j + 1] @ (Q[:, :j + 1].conj().T @ w)
        bb = float(np.sqrt(max(np.vdot(w, w).real, 0.0)))
        beta[j] = bb
        if bb < 1e-12 * max(1.0, abs(a)):
            m = j + 1
            break
        q = w / bb
    T = np.diag(alpha[:m]) + np.diag(beta[:m - 1], 1) + np.diag(beta[:m - 1], -1)
    theta, Y = np.linalg.eigh(T)
    res = np.abs(beta[m - 1] * Y[-1, :])
    return float(theta[0] - padding - res[0]), float(theta[-1] + padding + res[-1])


# ------------------------------------------------- exact diagonalisation (ED)

def kpm_moments_ed(H: np.ndarray, psi: np.ndarray, center: float, half_width: float,
                   n_moments: int, per_column: bool = False):
    """KPM moments of the dense Hermitian operator H on the sample columns of
    psi by exact diagonalisation (FP64 LAPACK): with H~ = (H - center) /
    half_width = U diag(x) U^H, mu_n = (1/R) sum_q sum_k |(U^H psi_q)_k|^2
    T_n(x_k), the limit the Chebyshev recurrence of kpm_dos_moments
    (rsatb/calc/dos.hpp:125-190) reaches without rounding.  Real moments
    (complex dtype, zero imaginary part, like kpm_moments' output)."""
    x, U = np.linalg.eigh((np.asarray(H) - center * np.eye(H.shape[0])) / half_width)
    w = np.abs(U.conj().T @ np.asarray(psi)) ** 2            # (n_states, R)
    th = np.arccos(np.clip(x, -1.0, 1.0))
    T = np.cos(np.arange(n_moments)[:, None] * th[None, :])  # (n_moments, n_states)
    col = T @ w                                              # (n_moments, R)
    mu = col.mean(axis=1).astype(np.complex128)
    if per_column:
        return mu, col.astype(np.complex128)
    return mu


def jackson_delta_matrix(E: np.ndarray, levels: np.ndarray, center: float, half_width: float,
                         n_moments: int, kernel: int = 1) -> np.ndarray:
    """d[k, n]: the kernel-damped Chebyshev series of delta(E_k - levels_n)
    in 1/eV, as evaluate_kpm_density builds a density (rsatb/calc/kpm.hpp:
    206-241: g_0 + 2 sum_m g_m T_m(x) T_m(x_n), over pi sqrt(1 - x^2)), the
    energy argument x = (E - center) / half_width (the levels' clipped to
    [-1, 1]) and one more 1/half_width for energy units."""
    g = kernel_weights(kernel, n_moments)
    x = (np.asarray(E) - center) / half_width
    y = np.clip((np.asarray(levels) - center) / half_width, -1.0, 1.0)
    tx = np.arccos(np.clip(x, -1.0, 1.0))
    ty = np.arccos(y)
    out = np.full((x.size, y.size), g[0])
    for m0 in range(1, n_moments, 256):
        m = np.arange(m0, min(n_moments, m0 + 256))
        out += 2.0 * (np.cos(np.outer(tx, m)) * g[m]) @ np.cos(np.outer(m, ty))
    return out / (np.pi * np.sqrt(np.maximum(1e-14, 1.0 - x ** 2)))[:, None] / half_width


def kubo_greenwood_ed(H: np.ndarray, V: np.ndarray, center: float, half_width: float,
                      n_moments: int, kernel: int = 1):
    """The exact-trace limit of the FFT-Chebyshev Greenwood accumulation
    (rsatb/calc/fftcheb_transport.hpp:270-525, 543-660) on the dense
    Hermitian H and velocity V, by exact diagonalisation: on the ascending
    Chebyshev-node grid E_k of n_moments points,
        K(E_k) = (1/4N) sum_nm |V_nm|^2 d(E_k - e_n) d(E_k - e_m)
    with d the damped delta of jackson_delta_matrix and V_nm in H's
    eigenbasis.  It is what dc_spectrum_fftcheb returns at prefactor 1 when
    its samples are the N unit vectors (J = -V / (2 half_width), the delta
    series' rescaled-to-energy factors, and the 1/R sample average give the
    1/4N).  Returns (energy, K)."""
    N = H.shape[0]
    e, U = np.linalg.eigh(np.asarray(H))
    Wnm = np.abs(U.conj().T @ np.asarray(V) @ U) ** 2
    k = np.arange(n_moments)
    E = center + half_width * np.cos(np.pi * (n_moments - 1 - k + 0.5) / n_moments)
    d = jackson_delta_matrix(E, e, center, half_width, n_moments, kernel)
    K = np.einsum("kn,nm,km->k", d, Wnm, d) / (4.0 * N)
    return E, K


def graph_seed_dense(S: np.ndarray, row_ptr: np.ndarray, col_ind: np.ndarray, b: int):
    """The graph-local seed of inverse_sqrt on the host, for any pattern
    (rsatb/calc/isqrtm.hpp:149-232 with the eigen route of
    isqrt_action.hpp:766-795): block row i of Z is block row i of the clamped
    inverse square root of S restricted to {i} + neighbours(i) (the columns
    of S's row i).  S dense (N x N); returns Z dense with S's block pattern."""
    n = row_ptr.size - 1
    Z = np.zeros_like(S)
    for i in range(n):
        members = np.asarray(col_ind[row_ptr[i]:row_ptr[i + 1]])
        idx = (members[:, None] * b + np.arange(b)[None, :]).reshape(-1)
        slot = int(np.flatnonzero(members == i)[0])
        X = isqrt_columns_eigen(S[np.ix_(idx, idx)], slot * b, b).T  # rows at i
        Z[i * b:(i + 1) * b, idx] = X
    return Z


def max_block_residual(X: np.ndarray, b: int) -> float:
    """max over b x b blocks of ||(X - I)[i, j]||_F (rsatb/calc/isqrtm.hpp:
    360-405; a dense X stores every block)."""
    n = X.shape[0] // b
    D = (X - np.eye(X.shape[0])).reshape(n, b, n, b)
    return float(np.sqrt((D ** 2).sum(axis=(1, 3))).max())


def ns_refine_dense(S: np.ndarray, Z0: np.ndarray, b: int, tol: float = 1e-7,
                    maxit: int = 20) -> tuple[np.ndarray, dict]:
    """Dense FP64 restatement of inverse_sqrt's refinement loop
    (rsatb/calc/isqrtm.hpp:620-800) from the seed Z0 with no drop threshold
    and X reformed every step: X = Z^T S Z (symmetrised), stop when the max
    block residual is <= tol, after maxit steps, on a plateau
    (|norm_prev - norm| <= 0.005 norm) or, above 100, as diverged;
    P = 1.875 I - 1.25 X + 0.375 X^2, Z <- Z P.  Returns (Z, report dict)."""
    Z = Z0.copy()
    I = np.eye(S.shape[0])

    def reform(Zc):
        X = Zc.T @ S @ Zc
        return 0.5 * (X + X.T)

    X = reform(Z)
    norm = max_block_residual(X, b)
    norm_pre, count, diverged = 0.0, 0, False
    while norm > tol and count < maxit and abs(norm_pre - norm) > 0.005 * norm:
        if norm > 100.0:
            diverged = True
            break
        norm_pre = norm
        P = 1.875 * I - 1.25 * X + 0.375 * (X @ X)
        P = 0.5 * (P + P.T)
        Z = Z @ P
        X = reform(Z)
        norm = max_block_residual(X, b)
        count += 1
    return Z, {"steps": count, "converged": norm <= tol, "hit_maxiter": count >= maxit,
               "diverged": diverged, "residual": norm}


def chain_overlap(n: int, diag: float, off: float):
    """The 1-D chain overlaps of rsatb/calc/test/test_isqrtm.cpp (:21-39,
    :132-151): diag on the diagonal, off on both neighbours, no periodic
    wrap; returns (dense S, row_ptr, col_ind) with 1 x 1 blocks."""
    S = np.diag(np.full(n, float(diag)))
    i = np.arange(n - 1)
    S[i, i + 1] = S[i + 1, i] = off
    rows, cols = np.nonzero(S)
    row_ptr = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=n))]).astype(np.int32)
    return S, row_ptr, cols.astype(np.int32)


def graph_seed_grad_s(S: np.ndarray, row_ptr: np.ndarray, col_ind: np.ndarray, b: int,
                      dZ: np.ndarray) -> np.ndarray:
    """TEST INFRASTRUCTURE (the reference has no differentiation code): the
    gradient with respect to S of <dZ, Z(S)>, Z = graph_seed_dense(S, ...),
    under symmetric perturbations of S: for every row i, with
    M_i = U diag(w) U^T, E the rows of dZ at i's block placed in i's slot,
    D_i = U (F o (U^T E U)) U^T, F_kl = (f(w_k) - f(w_l)) / (w_k - w_l) for
    f(x) = x^-1/2 (f' on the diagonal); the symmetric parts of the D_i summed
    into a dense N x N result (entries outside S's pattern stay 0)."""
    n = row_ptr.size - 1
    G = np.zeros_like(S)
    for i in range(n):
        members = np.asarray(col_ind[row_ptr[i]:row_ptr[i + 1]])
        idx = (members[:, None] * b + np.arange(b)[None, :]).reshape(-1)
        slot = int(np.flatnonzero(members == i)[0])
        w, U = np.linalg.eigh(S[np.ix_(idx, idx)])
        f = 1.0 / np.sqrt(w)
        with np.errstate(divide="ignore", invalid="ignore"):
            F = (f[:, None] - f[None, :]) / (w[:, None] - w[None, :])
        close = np.abs(w[:, None] - w[None, :]) <= 1e-12 * np.abs(w).max()
        fp = -0.5 * w ** -1.5
        F = np.where(close, 0.5 * (fp[:, None] + fp[None, :]), F)
        E = np.zeros((idx.size, idx.size))
        E[slot * b:(slot + 1) * b, :] = dZ[i * b:(i + 1) * b, idx]
        D = U @ (F * (U.T @ E @ U)) @ U.T
        G[np.ix_(idx, idx)] += 0.5 * (D + D.T)
    return G


def ns_inverse_sqrt_dense(S: np.ndarray, tol: float = 1e-11, maxit: int = 60):
    """Dense FP64 restatement of rsatb::calc::inverse_sqrt's Newton-Schulz
    loop (rsatb/calc/isqrtm.hpp:613-700 and the residual of :370-405 on a
    dense matrix, ||X - I||_F): X = Z S Z^T, P = 1.875 I - 1.25 X +
    0.375 X^2, Z <- P Z, from Z0 = I / sqrt(max row sum |S|), while
    norm > tol, count < maxit and |norm_pre - norm| > 0.005 norm; a residual
    above 100 is a divergence.  Returns (Z, report dict)."""
    n = S.shape[0]
    s = np.abs(S).sum(axis=1).max()
    Z = np.eye(n) / np.sqrt(s)
    I = np.eye(n)

    def resid(Z):
        X = Z @ S @ Z.T
        return X, float(np.linalg.norm(X - I))

    X, norm = resid(Z)
    norm_pre, count, diverged = 0.0, 0, False
    while norm > tol and count < maxit and abs(norm_pre - norm) > 0.005 * norm:
        if norm > 100.0:
            diverged = True
            break
        norm_pre = norm
        P = 1.875 * I - 1.25 * X + 0.375 * X @ X
        Z = P @ Z
        count += 1
        X, norm = resid(Z)
    return Z, {"residual": norm, "iterations": count, "diverged": diverged,
               "converged": (not diverged) and norm <= tol,
               "hit_maxiter": (not diverged) and count >= maxit and norm > tol}


def spd_from_spectrum(lam: np.ndarray, seed: int) -> np.ndarray:
    """Q diag(lam) Q^T with Q from the QR of a seeded Gaussian matrix, the
    construction of the reference's isqrt benchmark problems
    (rsatb/calc/test/benchmark_isqrt_action.cpp:87-140)."""
    rng = np.random.default_rng(seed)
    n = lam.size
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    A = (Q * lam) @ Q.T
    return 0.5 * (A + A.T)


# ------------------------------------------------------- adjoint KPM (reference)

def kpm_plain_moments_dense(H: np.ndarray, psi: np.ndarray, center: float, half_width: float,
                            n_moments: int) -> np.ndarray:
    """mu_n = (1/R) sum_s psi_s^T T_n(A) psi_s, A = (H - c)/hw, dense FP64
    (Chebyshev::compute_moments, rsatb/calc/cheby.hpp:479-514, column-averaged)."""
    A = (H - center * np.eye(H.shape[0])) / half_width
    R = psi.shape[1]
    t0, t1 = psi, A @ psi
    mu = np.zeros(n_moments)
    for n in range(n_moments):
        if n == 0:
            t = t0
        elif n == 1:
            t = t1
        else:
            t0, t1 = t1, 2.0 * A @ t1 - t0
            t = t1
        mu[n] = float(np.sum(psi * t)) / R
    return mu


def kpm_moments_vjp_dense(H: np.ndarray, psi: np.ndarray, center: float, half_width: float,
                          n_moments: int, dmu: np.ndarray) -> np.ndarray:
    """Dense FP64 reference gradient d(sum_n dmu_n mu_n)/dH of the plain
    moments by reverse-mode differentiation of the three-term recurrence
    (TEST INFRASTRUCTURE; the reference has no differentiation code):
    lambda_n = (dmu_n/R) psi + 2 A lambda_{n+1} - lambda_{n+2},
    G = [lambda_1 t_0^T + 2 sum_{n>=1} lambda_{n+1} t_n^T] / hw."""
    N = H.shape[0]
    A = (H - center * np.eye(N)) / half_width
    R = psi.shape[1]
    M = n_moments
    t = [psi]
    if M > 1:
        t.append(A @ psi)
    for n in range(2, M):
        t.append(2.0 * A @ t[-1] - t[-2])
    lam = [np.zeros_like(psi)] * (M + 2)
    lam = list(lam)
    for n in range(M - 1, 0, -1):
        lam[n] = (dmu[n] / R) * psi + 2.0 * A @ lam[n + 1] - lam[n + 2]
    G = np.zeros((N, N))
    for n in range(0, M - 1):
        G += (1.0 if n == 0 else 2.0) * lam[n + 1] @ t[n].T
    return G / half_width


def kpm_moments_vjp_sparse(H, psi: np.ndarray, center: float, half_width: float,
                           n_moments: int, dmu: np.ndarray):
    """The same reverse-mode gradient with a scipy.sparse H (CSR, FP64),
    sampled on H's pattern: returns (mu, grad data aligned with H.data).
    All t_n are kept (no checkpoints): the CPU baseline of the adjoint."""
    import scipy.sparse as sp
    A = (H - center * sp.identity(H.shape[0], format="csr")) / half_width
    A = A.tocsr()
    R = psi.shape[1]
    M = n_moments
    t = [psi]
    if M > 1:
        t.append(A @ psi)
    for n in range(2, M):
        t.append(2.0 * (A @ t[-1]) - t[-2])
    mu = np.array([float(np.sum(psi * tn)) / R for tn in t])
    lam = [None] * (M + 2)
    z = np.zeros_like(psi)
    lam[M] = z
    lam[M + 1] = z
    for n in range(M - 1, 0, -1):
        lam[n] = (dmu[n] / R) * psi + 2.0 * (A @ lam[n + 1]) - lam[n + 2]
    Hc = H.tocsr()
    rows = np.repeat(np.arange(Hc.shape[0]), np.diff(Hc.indptr))
    cols = Hc.indices
    g = np.zeros(cols.size)
    for n in range(0, M - 1):
        w = 1.0 if n == 0 else 2.0
        g += w * np.einsum("ij,ij->i", lam[n + 1][rows], t[n][cols])
    return mu, g / half_width
