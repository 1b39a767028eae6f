"""Device-resident stand-ins for the vbcsr types the hot path consumes.

vbcsr (DeepElectron/vbcsr, pinned 1d0dc39 by the reference's
CMakeLists.txt:389) provides ``BlockSpMat`` and ``DistMultiVector`` to
RSATB; it is not vendored, so this module defines the subset the KPM path
calls (rsatb/calc/cheby.hpp:599-606, dos.hpp:140-171), backed by the
rsatb_b200 C ABI.  Device memory comes from PyTorch (plumbing only): a
multivector is a CUDA tensor of shape (N, R), row-major like vbcsr's.
"""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np
import torch

from . import _capi
from ._capi import check, lib

_DT_CODE = {torch.float64: _capi.F64, torch.float32: _capi.F32,
            torch.complex128: _capi.C128, torch.complex64: _capi.C64}
_NP_OF_CODE = {_capi.F64: np.float64, _capi.F32: np.float32,
               _capi.C128: np.complex128, _capi.C64: np.complex64}


def dtype_code(t: torch.dtype) -> int:
    try:
        return _DT_CODE[t]
    except KeyError:
        raise TypeError(f"unsupported dtype {t}") from None


class Context:
    """One rsatb context per CUDA device, launching on torch's current stream."""

    _lock = threading.Lock()
    _by_device: dict[int, "Context"] = {}

    def __init__(self, device: int):
        h = C.c_void_p()
        check(lib().rsatb_ctx_create(device, C.byref(h)))
        self.handle = h
        self.device = device
        self._stream = None

    @classmethod
    def get(cls, device=None) -> "Context":
        if not torch.cuda.is_available():
            raise RuntimeError("rsatb_b200 needs a CUDA device (sm_100a); none is visible")
        dev = torch.cuda.current_device() if device is None else int(
            torch.device(device).index if isinstance(device, (str, torch.device)) else device)
        with cls._lock:
            ctx = cls._by_device.get(dev)
            if ctx is None:
                ctx = cls(dev)
                cls._by_device[dev] = ctx
        ctx.bind_stream()
        return ctx

    def bind_stream(self) -> None:
        # cuda_stream is 0 for torch's default stream, which the C ABI reads as
        # the legacy default stream: the same stream torch launches on.
        s = torch.cuda.current_stream(self.device).cuda_stream
        if s != self._stream:
            check(lib().rsatb_ctx_set_stream(self.handle, C.c_void_p(s)))
            self._stream = s

    def synchronize(self) -> None:
        check(lib().rsatb_ctx_synchronize(self.handle))

    def launch_count(self) -> int:
        return int(lib().rsatb_ctx_launch_count(self.handle))


def context(device=None) -> Context:
    return Context.get(device)


class BlockSpMat:
    """vbcsr BlockSpMat<T> with a uniform block size, resident on the GPU.

    ``values`` is (nnz_blocks, b, b) row-major blocks (real or complex).
    ``imaginary=True`` stores real values W for the matrix i*W (a velocity
    at a real k-point, V = i [H, x]).  Move-only in spirit: the handle is
    released when the object is collected.
    """

    def __init__(self, row_ptr, col_ind, values, block_size: int, n_block_cols: int | None = None,
                 dtype=None, imaginary: bool = False, device=None, _handle=None):
        self.ctx = context(device)
        if _handle is not None:
            self.handle = _handle
            self._read_info()
            return
        row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
        col_ind = np.ascontiguousarray(col_ind, dtype=np.int32)
        vals = np.asarray(values)
        if dtype is None:
            dtype = np.complex128 if np.iscomplexobj(vals) else np.float64
        vals = np.ascontiguousarray(vals, dtype=dtype)
        code = {np.dtype(np.float64): _capi.F64, np.dtype(np.float32): _capi.F32,
                np.dtype(np.complex128): _capi.C128, np.dtype(np.complex64): _capi.C64}[vals.dtype]
        nbr = row_ptr.size - 1
        nbc = nbr if n_block_cols is None else int(n_block_cols)
        h = C.c_void_p()
        flags = _capi.BSR_IMAGINARY_UNIT if imaginary else 0
        check(lib().rsatb_bsr_create(self.ctx.handle, nbr, nbc, int(block_size), col_ind.size,
                                     row_ptr.ctypes.data, col_ind.ctypes.data, vals.ctypes.data,
                                     code, flags, C.byref(h)))
        self.handle = h
        self._read_info()

    def _read_info(self):
        nbr, nbc, b = C.c_int(), C.c_int(), C.c_int()
        nnz, dt, fl = C.c_int64(), C.c_int(), C.c_uint()
        check(lib().rsatb_bsr_info(self.handle, C.byref(nbr), C.byref(nbc), C.byref(b),
                                   C.byref(nnz), C.byref(dt), C.byref(fl)))
        self.n_block_rows, self.n_block_cols, self.block_size = nbr.value, nbc.value, b.value
        self.nnz_blocks, self.dtype_code, self.flags = nnz.value, dt.value, fl.value

    @property
    def shape(self):
        return (self.n_block_rows * self.block_size, self.n_block_cols * self.block_size)

    @property
    def imaginary(self) -> bool:
        return bool(self.flags & _capi.BSR_IMAGINARY_UNIT)

    @property
    def is_double(self) -> bool:
        return self.dtype_code in (_capi.F64, _capi.C128)

    @property
    def is_complex(self) -> bool:
        return self.dtype_code in (_capi.C128, _capi.C64)

    def value_bytes(self) -> int:
        return self.nnz_blocks * self.block_size ** 2 * np.dtype(_NP_OF_CODE[self.dtype_code]).itemsize

    def index_bytes(self) -> int:
        return 4 * (self.n_block_rows + 1 + self.nnz_blocks)

    def adjoint(self) -> "BlockSpMat":
        """A^H as a new matrix (the operator of mult_dense_adjoint)."""
        h = C.c_void_p()
        check(lib().rsatb_bsr_adjoint(self.ctx.handle, self.handle, C.byref(h)))
        return BlockSpMat(None, None, None, 0, device=self.ctx.device, _handle=h)

    def astype(self, precision: str) -> "BlockSpMat":
        """'f64' or 'f32' copy (complex stays complex)."""
        if precision == "f64":
            code = _capi.C128 if self.is_complex else _capi.F64
        elif precision == "f32":
            code = _capi.C64 if self.is_complex else _capi.F32
        else:
            raise ValueError(precision)
        h = C.c_void_p()
        check(lib().rsatb_bsr_convert(self.ctx.handle, self.handle, code, C.byref(h)))
        return BlockSpMat(None, None, None, 0, device=self.ctx.device, _handle=h)

    def values_tensor(self) -> torch.Tensor:
        """A view of the device values (nnz_blocks, b, b) as a torch tensor (copy)."""
        n = self.nnz_blocks * self.block_size ** 2
        dt = {_capi.F64: torch.float64, _capi.F32: torch.float32,
              _capi.C128: torch.complex128, _capi.C64: torch.complex64}[self.dtype_code]
        out = torch.empty(n, dtype=dt, device=f"cuda:{self.ctx.device}")
        self.ctx.bind_stream()
        src = lib().rsatb_bsr_values(self.handle)
        nbytes = out.numel() * out.element_size()
        check(lib().rsatb_copy_to_device(self.ctx.handle, C.c_void_p(out.data_ptr()),
                                         C.c_void_p(src), nbytes))
        return out.view(self.nnz_blocks, self.block_size, self.block_size)

    def to_arrays(self):
        """The matrix on the host as lattice.BsrArrays (row_ptr, col_ind and
        values (nnz_blocks, b, b) copied from the device)."""
        from .lattice import BsrArrays
        rp = np.zeros(self.n_block_rows + 1, dtype=np.int32)
        ci = np.zeros(max(self.nnz_blocks, 1), dtype=np.int32)
        check(lib().rsatb_bsr_pattern(self.ctx.handle, self.handle, rp.ctypes.data,
                                      ci.ctypes.data))
        vals = self.values_tensor().cpu().numpy()
        return BsrArrays(rp, ci[:self.nnz_blocks], vals, self.block_size, self.n_block_cols)

    def set_values(self, values: torch.Tensor) -> None:
        """Overwrites the block values from a device tensor of matching size."""
        v = values.contiguous()
        if v.numel() != self.nnz_blocks * self.block_size ** 2 or dtype_code(v.dtype) != self.dtype_code:
            raise ValueError("set_values: size or dtype mismatch")
        self.ctx.bind_stream()
        check(lib().rsatb_bsr_set_values(self.ctx.handle, self.handle, C.c_void_p(v.data_ptr()),
                                         _capi.BSR_DEVICE_POINTERS))
        self._adj = None

    def mult_dense(self, X: torch.Tensor, Y: torch.Tensor, alpha: float = 1.0) -> torch.Tensor:
        """Y = alpha * A X (vbcsr BlockSpMat::mult_dense)."""
        _check_panel(X, self.shape[1])
        _check_panel(Y, self.shape[0])
        if X.dtype != Y.dtype:
            raise TypeError("X and Y dtypes differ")
        self.ctx.bind_stream()
        check(lib().rsatb_bsr_mult_dense(self.ctx.handle, self.handle, C.c_void_p(X.data_ptr()),
                                         C.c_void_p(Y.data_ptr()), X.shape[1],
                                         dtype_code(X.dtype), float(alpha)))
        return Y

    def mult(self, x: torch.Tensor, y: torch.Tensor, alpha: float = 1.0) -> torch.Tensor:
        """y = alpha * A x for one vector (N,) (vbcsr BlockSpMat::mult)."""
        self.mult_dense(x.reshape(-1, 1), y.reshape(-1, 1), alpha)
        return y

    def mult_optimized(self, X: torch.Tensor, Y: torch.Tensor) -> torch.Tensor:
        """Y = A X; the device path is the same fused kernel as mult_dense."""
        return self.mult_dense(X, Y)

    def _adjoint_cached(self) -> "BlockSpMat":
        adj = getattr(self, "_adj", None)
        if adj is None:
            adj = self.adjoint()
            self._adj = adj
        return adj

    def mult_dense_adjoint(self, X: torch.Tensor, Y: torch.Tensor,
                           alpha: float = 1.0) -> torch.Tensor:
        """Y = alpha * A^H X (vbcsr BlockSpMat::mult_dense_adjoint); A^H is built
        once and kept (invalidated by set_values)."""
        return self._adjoint_cached().mult_dense(X, Y, alpha)

    def mult_adjoint(self, x: torch.Tensor, y: torch.Tensor, alpha: float = 1.0) -> torch.Tensor:
        """y = alpha * A^H x for one vector."""
        self._adjoint_cached().mult_dense(x.reshape(-1, 1), y.reshape(-1, 1), alpha)
        return y

    def duplicate(self) -> "BlockSpMat":
        """An independent copy (same precision)."""
        return self.astype("f64" if self.is_double else "f32")

    def get_block_density(self) -> float:
        """Stored blocks over all block positions."""
        return self.nnz_blocks / float(max(1, self.n_block_rows * self.n_block_cols))

    def block_size_elements(self) -> int:
        return self.block_size * self.block_size

    def __del__(self):
        h = getattr(self, "handle", None)
        if h and _capi._lib is not None:
            try:
                torch.cuda.current_stream(self.ctx.device).synchronize()
                lib().rsatb_bsr_destroy(h)
            except Exception:
                pass
            self.handle = None


def _check_panel(X: torch.Tensor, n_rows: int) -> None:
    if not X.is_cuda or X.dim() != 2 or not X.is_contiguous():
        raise ValueError("multivectors are contiguous 2-D CUDA tensors (N, R)")
    if X.shape[0] != n_rows:
        raise ValueError(f"multivector has {X.shape[0]} rows, operator expects {n_rows}")
    dtype_code(X.dtype)


class DistMultiVector:
    """vbcsr DistMultiVector<T>: N x R row-major panel on the GPU."""

    def __init__(self, n_rows: int, num_vectors: int, dtype=torch.complex128, device=None,
                 data: torch.Tensor | None = None):
        ctx = context(device)
        if data is None:
            data = torch.zeros(n_rows, num_vectors, dtype=dtype, device=f"cuda:{ctx.device}")
        self.data = data
        self.ctx = ctx

    @property
    def num_vectors(self) -> int:
        return self.data.shape[1]

    @property
    def local_rows(self) -> int:
        return self.data.shape[0]

    def set_random(self, seed: int, normalize: bool = True, atom_index=None,
                   orbitals_per_atom: int = 1, kind: int | None = None,
                   n_rows_global: int | None = None, first_column: int = 0) -> "DistMultiVector":
        """Seeded sample vectors (SampleVectors::initialize); see rsatb_set_random."""
        set_random(self.data, seed, normalize=normalize, atom_index=atom_index,
                   orbitals_per_atom=orbitals_per_atom, kind=kind, n_rows_global=n_rows_global,
                   first_column=first_column)
        return self

    def dot(self, other: "DistMultiVector") -> np.ndarray:
        """Per-column <self|other> (conjugate-linear in self), FP64."""
        a = self.data.to(torch.complex128)
        b = other.data.to(torch.complex128)
        return (a.conj() * b).sum(0).cpu().numpy()

    def copy_from(self, other: "DistMultiVector") -> None:
        self.data.copy_(other.data)

    def axpby(self, a, x: "DistMultiVector", b) -> None:
        """self = a * x + b * self."""
        self.data.mul_(b).add_(x.data, alpha=a)

    def scale(self, s) -> None:
        self.data.mul_(s)

    def axpy(self, a, x: "DistMultiVector") -> None:
        """self += a * x."""
        self.data.add_(x.data, alpha=a)

    def bdot(self, other: "DistMultiVector") -> np.ndarray:
        """Per-column bilinear sum_i self_i other_i (no conjugation), FP64."""
        a = self.data.to(torch.complex128)
        b = other.data.to(torch.complex128)
        return (a * b).sum(0).cpu().numpy()

    def swap(self, other: "DistMultiVector") -> None:
        """Exchanges the two panels (no copy)."""
        self.data, other.data = other.data, self.data

    def set_constant(self, value) -> None:
        self.data.fill_(value)

    def get_col(self, j: int) -> torch.Tensor:
        """Column j as a new (N,) device tensor."""
        return self.data[:, j].clone()

    def set_col(self, j: int, v: torch.Tensor) -> None:
        self.data[:, j].copy_(v)

    def row_data(self, row: int) -> torch.Tensor:
        """Row `row` of the panel (a view)."""
        return self.data[row]

    def __call__(self, row: int, col: int):
        return self.data[row, col].item()


def set_random(out: torch.Tensor, seed: int, normalize: bool = True, atom_index=None,
               orbitals_per_atom: int = 1, kind: int | None = None,
               n_rows_global: int | None = None, first_column: int = 0) -> torch.Tensor:
    """Fills the (N, R) tensor with seeded sample vectors (Philox-4x32-10).

    kind: RANDOM_PHASE (complex default), RANDOM_RADEMACHER (real default)
    or RANDOM_UNIFORM.  atom_index: stable ids of the N/orbitals_per_atom
    atoms, default 0..n_atoms-1.
    """
    if not out.is_cuda or out.dim() != 2 or not out.is_contiguous():
        raise ValueError("set_random needs a contiguous (N, R) CUDA tensor")
    ctx = context(out.device)
    n_rows, R = out.shape
    if n_rows % orbitals_per_atom:
        raise ValueError("rows are not a whole number of atoms")
    n_atoms = n_rows // orbitals_per_atom
    ids = np.arange(n_atoms, dtype=np.int64) if atom_index is None else np.ascontiguousarray(
        atom_index, dtype=np.int64)
    if ids.size != n_atoms:
        raise ValueError("atom_index length differs from the atom count")
    if kind is None:
        kind = _capi.RANDOM_PHASE if out.is_complex() else _capi.RANDOM_RADEMACHER
    check(lib().rsatb_set_random(ctx.handle, C.c_uint64(seed), int(kind), int(normalize),
                                 ids.ctypes.data, n_atoms, orbitals_per_atom,
                                 int(n_rows_global if n_rows_global else n_rows), R,
                                 int(first_column), dtype_code(out.dtype),
                                 C.c_void_p(out.data_ptr())))
    # ids is host memory read by a stream-ordered copy: wait for it.
    ctx.synchronize()
    return out
