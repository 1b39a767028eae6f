"""The C ABI: the library loads and exports every function include/*.h
declares (CPU), and reports bad arguments as status codes (GPU)."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_functions() -> list[str]:
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*[A-Za-z_][\w\s\*]*?\b(rsatb_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "rsatb_kpm_dos_moments" in names and "rsatb_last_error" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    from rsatb_b200 import _capi
    lib = C.CDLL(str(_capi.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_binding_covers_header():
    from rsatb_b200 import _capi
    assert set(declared_functions()) <= set(_capi.exported_symbols())


def test_no_device_entry_point_needs_a_gpu_to_load():
    """Loading and querying the version works without a GPU."""
    from rsatb_b200 import _capi
    assert _capi.lib().rsatb_version() >= 100
    assert _capi.lib().rsatb_last_error() is not None


@pytest.mark.gpu
def test_invalid_arguments_are_status_codes():
    import torch
    from rsatb_b200 import _capi
    from rsatb_b200.vbcsr import BlockSpMat, context
    ctx = context()
    lib = _capi.lib()
    h = C.c_void_p()
    # column out of range (arrays kept alive across the call)
    ptr = np.array([0, 1, 2], np.int32)
    ind = np.array([0, 5], np.int32)
    vals = np.ones(2)
    st = lib.rsatb_bsr_create(ctx.handle, 2, 2, 1, 2, ptr.ctypes.data, ind.ctypes.data,
                              vals.ctypes.data, _capi.F64, 0, C.byref(h))
    assert st == 1 and b"out of range" in lib.rsatb_last_error()
    A = BlockSpMat([0, 1, 2], [0, 1], np.ones((2, 1, 1)), 1)
    X = torch.ones(2, 3, dtype=torch.float64, device="cuda")
    with pytest.raises(_capi.RsatbError, match="InvalidArgument"):
        A.mult_dense(X, X)  # in place
    Y = torch.ones(2, 3, dtype=torch.float32, device="cuda")
    with pytest.raises(_capi.RsatbError, match="precision"):
        lib_st = lib.rsatb_bsr_mult_dense(ctx.handle, A.handle, C.c_void_p(Y.data_ptr()),
                                          C.c_void_p(Y.data_ptr() + 0), 3, _capi.F32, 1.0)
        _capi.check(lib_st)
    op = _capi.ChebOp(_capi.FORM_ORTHOGONAL, A.handle, None, None, 0.0, 0.0)
    mu = np.zeros(8)
    st = lib.rsatb_kpm_dos_moments(ctx.handle, C.byref(op), C.c_void_p(X.data_ptr()), 3,
                                   _capi.F64, 4, 1,
                                   mu.ctypes.data_as(C.POINTER(C.c_double)), None)
    assert st == 1 and b"half_width" in lib.rsatb_last_error()
    op.form = 7
    op.half_width = 1.0
    st = lib.rsatb_kpm_dos_moments(ctx.handle, C.byref(op), C.c_void_p(X.data_ptr()), 3,
                                   _capi.F64, 4, 1,
                                   mu.ctypes.data_as(C.POINTER(C.c_double)), None)
    assert st == 18  # NotSupported


def _ctx_first_functions() -> list[str]:
    """Entry points returning a status whose first parameter is the context."""
    text = "".join(h.read_text() for h in sorted((ROOT / "include").glob("*.h")))
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\bint\s+(rsatb_\w+)\s*\(\s*rsatb_ctx_t\s+ctx\b", text)))


def test_null_context_is_a_status_code_everywhere():
    """Every entry point taking a context refuses a null one with
    RSATB_INVALID_ARGUMENT and a message, before touching any other argument
    (no GPU involved); destroying a null context is a no-op."""
    from rsatb_b200 import _capi
    lib = _capi.lib()
    names = [n for n in _ctx_first_functions() if n != "rsatb_ctx_destroy"]
    assert len(names) >= 25
    for name in names:
        fn = getattr(lib, name)
        args = [None]
        for t in fn.argtypes[1:]:
            is_pointer = (t is C.c_void_p or t is C.c_char_p
                          or (isinstance(t, type) and issubclass(t, C._Pointer)))
            args.append(None if is_pointer else t(0))
        assert fn(*args) == 1, name   # RSATB_INVALID_ARGUMENT
        assert b"null context" in lib.rsatb_last_error(), name
    assert lib.rsatb_ctx_destroy(None) == 0
