"""The allocation-free KPM entry point, rsatb_kpm_dos_moments_noalloc.

It exists for callers that cannot allocate device memory (a process whose
device memory is all reserved by another allocator, or a loop that must not
take cudaMalloc's device-wide synchronisation): it keeps every temporary in a
fixed 32 MiB static device array.  This file checks, through the C ABI,
that two calls in a row give the same moments as rsatb_kpm_dos_moments
(within the 1e-10 moment tolerance of the other KPM tests), that the first
call ever made on a new context takes no device memory (the context has not
allocated its counters or scratch yet, which is the case the entry point is
for), that a bounded wait that gives up fails the call instead of returning
wrong moments, and that a problem too large for the array is refused.  It
is collected last so that a failure here never hides the other tests, and
it builds everything it needs itself, so it also passes alone in a fresh
process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10  # relative to mu_0, as in tests/test_kpm_gpu.py


def _moments(fn, ctx, op, psi, dtype_code, n_moments, doubled):
    mu = np.zeros(2 * n_moments)
    col = np.zeros(2 * n_moments * psi.shape[1])
    P = C.POINTER(C.c_double)
    st = fn(ctx.handle, C.byref(op), C.c_void_p(psi.data_ptr()), psi.shape[1], dtype_code,
            n_moments, int(doubled), mu.ctypes.data_as(P), col.ctypes.data_as(P))
    return st, mu.view(np.complex128), col.view(np.complex128)


def _operators():
    """(name, Chebyshev, psi) cases: orthogonal graphene with complex phases
    and sandwich diamond with real Rademacher vectors."""
    import torch
    from rsatb_b200 import lattice
    from rsatb_b200.calc import Chebyshev, ISQRTMPreconditioner
    from rsatb_b200.isqrt import graph_inverse_sqrt_host
    from rsatb_b200.vbcsr import BlockSpMat, set_random
    H, _, _ = lattice.graphene(12, 12)
    g = Chebyshev(BlockSpMat(H.row_ptr, H.col_ind, H.values, 1), -8.7, 8.7)
    psi_g = torch.empty(H.n_rows, 8, dtype=torch.complex128, device="cuda")
    set_random(psi_g, 20240917)
    Hd, S = lattice.diamond_lcao(L=2, seed=3)
    Z = graph_inverse_sqrt_host(S)
    pre = ISQRTMPreconditioner(BlockSpMat(Z.row_ptr, Z.col_ind, Z.values, 8))
    d = Chebyshev(BlockSpMat(Hd.row_ptr, Hd.col_ind, Hd.values, 8), -14.0, 14.0,
                  preconditioner=pre)
    psi_d = torch.empty(Hd.n_rows, 16, dtype=torch.float64, device="cuda")
    set_random(psi_d, 7, orbitals_per_atom=8)
    return [("graphene", g, psi_g), ("diamond-sandwich", d, psi_d),
            ("diamond-sandwich-f32", d.astype("f32"), psi_d.to(torch.float32))]


def test_noalloc_matches_allocating_entry_point_twice():
    from rsatb_b200 import _capi
    from rsatb_b200.vbcsr import context, dtype_code
    ctx = context()
    lib = _capi.lib()
    for name, cheby, psi in _operators():
        op = cheby.c_op()
        code = dtype_code(psi.dtype)
        for doubled in (True, False):
            st, want, want_col = _moments(lib.rsatb_kpm_dos_moments, ctx, op, psi, code, 96,
                                          doubled)
            assert st == 0, lib.rsatb_last_error()
            for call in range(2):  # the array keeps the previous call's contents
                st, got, got_col = _moments(lib.rsatb_kpm_dos_moments_noalloc, ctx, op, psi,
                                            code, 96, doubled)
                assert st == 0, lib.rsatb_last_error()
                scale = np.abs(want).max()
                assert np.abs(got - want).max() <= TOL * scale, (name, doubled, call)
                assert np.abs(got_col - want_col).max() <= TOL * scale, (name, doubled, call)


def test_noalloc_refuses_problems_beyond_its_array():
    import torch
    from rsatb_b200 import _capi
    from rsatb_b200 import lattice
    from rsatb_b200.calc import Chebyshev
    from rsatb_b200.vbcsr import BlockSpMat, context, dtype_code, set_random
    ctx = context()
    H, _, _ = lattice.graphene(60, 60)  # 7,200 rows
    cheby = Chebyshev(BlockSpMat(H.row_ptr, H.col_ind, H.values, 1), -8.7, 8.7)
    psi = torch.empty(H.n_rows, 256, dtype=torch.complex128, device="cuda")  # 3 x 29 MB panels
    set_random(psi, 1)
    st, _, _ = _moments(_capi.lib().rsatb_kpm_dos_moments_noalloc, ctx, cheby.c_op(), psi,
                        dtype_code(psi.dtype), 16, True)
    assert st == 1  # RSATB_INVALID_ARGUMENT
    assert b"32 MiB" in _capi.lib().rsatb_last_error()


def test_noalloc_first_call_on_a_fresh_context_takes_no_device_memory():
    """A caller whose device memory belongs to another allocator makes its
    first call on a context that has allocated nothing yet.  The call must
    not allocate either: the free device memory is the same before and after
    it, and the moments equal the allocating entry point's."""
    import torch
    from rsatb_b200 import _capi
    from rsatb_b200.vbcsr import Context, context, dtype_code
    lib = _capi.lib()
    cases = _operators()
    # Load the library's modules and the static array once (the first call
    # on a device reserves it), on the shared context.
    for _, cheby, psi in cases:
        st, _, _ = _moments(lib.rsatb_kpm_dos_moments_noalloc, context(), cheby.c_op(), psi,
                            dtype_code(psi.dtype), 64, True)
        assert st == 0, lib.rsatb_last_error()
    for name, cheby, psi in cases:
        fresh = Context(torch.cuda.current_device())
        try:
            fresh.bind_stream()
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info()[0]
            st, got, _ = _moments(lib.rsatb_kpm_dos_moments_noalloc, fresh, cheby.c_op(), psi,
                                  dtype_code(psi.dtype), 64, True)
            torch.cuda.synchronize()
            free1 = torch.cuda.mem_get_info()[0]
            assert st == 0, lib.rsatb_last_error()
            assert free1 == free0, (name, free0 - free1)
        finally:
            lib.rsatb_ctx_destroy(fresh.handle)
        st, want, _ = _moments(lib.rsatb_kpm_dos_moments, context(), cheby.c_op(), psi,
                               dtype_code(psi.dtype), 64, True)
        assert st == 0, lib.rsatb_last_error()
        assert np.abs(got - want).max() <= TOL * np.abs(want).max(), name


def test_noalloc_reports_a_bounded_wait_that_gave_up(monkeypatch):
    """The bulk-copy step kernel's bounded wait, armed for bytes no copy
    delivers (a 5 ms limit, no copy issued), sets the fault word in the
    static array's header; the call then fails with RSATB_CUDA_ERROR instead
    of returning its moments, and the next call is correct again."""
    from rsatb_b200 import _capi
    from rsatb_b200.vbcsr import context, dtype_code
    lib = _capi.lib()
    name, cheby, psi = _operators()[2]  # FP32 sandwich, 8x8 blocks, W = 16
    op = cheby.c_op()
    code = dtype_code(psi.dtype)
    monkeypatch.setenv("RSATB_STEP_KERNEL", "bulk")
    monkeypatch.setenv("RSATB_TEST_BULK_WAIT", "1")
    st, _, _ = _moments(lib.rsatb_kpm_dos_moments_noalloc, context(), op, psi, code, 32, True)
    assert st == 16, (st, lib.rsatb_last_error())  # RSATB_CUDA_ERROR
    assert b"bounded wait" in lib.rsatb_last_error()
    monkeypatch.delenv("RSATB_TEST_BULK_WAIT")
    monkeypatch.delenv("RSATB_STEP_KERNEL")
    st, got, _ = _moments(lib.rsatb_kpm_dos_moments_noalloc, context(), op, psi, code, 32, True)
    assert st == 0, lib.rsatb_last_error()
    st, want, _ = _moments(lib.rsatb_kpm_dos_moments, context(), op, psi, code, 32, True)
    assert st == 0, lib.rsatb_last_error()
    assert np.abs(got - want).max() <= 1e-6 * np.abs(want).max(), name
