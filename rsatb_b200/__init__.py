"""rsatb_b200: RSATB's KPM / S^-1/2 / FFT-Chebyshev hot path on NVIDIA B200.

The numerical work runs in the sm_100a CUDA library behind the C ABI of
``include/rsatb_b200.h`` (built in-tree by ``python -m rsatb_b200.build``);
the Python modules mirror the reference's calc-layer API over it.  Importing
the package loads nothing: the library is opened by the first module that
calls into it, so the numpy-only modules (``lattice``) can be used on a host
without the library or a GPU.
"""

__all__ = ["RsatbError", "LIB_PATH"]


def __getattr__(name):
    if name in ("RsatbError", "LIB_PATH"):
        from . import _capi
        return getattr(_capi, name)
    raise AttributeError(f"module 'rsatb_b200' has no attribute {name!r}")


def native_library():
    """Loads the CUDA library; raises if it is not built."""
    from . import _capi
    return _capi.lib()
