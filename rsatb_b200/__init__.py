"""rsatb_b200: RSATB's KPM / S^-1/2 / FFT-Chebyshev hot path on NVIDIA B200.

The numerical work runs in the sm_100a CUDA library behind the C ABI of
``include/rsatb_b200.h`` (built in-tree by ``python -m rsatb_b200.build``);
the Python modules mirror the reference's calc-layer API over it.
"""
from ._capi import RsatbError, LIB_PATH  # noqa: F401

__all__ = ["RsatbError", "LIB_PATH"]


def native_library():
    """Loads the CUDA library; raises if it is not built."""
    from . import _capi
    return _capi.lib()
