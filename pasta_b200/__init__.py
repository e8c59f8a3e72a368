"""pasta_b200: B200 (sm_100a) implementation of PASTA's per-particle
model-evaluation + chi2 hot path behind the reference's Python API.

``pasta_b200.pasta`` is the drop-in module (same names as the reference's
PyO3 module ``pasta``); ``include/pasta_b200.h`` is the C ABI underneath.
"""
from . import _ffi  # noqa: F401

__version__ = "0.1.0"


def library_path() -> str:
    return _ffi.LIB_PATH
