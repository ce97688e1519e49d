"""B200 replacement of MFIX's linear-equation hot path (SOLVE_LIN_EQ -> LEQ_BICGS).

The product is the CUDA library ``libmfixgpu.so`` behind the C ABI of
``include/mfixgpu.h``; this package loads it and mirrors the reference's
Fortran interface in Python (:mod:`mfix_b200.leq`).  There is no CPU fallback:
if the library is missing or no GPU is visible, calls fail loudly.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmfixgpu.so")
_lib = None


def lib() -> ctypes.CDLL:
    """The loaded CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m mfix_b200.build` (no CPU fallback exists)")
        _lib = ctypes.CDLL(LIB_PATH)
        from . import leq as _leq

        _leq._declare(_lib)
    return _lib


__all__ = ["lib", "LIB_PATH"]
