"""Loader for the in-tree CUDA library.  There is no CPU fallback: a missing
or unloadable library raises."""
from __future__ import annotations

import ctypes
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libsifv_b200.so")
_lib = None


def load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"CUDA library {LIB_PATH} is not built; run `python -m semiimplicitfv_b200.build`")
        _lib = ctypes.CDLL(LIB_PATH)
    return _lib
