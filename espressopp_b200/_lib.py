"""Loads the CUDA library libespp_b200.so that sits next to this file.

There is no CPU fallback: if the library is missing or no CUDA device is visible the
calls fail with an error naming the cause.
"""
import ctypes
import os

from . import _abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "libespp_b200.so")
_lib = None


def load_library():
    """Returns the bound ctypes handle of libespp_b200.so (built in place if absent)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY_PATH):
            from . import build
            build.build()
        if not os.path.exists(LIBRARY_PATH):
            raise RuntimeError("libespp_b200.so is missing; run python -m espressopp_b200.build")
        _lib = _abi.bind(ctypes.CDLL(LIBRARY_PATH))
    return _lib
