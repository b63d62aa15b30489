"""The CUDA library loads without a GPU and exports every entry point of the header."""
import os
import re

import pytest

import espressopp_b200
from espressopp_b200 import _abi

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_symbols():
    with open(os.path.join(REPO, "include", "espp_b200.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"ESPP_API\s+\w+\s+(espp_\w+)\s*\(", text)))


def test_header_declares_all_bound_prototypes():
    syms = _header_symbols()
    assert len(syms) >= 30
    assert set(_abi.PROTOTYPES) <= set(syms)


def test_library_exports_every_header_symbol():
    lib = espressopp_b200.load_library()
    for name in _header_symbols():
        assert hasattr(lib, name), name
    assert lib.espp_abi_version() == 1


def test_error_path_without_device_or_bad_args():
    import ctypes
    import numpy as np
    lib = espressopp_b200.load_library()
    h = ctypes.c_void_p()
    box = np.array([10.0, 10.0, 10.0])
    cg = np.array([0, 3, 3], np.int32)
    rc = lib.espp_system_create(_abi.dptr(box), 0.3, _abi.i32ptr(cg), 0, 1, ctypes.byref(h))
    assert rc != 0
    assert "cell grid" in _abi.last_error(lib)
