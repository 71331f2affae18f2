"""Host-side checks of the C ABI that need no GPU: the library loads, exports every entry point
declared in include/mmb200.h, validates its arguments before touching the device, and its pure
host logic (padding rules) matches the reference."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "mmb200.h")).read()
    return sorted(set(re.findall(r"MM_API\s+[\w\s\*]+?\b(mm_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def L():
    from micromagnum_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        _lib.build()
    return _lib.lib()


def test_exports_every_declared_symbol(L):
    from micromagnum_b200 import _lib
    names = declared_symbols()
    assert len(names) >= 30
    for name in names:
        assert hasattr(L, name), name
    # the Python binding covers the same set
    assert sorted(_lib.EXPORTED) == names


def test_abi_version(L):
    assert L.mm_abi_version() == 1


def test_invalid_arguments_rejected_on_host(L):
    from micromagnum_b200 import _lib
    st = L.mm_exchange(0, 0, 4, 4, 1e-9, 1e-9, 1e-9, 0, 0, 0, None, None, None, None, None, None)
    assert st == 1
    assert b"invalid" in L.mm_last_error()
    assert L.mm_llge(7, 10, None, None, None, None, None, None) == 1
    h = ctypes.c_void_p()
    cfg = _lib.mm_solver_config()
    cfg.nx, cfg.ny, cfg.nz = 4, 4, 1
    cfg.dx = cfg.dy = cfg.dz = 1e-9
    cfg.eps_abs = cfg.eps_rel = cfg.h0 = 0.0  # invalid tolerances
    mat = (_lib.mm_material * 1)()
    assert L.mm_solver_create(ctypes.byref(h), ctypes.byref(cfg), 1, mat, None, None, None) == 1
    assert L.mm_solver_create(ctypes.byref(h), ctypes.byref(cfg), 300, mat, None, None, None) == 1
    assert L.mm_demag_tensor(4, 4, 4, 1e-9, 1e-9, 1e-9, 4, 4, 4, None, None) == 1
    assert L.mm_demag_tensor(4, 4, 4, 1e-9, 1e-9, 1e-9, 4, 8, 8, ctypes.c_void_p(1), None) == 4  # periodic


@pytest.mark.parametrize("padding", range(6))
def test_round_tensor_dimension_matches_reference(L, oracle_mod, ref_available, padding):
    dims = list(range(1, 130)) + [200, 256, 511, 512, 1024]
    for d in dims:
        ours = L.mm_round_tensor_dimension(d, 0, padding)
        assert ours == oracle_mod.round_tensor_dimension(d, False, padding)
        if ref_available:
            assert ours == oracle_mod.reference().mmref_round_tensor_dimension(d, 0, padding)
        assert L.mm_round_tensor_dimension(d, 1, padding) == d
