"""CPU checks of the C ABI library: it builds, loads, and exports every
entry point include/alluvion_b200.h declares; host-side argument and device
checks return status codes instead of crashing (no GPU needed)."""
import ctypes
import os
import re

import pytest

from alluvion_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            names += re.findall(r"^AL_API\s+[\w\s\*]+?\b(al_\w+)\s*\(", text, re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = _capi.lib()
    declared = header_functions()
    assert declared, "no AL_API declarations found"
    for name in declared:
        assert hasattr(lib, name), name
    # the ctypes binding covers exactly the header
    assert set(_capi.declared_symbols()) == set(declared)


def test_status_strings():
    lib = _capi.lib()
    for code in _capi.STATUS:
        assert lib.al_status_string(code)


def test_engine_create_reports_missing_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    status = _capi.lib().al_engine_create(0, ctypes.byref(h))
    assert status == 8  # AL_ERR_NO_DEVICE
    assert not h.value
    assert _capi.lib().al_last_error()


def test_null_arguments_rejected():
    lib = _capi.lib()
    assert lib.al_grid_sort_f32(None, None, None, None, 0, None, None, None, None, None) == 2
    assert lib.al_engine_create(0, None) == 2
