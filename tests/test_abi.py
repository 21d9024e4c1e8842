"""The C-ABI library loads without a GPU and exports every entry point of include/mdft_b200.h."""
import ctypes
import os
import re

import pytest

from mdft_b200 import engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "mdft_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*(mdft_\w+)\s*\(", text, re.M)))


def test_header_and_binding_agree():
    assert declared_functions() == sorted(engine.SIGNATURES)


def test_library_exports_every_symbol():
    if not os.path.exists(engine.library_path()):
        pytest.fail("libmdft_b200.so not built")
    L = ctypes.CDLL(engine.library_path())
    for name in declared_functions():
        assert hasattr(L, name), name


def test_argument_errors_without_gpu():
    L = engine.lib()
    d = engine._Desc(15, 16, 16, 8.0, 8.0, 8.0, 1, 2, 298.0, 0.0333, b"/nonexistent", 0, 0)
    h = ctypes.c_void_p()
    assert L.mdft_create(ctypes.byref(d), ctypes.byref(h)) == -1
    assert b"even" in L.mdft_last_error()
    d = engine._Desc(16, 16, 16, 8.0, 8.0, 8.0, 7, 2, 298.0, 0.0333, b"/nonexistent", 0, 0)
    assert L.mdft_create(ctypes.byref(d), ctypes.byref(h)) == -1
    d = engine._Desc(16, 16, 16, 8.0, 8.0, 8.0, 1, 2, 298.0, 0.0333, b"/nonexistent/ck", 0, 0)
    assert L.mdft_create(ctypes.byref(d), ctypes.byref(h)) == -2
    assert b"cannot open" in L.mdft_last_error()
    assert L.mdft_destroy(None) == 0
